"""Served form: every request's diff is the same alone, in the mix and in the oracle.

Clients' requests go through the continuous-batching loop (several batches in flight, requests
joining whichever batch launches next) and, separately, through one handle per client that
checkpoints the same buffers one at a time.  Diff checksums must be identical request by request,
and equal to the checksum of the oracle's diff of the same client's buffers (the oracle
checkpoints each client's snapshots in order, as a baseline wherever the loop ran one, on a fresh
deduplicator wherever the loop moved the client to a fresh handle).
"""
import hashlib

import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import ListDeduplicator, TreeDeduplicator, synth
from reproducibility_icpp23_scalable_gpu_deduplication_b200.serve import CheckpointServer, percentile
from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import estimate_memory, parse_header

pytestmark = pytest.mark.gpu

SIZES = [1 << 20, (3 << 20) + 77, 200, 5 << 20, 64 << 10, (2 << 20) + 4096]


def drive(server, sizes, rounds, order_seed=1, snapshots=None):
    """Submit `rounds` requests per client in a shuffled interleaving, stepping the loop between.
    With `snapshots` (a dict), a host copy of every submitted buffer is kept under (client, k)."""
    import numpy as np

    series = [synth.DeviceSeries(n, 128, c, max_run=64) for c, n in enumerate(sizes)]
    order = [c for c in range(len(sizes)) for _ in range(rounds)]
    np.random.default_rng(order_seed).shuffle(order)
    reqs = {}
    count = [0] * len(sizes)
    for i, c in enumerate(order):
        while server.busy(c):
            server.step()
        buf = series[c].next()
        if snapshots is not None:
            snapshots[(c, count[c])] = buf.cpu().numpy().copy()
        reqs[(c, count[c])] = server.submit(c, buf)
        count[c] += 1
        if i % 3 == 2:          # requests arrive in small bursts: several join one batch
            server.step()
    server.drain()
    return reqs


def host_checksum(diff, block=4096):
    """TreeDeduplicator.diff_checksum of a host diff: MD5 over the Murmur3 digests of its
    `block`-byte blocks (the last one short) and its length"""
    n = len(diff)
    digests = b"".join(O.hash_bytes(diff[i:i + block], O.HASH_MURMUR3) for i in range(0, n, block))
    return hashlib.md5(digests + n.to_bytes(8, "little")).hexdigest()


def check_with_oracle(reqs, snapshots, approach="tree"):
    """every completed request's diff checksum equals the oracle's for the same client history"""
    Oracle = O.OracleListDeduplicator if approach == "list" else O.OracleTreeDeduplicator
    for c in sorted({c for c, _ in reqs}):
        o, k = None, 0
        while (c, k) in reqs:
            r = reqs[(c, k)]
            assert r.rc == 0 and r.checksum is not None, (c, k)
            if o is None or r.chkpt_id == 0:       # the loop gave the client a fresh handle
                o = Oracle(128)
            d = o.checkpoint(snapshots[(c, k)], r.baseline)
            assert o.current_id - 1 == r.chkpt_id, (c, k)
            assert host_checksum(d) == r.checksum, (c, k, r.baseline)
            k += 1


def alone(sizes, rounds, dedup=TreeDeduplicator):
    out = {}
    for c, n in enumerate(sizes):
        s = synth.DeviceSeries(n, 128, c, max_run=64)
        h = dedup(128)
        for k in range(rounds):
            h.checkpoint_device(s.next(), k == 0)
            out[(c, k)] = h.diff_checksum()
        h.close()
    return out


def test_served_same_alone_and_in_mix(cuda):
    rounds = 4
    srv = CheckpointServer(hbm_budget=8e9, max_batch=4, max_inflight=2, checksum=True)
    snaps = {}
    reqs = drive(srv, SIZES, rounds, snapshots=snaps)
    assert all(r.rc == 0 for r in reqs.values())
    check_with_oracle(reqs, snaps)
    assert srv.batches < len(reqs)          # some requests shared a batch
    lat = [r.latency for r in reqs.values()]
    assert percentile(lat, 50) > 0 and percentile(lat, 99) >= percentile(lat, 50)
    want = alone(SIZES, rounds)
    for key, r in reqs.items():
        assert r.checksum == want[key], key
    srv.close()


def test_served_plain_mode_same(cuda):
    rounds = 3
    srv = CheckpointServer(hbm_budget=8e9, plain=True, checksum=True)
    snaps = {}
    reqs = drive(srv, SIZES, rounds, order_seed=2, snapshots=snaps)
    check_with_oracle(reqs, snaps)
    want = alone(SIZES, rounds)
    for key, r in reqs.items():
        assert r.rc == 0 and r.checksum == want[key], key
    srv.close()


@pytest.mark.parametrize("plain", [False, True])
def test_served_list_approach(cuda, plain):
    """approach="list": one ListDeduplicator per client; every request's list diff equals the
    one its client's buffers give checkpointed alone"""
    rounds = 3
    srv = CheckpointServer(hbm_budget=8e9, max_batch=4, max_inflight=2, checksum=True, plain=plain,
                           approach="list")
    snaps = {}
    reqs = drive(srv, SIZES, rounds, order_seed=5, snapshots=snaps)
    assert all(isinstance(c.handle, ListDeduplicator) for c in srv.clients.values())
    check_with_oracle(reqs, snaps, approach="list")
    want = alone(SIZES, rounds, ListDeduplicator)
    for key, r in reqs.items():
        assert r.rc == 0 and r.checksum == want[key], key
    srv.close()


def test_served_admission_budget(cuda):
    """a budget that holds two clients' state: the loop never exceeds it, evicts idle clients,
    and an evicted client's next request is a baseline"""
    sizes = [2 << 20] * 4
    budget = int(estimate_memory(2 << 20, 128) * 2.5)
    srv = CheckpointServer(hbm_budget=budget, max_batch=4, max_inflight=2, checksum=True)
    snaps = {}
    reqs = drive(srv, sizes, 3, order_seed=3, snapshots=snaps)
    assert all(r.rc == 0 for r in reqs.values())
    # a client that comes back after its eviction runs a baseline on a fresh handle; every
    # diff matches the oracle
    check_with_oracle(reqs, snaps)
    assert srv.peak_resident <= budget
    assert sum(1 for c in srv.clients.values() if c.handle is not None) <= 2
    srv.close()


def test_served_waits_without_eviction(cuda):
    """without eviction, a client that does not fit waits until the budget allows it (here: never
    while the others stay resident), and the loop reports it as not admitted"""
    import torch

    size = 1 << 20
    budget = int(estimate_memory(size, 128) * 1.5)
    srv = CheckpointServer(hbm_budget=budget, evict=False)
    a = torch.zeros(size, dtype=torch.uint8, device="cuda")
    b = torch.ones(size, dtype=torch.uint8, device="cuda")
    r0 = srv.submit(0, a)
    r1 = srv.submit(1, b)
    for _ in range(50):
        srv.step()
        if r0.done is not None:
            break
    while r0.done is None:
        srv.step()
    srv.step()
    assert r0.rc == 0 and r1.admitted is None and r1.done is None
    srv.close()


def test_served_diff_header(cuda):
    """first request of a client is its baseline, later ones reference it"""
    import numpy as np

    srv = CheckpointServer(hbm_budget=8e9)
    reqs = drive(srv, SIZES[:2], 2)
    for c in range(2):
        h = srv.clients[c].handle
        hdr = parse_header(np.frombuffer(bytes(h.copy_diff()), np.uint8))
        assert hdr["chkpt_id"] == 1 and hdr["ref_id"] == 0
    assert all(r.rc == 0 for r in reqs.values())
    srv.close()


def test_served_diffs_copied_to_host(cuda):
    """with host copy-back, a request completes with its diff in pinned host memory, byte-equal
    to the diff of the same client's buffers checkpointed alone"""
    rounds = 3
    sizes = SIZES[:4]
    for plain in (False, True):
        srv = CheckpointServer(hbm_budget=8e9, max_batch=4, max_inflight=2, plain=plain)
        srv.enable_host_copy({c: n for c, n in enumerate(sizes)})
        reqs = drive(srv, sizes, rounds, order_seed=4)
        got = {k: bytes(r.host.numpy() if hasattr(r.host, "numpy") else r.host) for k, r in reqs.items()}
        srv.close()
        for c, n in enumerate(sizes):
            s = synth.DeviceSeries(n, 128, c, max_run=64)
            h = TreeDeduplicator(128)
            for k in range(rounds):
                h.checkpoint_device(s.next(), k == 0)
                # each request's host view stays valid until the client's next request completes:
                # only the last one per client is still intact here
                if k == rounds - 1:
                    assert got[(c, k)] == bytes(h.copy_diff()), (plain, c, k)
            h.close()
