"""Batched checkpoints (b2d_batch_checkpoint) against one-at-a-time checkpoints and the oracle.

Every handle's diff from a batch must be byte-identical to the diff the same handle type
produces when it checkpoints the same buffer alone (b2d_checkpoint_device), for buffers of
uneven sizes, short last chunks, several chunk sizes and both hash kinds in one batch (which
puts them in different hashing groups or on the per-buffer hashing path).
"""
import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import (HASH_MD5, HASH_MURMUR3, CheckpointBatch,
                                                                    TreeDeduplicator, synth)

pytestmark = pytest.mark.gpu

# (bytes, chunk size, hash kind): uneven sizes, a short last chunk, buffers smaller than one
# 256-chunk tile and than one chunk, chunk sizes that stage in 128/64-byte units, one that
# cannot be staged (100 B: per-buffer hashing path) and an MD5 buffer
SPECS = [
    (1 << 20, 128, HASH_MURMUR3),
    ((3 << 20) + 77, 128, HASH_MURMUR3),
    (200, 128, HASH_MURMUR3),
    (100, 128, HASH_MURMUR3),
    (5 << 20, 128, HASH_MURMUR3),
    (64 << 10, 64, HASH_MURMUR3),
    ((2 << 20) + 4096 * 3, 4096, HASH_MURMUR3),
    ((1 << 20) + 300, 100, HASH_MURMUR3),
    ((2 << 20) + 256 * 5 + 17, 256, HASH_MD5),
    (777 * 128, 128, HASH_MURMUR3),
]


def series(i, nbytes, cs):
    return synth.ByteSeries(nbytes, cs, lambda rng, n: synth.plan_varied(rng, n, 64), 7, buf_id=i, device="cuda")


def diffs_alone(specs, rounds, baselines):
    """reference result: each buffer through its own handle, one checkpoint at a time"""
    out = []
    for i, (nb, cs, kind) in enumerate(specs):
        s = series(i, nb, cs)
        d = TreeDeduplicator(cs, kind)
        per = []
        for r in range(rounds):
            x = s.next()
            d.checkpoint_device(x, baselines[r][i])
            per.append(bytes(d.copy_diff()))
        d.close()
        out.append(per)
    return out


def run_batch(specs, rounds, baselines, batch, zero_buf=None):
    ss = [series(i, nb, cs) for i, (nb, cs, _) in enumerate(specs)]
    hs = [TreeDeduplicator(cs, kind) for (_, cs, kind) in specs]
    got = [[] for _ in specs]
    for r in range(rounds):
        bufs = [s.next() for s in ss]
        rcs = batch.checkpoint(hs, bufs, baselines[r])
        assert rcs == [0] * len(specs)
        for i, h in enumerate(hs):
            got[i].append(bytes(h.copy_diff()))
            assert h.current_id == r + 1
    return got, hs, ss


def test_batch_equals_alone(cuda):
    rounds = 4
    baselines = [[True] * len(SPECS)] + [[False] * len(SPECS) for _ in range(rounds - 1)]
    baselines[2][3] = True   # a forced baseline in the middle of the batch
    want = diffs_alone(SPECS, rounds, baselines)
    with CheckpointBatch() as b:
        got, hs, _ = run_batch(SPECS, rounds, baselines, b)
        assert b.launch_count() > 0
        dev_s, host_s = b.times()
        assert dev_s > 0 and host_s >= dev_s * 0.5
    for i in range(len(SPECS)):
        for r in range(rounds):
            assert got[i][r] == want[i][r], (i, r, SPECS[i])


def test_batch_small_against_oracle(cuda):
    """the small buffers of the batch checked against the oracle directly, with restarts"""
    import torch

    specs = [(200, 128, HASH_MURMUR3), (4096 + 50, 64, HASH_MURMUR3), (8 * 1024 + 3, 100, HASH_MURMUR3),
             (64 * 1024, 256, HASH_MD5)]
    rounds = 3
    baselines = [[True] * len(specs)] + [[False] * len(specs) for _ in range(rounds - 1)]
    with CheckpointBatch() as b:
        got, hs, ss = run_batch(specs, rounds, baselines, b)
    for i, (nb, cs, kind) in enumerate(specs):
        s = synth.ByteSeries(nb, cs, lambda rng, n: synth.plan_varied(rng, n, 64), 7, buf_id=i)
        o = O.OracleTreeDeduplicator(cs, kind)
        od = [o.checkpoint(s.next(), r == 0) for r in range(rounds)]
        assert got[i] == od, i
        # the reference's restart is lossy for some tree shapes: match the oracle, status included
        want, orc = O.restart(od, rounds - 1)
        out = torch.zeros(nb, dtype=torch.uint8, device="cuda")
        grc = hs[i].restart(out, got[i], rounds - 1, check_status=False)
        assert (grc == 0) == (orc == 0), (i, grc, orc)
        assert out.cpu().numpy().tobytes() == want.tobytes(), i


def test_batch_zero_and_repeated_buffers(cuda):
    """buffers full of duplicates (all-zero, one repeated chunk) stress the map inside the batch"""
    import torch

    cs = 128
    a = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    pat = torch.arange(cs, dtype=torch.uint8, device="cuda").repeat((2 << 20) // cs)
    hs = [TreeDeduplicator(cs) for _ in range(2)]
    alone = [TreeDeduplicator(cs) for _ in range(2)]
    with CheckpointBatch(streams=2, tiles_per_pop=2) as b:
        for r in range(3):
            if r:
                a[r * 1000 * cs:(r * 1000 + 7) * cs] = r
                pat[5 * cs * r:(5 * r + 3) * cs] = 255
            b.checkpoint(hs, [a, pat])
            for h, al, x in zip(hs, alone, (a, pat)):
                al.checkpoint_device(x, r == 0)
                assert bytes(h.copy_diff()) == bytes(al.copy_diff()), r


def test_batch_autotune_keeps_output(cuda):
    """the tuner measures one setting per incremental round; output never changes"""
    specs = SPECS[:3] + SPECS[5:7]
    with CheckpointBatch(autotune=True) as b:
        # one baseline round (not scored), seven scored incremental rounds (one of them resizes
        # every map for the load-factor knob), then the result
        rounds = 9
        baselines = [[True] * len(specs)] + [[False] * len(specs) for _ in range(rounds - 1)]
        got, _, _ = run_batch(specs, rounds, baselines, b)
        assert b.get_param("tuned") == 1
        for k in ("shared", "leaf_stages", "leaf_ctas_per_sm", "tiles_per_pop", "streams", "warp_bands",
                  "map_headroom_pct"):
            b.get_param(k)
        assert b.get_param("warp_bands") in (0, 3) and b.get_param("map_headroom_pct") in (125, 150)
    want = diffs_alone(specs, rounds, baselines)
    assert got == want


def test_batch_rejects_duplicate_handles(cuda):
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError

    h = TreeDeduplicator(128)
    x = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    with CheckpointBatch() as b:
        with pytest.raises(B2DError):
            b.checkpoint([h, h], [x, x])


@pytest.mark.parametrize("baseline_first", [False, True])
def test_rejected_batch_changes_no_handle(cuda, baseline_first):
    """a batch whose second entry is invalid (length changed without a baseline, or empty) is
    rejected before any handle is prepared: the first handle's next checkpoint still diffs
    against its previous one, as the oracle does"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError

    s0 = synth.ByteSeries(64 << 10, 128, synth.plan_plain_64m, 1, 5)
    s1 = synth.ByteSeries(32 << 10, 128, synth.plan_plain_64m, 1, 6)
    a = [s0.next().copy() for _ in range(2)]
    b0 = s1.next().copy()
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    h0, h1 = TreeDeduplicator(128), TreeDeduplicator(128)
    o = O.OracleTreeDeduplicator(128)
    assert h0.checkpoint(dev(a[0]), True) == o.checkpoint(a[0], True)
    h1.checkpoint(dev(b0), True)
    bad = [torch.zeros(len(b0) + 128, dtype=torch.uint8, device="cuda"),
           torch.empty(0, dtype=torch.uint8, device="cuda")]
    with CheckpointBatch() as batch:
        for x, code in zip(bad, (-10, -1)):
            rcs = batch.checkpoint([h0, h1], [dev(a[1]), x], [baseline_first, False], check_status=False)
            assert rcs[1] == code, rcs
            with pytest.raises(B2DError):
                batch.checkpoint([h0, h1], [dev(a[1]), x], [baseline_first, False])
    assert h0.checkpoint(dev(a[1]), False) == o.checkpoint(a[1], False)
    h0.close()
    h1.close()


def test_empty_buffer_rejected(cuda):
    """an empty buffer is an argument error and leaves the handle as it was"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError

    s = synth.ByteSeries(16 << 10, 128, synth.plan_plain_64m, 1, 8)
    bufs = [s.next().copy() for _ in range(2)]
    h = TreeDeduplicator(128)
    o = O.OracleTreeDeduplicator(128)
    with pytest.raises(B2DError) as e:
        h.checkpoint(torch.empty(0, dtype=torch.uint8, device="cuda"), True)
    assert e.value.code == -1
    for i, x in enumerate(bufs):
        assert h.checkpoint(torch.from_numpy(x).cuda(), i == 0) == o.checkpoint(x, i == 0)
        with pytest.raises(B2DError):
            h.checkpoint(torch.empty(0, dtype=torch.uint8, device="cuda"), False)
    h.close()


@pytest.mark.parametrize("mode,batch_diff,batch_forest",
                         [(0, 1, 1), (1, 1, 1), (2, 1, 1), (0, 1, 0), (1, 1, 0), (0, 0, 0), (1, 0, 1)])
def test_batch_graph_modes_same(cuda, mode, batch_diff, batch_forest):
    """direct launches, graph replay and graph-from-second-batch, with the forest phases and the
    diff assembly shared across handles or per handle, give the same diffs"""
    specs = SPECS[:4] + SPECS[7:9]
    rounds = 3
    baselines = [[True] * len(specs)] + [[False] * len(specs) for _ in range(rounds - 1)]
    with CheckpointBatch(graph=mode, batch_diff=batch_diff, batch_forest=batch_forest) as b:
        got, _, _ = run_batch(specs, rounds, baselines, b)
        assert b.get_param("graph") == mode
        assert b.get_param("graphs") == {0: 0, 1: 1, 2: 1}[mode]
    assert got == diffs_alone(specs, rounds, baselines)
