"""GPU parity of the list approach (ListDeduplicator) through the C ABI against the oracle.

Bit-exact comparisons: every diff (header, first-occurrence list, repeat table, shifted pairs,
data) and every restarted buffer, from host diffs and from device-resident diffs; list handles
in batches against their one-at-a-time diffs.
"""
import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import HASH_MD5, HASH_MURMUR3, ListDeduplicator, synth
from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import parse_header

pytestmark = pytest.mark.gpu


def to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_both(bufs, cs, kind=HASH_MURMUR3, baselines=None, restart=True):
    import torch

    g = ListDeduplicator(cs, kind)
    o = O.OracleListDeduplicator(cs, kind)
    gd, od = [], []
    for i, b in enumerate(bufs):
        mb = (i == 0) if baselines is None else bool(baselines[i])
        gd.append(g.checkpoint(to_dev(b), mb))
        od.append(o.checkpoint(b, mb))
        assert len(gd[-1]) == len(od[-1]), (i, parse_header(gd[-1]), parse_header(od[-1]))
        assert gd[-1] == od[-1], (i, parse_header(gd[-1]))
        assert (g.num_first_ocur(), g.num_shift_dupl()) == (o.num_first_ocur(), o.num_shift_dupl())
    if restart:
        dev_diffs = [to_dev(np.frombuffer(x, np.uint8)) for x in gd]
        for i, b in enumerate(bufs):
            want, rc = O.list_restart(od, i)
            out = torch.zeros(len(b), dtype=torch.uint8, device="cuda")
            grc = g.restart(out, gd, i, check_status=False)
            assert (grc == 0) == (rc == 0), (i, grc, rc)
            assert out.cpu().numpy().tobytes() == want.tobytes(), i
            out.zero_()
            drc = g.restart_device(out, dev_diffs, i, check_status=False)
            assert drc == grc, (i, drc, grc)
            assert out.cpu().numpy().tobytes() == want.tobytes(), i
    g.close()
    return gd


def test_list_chkpt_random(cuda):
    """test/list_chkpt.cpp: random 1 MiB checkpoints (every chunk new each time)"""
    rng = np.random.default_rng(1931)
    run_both([rng.integers(0, 256, 1 << 20, dtype=np.uint8) for _ in range(4)], 128)


@pytest.mark.parametrize("cs", [1, 7, 16, 64, 100, 128, 256, 4096])
@pytest.mark.parametrize("kind", [HASH_MURMUR3, HASH_MD5])
def test_list_chunk_sizes(cuda, cs, kind):
    nbytes = 96 * 1024 + 37 if cs > 1 else 3000
    s = synth.ByteSeries(nbytes, cs, synth.plan_plain_64m, 1, cs)
    run_both([s.next().copy() for _ in range(4)], cs, kind)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 13, 1000, 4097])
def test_list_chunk_counts(cuda, n):
    cs = 64
    s = synth.ByteSeries(n * cs, cs, synth.plan_plain_64m, 1, 2000 + n)
    run_both([s.next().copy() for _ in range(4)], cs)


def test_list_duplicates_and_zero_pages(cuda):
    """many equal chunks within and across checkpoints: the lowest chunk index owns a digest"""
    rng = np.random.default_rng(11)
    cs, n = 64, 3 * 1024 + 5
    bufs = []
    for k in range(5):
        b = np.zeros(n * cs, np.uint8)
        pat = rng.integers(0, 4, n)
        for v in range(1, 4):
            b.reshape(n, cs)[pat == v] = v + k % 2
        bufs.append(b)
    run_both(bufs, cs)
    run_both(bufs, cs, HASH_MD5)


def test_list_baseline_mid_sequence(cuda):
    s = synth.ByteSeries(256 * 1024, 128, synth.plan_plain_64m, 1, 78)
    run_both([s.next().copy() for _ in range(6)], 128, baselines=[1, 0, 0, 1, 0, 0])


def test_list_series_8m(cuda):
    """the plain workload's edit pattern (runs of changed chunks, shifted copies, zero pages)"""
    s = synth.plain_64m(nbytes=8 << 20)
    run_both([s.next().copy() for _ in range(5)], 128)


def test_list_revert_and_swap(cuda):
    """a chunk changing back to an older value, and two buffers alternating"""
    rng = np.random.default_rng(3)
    a = rng.integers(0, 256, 64 * 64, dtype=np.uint8)
    b = rng.integers(0, 256, 64 * 64, dtype=np.uint8)
    run_both([a, b, a, b], 64)


def test_list_md5_float_series(cuda):
    s = synth.FloatSeries(16 << 20)
    run_both([s.next().copy() for _ in range(3)], 256, HASH_MD5)


# (bytes, chunk size, approach): uneven sizes, short last chunks, a buffer smaller than a tile,
# one that cannot be staged (100 B chunks: per-buffer hashing in its branch)
MIXED = [(1 << 20, 128, "list"), ((3 << 20) + 77, 128, "tree"), (200, 128, "list"),
         ((2 << 20) + 300, 100, "list"), (5 << 20, 128, "tree"), (64 << 10, 64, "list")]


def _series(i, nbytes, cs):
    return synth.ByteSeries(nbytes, cs, lambda rng, n: synth.plan_varied(rng, n, 64), 11, buf_id=i, device="cuda")


def _handle(kind, cs):
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import TreeDeduplicator

    return (ListDeduplicator if kind == "list" else TreeDeduplicator)(cs)


@pytest.mark.parametrize("specs", [MIXED, [x for x in MIXED if x[2] == "list"]], ids=["mixed", "lists"])
@pytest.mark.parametrize("shared", [1, 0])
@pytest.mark.parametrize("graph", [0, 2])
def test_list_handles_in_batches(cuda, specs, shared, graph):
    """list handles in a batch (with tree handles, or alone): every handle's diff equals the diff
    it gives checkpointing alone, over baselines, incremental rounds and a mid-series baseline"""
    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import CheckpointBatch

    rounds = 5
    baselines = [[True] * len(specs)] + [[False] * len(specs) for _ in range(rounds - 1)]
    baselines[3][0] = True
    want = []
    for i, (nb, cs, kind) in enumerate(specs):
        s, h = _series(i, nb, cs), _handle(kind, cs)
        per = []
        for r in range(rounds):
            h.checkpoint_device(s.next(), baselines[r][i])
            per.append(bytes(h.copy_diff()))
        h.close()
        want.append(per)
    batch = CheckpointBatch(shared=shared, graph=graph)
    ss = [_series(i, nb, cs) for i, (nb, cs, _) in enumerate(specs)]
    hs = [_handle(kind, cs) for (_, cs, kind) in specs]
    for r in range(rounds):
        batch.checkpoint(hs, [s.next() for s in ss], baselines[r])
        for i, h in enumerate(hs):
            assert bytes(h.copy_diff()) == want[i][r], (r, i, specs[i])
    for h in hs:
        h.close()
    batch.close()


def test_list_long_chain_restart_windows(cuda):
    """13 list checkpoints: device-diff restarts cross two walk windows"""
    s = synth.ByteSeries(512 * 1024 + 64, 128, synth.plan_plain_64m, 1, 92)
    run_both([s.next().copy() for _ in range(13)], 128)
