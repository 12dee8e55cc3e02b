"""GPU parity: the CUDA path through the C ABI against the oracle and the golden fixtures.

Bit-exact comparisons throughout: digests, diff bytes (header, metadata order, data) and
restarted buffers.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import HASH_MD5, HASH_MURMUR3, TreeDeduplicator, synth
from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import hash_chunks, parse_header

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def to_dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_both(bufs, cs, kind=HASH_MURMUR3, baselines=None, restart=True, tma=True, params=None):
    """checkpoint every buffer on the GPU and in the oracle; assert identical diffs and restarts"""
    import torch

    g = TreeDeduplicator(cs, kind)
    if not tma:
        g.set_param("leaf_tma", 0)
    for k, v in (params or {}).items():
        g.set_param(k, v)
    o = O.OracleTreeDeduplicator(cs, kind)
    gd, od = [], []
    for i, b in enumerate(bufs):
        mb = (i == 0) if baselines is None else bool(baselines[i])
        x = to_dev(b)
        gd.append(g.checkpoint(x, mb))
        od.append(o.checkpoint(b, mb))
        assert len(gd[-1]) == len(od[-1]), (i, parse_header(gd[-1]), parse_header(od[-1]))
        assert gd[-1] == od[-1], (i, parse_header(gd[-1]))
        assert (g.num_first_ocur(), g.num_shift_dupl()) == (o.num_first_ocur(), o.num_shift_dupl())
    if restart:
        dev_diffs = [to_dev(np.frombuffer(x, np.uint8)) for x in gd]
        for i, b in enumerate(bufs):
            want, rc = O.restart(od, i)
            out = torch.zeros(len(b), dtype=torch.uint8, device="cuda")
            grc = g.restart(out, gd, i, check_status=False)
            assert (grc == 0) == (rc == 0), (i, grc, rc)
            assert out.cpu().numpy().tobytes() == want.tobytes(), i
            # the same chain from device-resident diffs
            out.zero_()
            drc = g.restart_device(out, dev_diffs, i, check_status=False)
            assert drc == grc, (i, drc, grc)
            assert out.cpu().numpy().tobytes() == want.tobytes(), i
    run_both.map_stats = g.map_stats()
    g.close()
    return gd


def test_hash_kat_gpu(cuda):
    import torch

    for e in load("hash_kat.json")["kat"]:
        L = e["len"]
        if L == 0:
            continue
        x = torch.frombuffer(bytearray.fromhex(e["data"]), dtype=torch.uint8).cuda()
        assert hash_chunks(x, L, HASH_MURMUR3).cpu().numpy().tobytes().hex() == e["murmur3"], L
        assert hash_chunks(x, L, HASH_MD5).cpu().numpy().tobytes().hex() == e["md5"], L


@pytest.mark.parametrize("case", sorted(load("test_cases.json")))
def test_reference_test_cases_gpu(cuda, case):
    c = load("test_cases.json")[case]
    bufs = [np.frombuffer(c["step0"].encode(), np.uint8), np.frombuffer(c["step1"].encode(), np.uint8)]
    gd = run_both(bufs, 1)
    assert gd[0].hex() == c["diff0"] and gd[1].hex() == c["diff1"]


@pytest.mark.parametrize("name", sorted(load("series.json")))
@pytest.mark.parametrize("tma", [True, False])
def test_series_golden_gpu(cuda, name, tma):
    g = load("series.json")[name]
    plan = synth.plan_plain_64m if g["generator"] == "plain_64m" else synth.plan_plain_4g
    s = synth.ByteSeries(g["nbytes"], g["chunk_size"], plan, 1, 0)
    bufs = [s.next().copy() for _ in range(g["checkpoints"])]
    gd = run_both(bufs, g["chunk_size"], g["hash"], tma=tma)
    assert [hashlib.sha256(x).hexdigest() for x in gd] == g["sha256"]


def test_plain_64m_full_size(cuda):
    """The CPU-runnable benchmark case at its full size: 64 MiB, chunk 128 B, 5 checkpoints."""
    s = synth.plain_64m()
    bufs = [s.next().copy() for _ in range(5)]
    run_both(bufs, 128)
    # restart reproduces every checkpoint (power-of-two chunk count)
    import torch

    o = O.OracleTreeDeduplicator(128)
    diffs = [o.checkpoint(b, i == 0) for i, b in enumerate(bufs)]
    g = TreeDeduplicator(128)
    out = torch.zeros(len(bufs[0]), dtype=torch.uint8, device="cuda")
    for i, b in enumerate(bufs):
        g.restart(out, diffs, i)
        assert torch.equal(out.cpu(), torch.from_numpy(b))


@pytest.mark.parametrize("cs", [1, 7, 16, 32, 48, 64, 100, 128, 192, 256, 512, 4096])
@pytest.mark.parametrize("kind", [HASH_MURMUR3, HASH_MD5])
def test_chunk_sizes(cuda, cs, kind):
    nbytes = 96 * 1024 + 37 if cs > 1 else 3000
    s = synth.ByteSeries(nbytes, cs, synth.plan_plain_64m, 1, cs)
    bufs = [s.next().copy() for _ in range(4)]
    run_both(bufs, cs, kind)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 13, 100, 1000, 4097])
def test_small_and_non_power_of_two_trees(cuda, n):
    cs = 64
    s = synth.ByteSeries(n * cs, cs, synth.plan_plain_64m, 1, 1000 + n)
    bufs = [s.next().copy() for _ in range(4)]
    run_both(bufs, cs)


def test_duplicate_heavy_and_zero_pages(cuda):
    """Many equal chunks and equal subtrees at several depths: first-insert-wins order."""
    rng = np.random.default_rng(11)
    cs, n = 64, 3 * 1024 + 5
    bufs = []
    base = np.zeros(n * cs, np.uint8)
    for k in range(5):
        b = base.copy()
        pat = rng.integers(0, 4, n)
        for v in range(1, 4):
            b.reshape(n, cs)[pat == v] = v + k
        bufs.append(b)
    run_both(bufs, cs)
    run_both(bufs, cs, HASH_MD5)


def test_make_baseline_mid_sequence(cuda):
    s = synth.ByteSeries(256 * 1024, 128, synth.plan_plain_64m, 1, 77)
    bufs = [s.next().copy() for _ in range(6)]
    run_both(bufs, 128, baselines=[1, 0, 0, 1, 0, 0])


def test_whole_buffer_shift_bug_compatible(cuda):
    rng = np.random.default_rng(3)
    a = rng.integers(0, 256, 8 * 64, dtype=np.uint8)
    b = rng.integers(0, 256, 8 * 64, dtype=np.uint8)
    run_both([a, b, a], 64)


def test_len_change_without_baseline_rejected(cuda):
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError

    g = TreeDeduplicator(128)
    g.checkpoint(torch.zeros(4096, dtype=torch.uint8, device="cuda"), True)
    with pytest.raises(B2DError):
        g.checkpoint(torch.zeros(8192, dtype=torch.uint8, device="cuda"), False)
    g.checkpoint(torch.ones(8192, dtype=torch.uint8, device="cuda"), True)


def test_md5_float_series(cuda):
    """The MD5 training-state workload at reduced size (64 MiB): float32 with noise, zero pages, repeats."""
    s = synth.FloatSeries(64 << 20)
    bufs = [s.next().copy() for _ in range(4)]
    run_both(bufs, 256, HASH_MD5)


def test_map_growth_keeps_output(cuda):
    """a map with minimal headroom and a low load limit grows (allocate + rehash) during the
    series; diffs and restarts stay identical to the oracle, also with CUDA-graph replay"""
    s = synth.varied(4 << 20, 128, max_run=256, config_id=4, buf_id=3)
    bufs = [s.next().copy() for _ in range(8)]
    for graph in (0, 1):
        run_both(bufs, 128, params={"map_headroom_pct": 100, "map_max_load_pct": 30, "graph": graph})
        slots, entries, grows, _, _ = run_both.map_stats
        assert grows >= 1 and entries <= 0.3 * slots


def test_diff_views_without_host_copy(cuda):
    """checkpoint(copy=False) returns a read-only view of the pinned host diff; the bytes equal
    the oracle's while that staging grows (a tiny all-zero baseline first, then a full one)"""
    s = synth.plain_64m(nbytes=4 << 20)
    bufs = [np.zeros(4 << 20, np.uint8)] + [s.next().copy() for _ in range(3)]
    g = TreeDeduplicator(128, HASH_MURMUR3)
    o = O.OracleTreeDeduplicator(128, HASH_MURMUR3)
    sizes = []
    for i, (b, mb) in enumerate(zip(bufs, [True, True, False, False])):
        v = g.checkpoint(to_dev(b), mb, copy=False)
        want = o.checkpoint(b, mb)
        assert isinstance(v, np.ndarray) and v.dtype == np.uint8 and not v.flags.writeable
        assert v.tobytes() == want, i
        sizes.append(v.size)
    assert sizes[0] < sizes[1] // 8
    g.close()


@pytest.mark.parametrize("unit", [16, 32, 64])
def test_narrow_staging_units(cuda, unit):
    """the staged hashing kernel with segments narrower than the chunk allows"""
    s = synth.plain_64m(nbytes=8 << 20)
    bufs = [s.next().copy() for _ in range(3)]
    run_both(bufs, 128, params={"leaf_unit": unit})


def test_long_chain_restart_windows(cuda):
    """a 13-checkpoint chain: restarts from device diffs walk the 12 older diffs in two windows
    (8 + 4) with the NodeIDs carried between them; every checkpoint restarts like the oracle"""
    s = synth.ByteSeries(512 * 1024 + 64, 128, synth.plan_plain_64m, 1, 91)
    run_both([s.next().copy() for _ in range(13)], 128)


def test_checkpoint_id_limit(cuda):
    """checkpoint ids keep counting across baselines, as in the reference; a handle takes ids up
    to 8190 and then refuses further checkpoints with B2D_ERR_UNSUPPORTED (the digest map keeps a
    13-bit checkpoint field), leaving its last checkpoint intact"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError

    x = torch.arange(4096, dtype=torch.int32, device="cuda").to(torch.uint8)
    g = TreeDeduplicator(64)
    for i in range(8191):
        g.checkpoint_device(x, i % 1000 == 0)
    assert g.current_id == 8191
    last = g.copy_diff().tobytes()
    for baseline in (False, True):
        with pytest.raises(B2DError) as e:
            g.checkpoint_device(x, baseline)
        assert e.value.code == -11
    assert g.current_id == 8191 and g.copy_diff().tobytes() == last
    g.close()


REF = load("ref_series.json")


@pytest.mark.parametrize("name", sorted(k for k in REF if k != "source"))
def test_reference_series_gpu(cuda, name):
    """every diff equals, by sha256, the one the reference's own code writes for the same series
    (src/tree_approach.cpp / src/list_approach.cpp compiled unmodified on a sequential Kokkos
    stand-in, tests/golden/ref_series.json), and every restart rebuilds the same buffer"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import ListDeduplicator

    e = REF[name]
    if e["generator"] == "dup_heavy":
        bufs = synth.duplicate_heavy(e["size"], e["chunk_size"], e["checkpoints"])
    else:
        plan = synth.plan_plain_64m if e["generator"] == "plain_64m" else synth.plan_plain_4g
        s = synth.ByteSeries(e["size"], e["chunk_size"], plan, 1, e["size"] % 1000)
        bufs = [s.next().copy() for _ in range(e["checkpoints"])]
    g = (ListDeduplicator if e["approach"] == "list" else TreeDeduplicator)(e["chunk_size"])
    diffs = [g.checkpoint(to_dev(b), bool(m)) for b, m in zip(bufs, e["baselines"])]
    assert [len(d) for d in diffs] == e["sizes"]
    assert [hashlib.sha256(d).hexdigest() for d in diffs] == e["sha256"]
    if e["restart_sha256"] is not None:
        dev = [to_dev(np.frombuffer(d, np.uint8)) for d in diffs]
        for k, want in enumerate(e["restart_sha256"]):
            out = torch.zeros(len(bufs[k]), dtype=torch.uint8, device="cuda")
            g.restart_device(out, dev, k)
            assert hashlib.sha256(out.cpu().numpy().tobytes()).hexdigest() == want, k
    g.close()
