"""The list-approach oracle (oracle/list_oracle.c) on the CPU.

The reference pins its list approach with test/list_chkpt.cpp: random 1 MiB checkpoints, each
restarted from the diffs so far must reproduce the data.  The same property is checked here,
plus the layout the diff must have in the reference's sequential order
(src/list_approach.cpp:79-257): first occurrences ascending by chunk, the repeat table ascending
by checkpoint, shifted pairs grouped by source checkpoint, the data section holding the first
occurrences' bytes.
"""
import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import parse_header


def split(diff):
    h = parse_header(diff)
    b = np.frombuffer(diff, np.uint8)
    F, P, S = h["num_first_ocur"], h["num_prior_chkpts"], h["num_shift_dupl"]
    first = b[32:32 + 4 * F].view(np.uint32)
    rows = b[32 + 4 * F:32 + 4 * F + 8 * P].view(np.uint32).reshape(-1, 2)
    pairs = b[32 + 4 * F + 8 * P:32 + 4 * F + 8 * P + 8 * S].view(np.uint32).reshape(-1, 2)
    data = b[32 + 4 * F + 8 * P + 8 * S:]
    return h, first, rows, pairs, data


@pytest.mark.parametrize("cs", [128, 64, 4096])
def test_list_chkpt_property(cs):
    """test/list_chkpt.cpp: ten random 1 MiB checkpoints, each restarts to its data"""
    rng = np.random.default_rng(1931)
    o = O.OracleListDeduplicator(cs)
    diffs = []
    for i in range(10):
        data = rng.integers(0, 256, 1 << 20, dtype=np.uint8)
        diffs.append(o.checkpoint(data, i == 0))
        out, rc = O.list_restart(diffs, i)
        assert rc == 0 and out.tobytes() == data.tobytes(), i


@pytest.mark.parametrize("n_chunks", [1, 2, 3, 5, 100, 1000, 4097])
def test_list_series_layout_and_restart(n_chunks):
    cs = 64
    rng = np.random.default_rng(n_chunks)
    base = rng.integers(0, 256, n_chunks * cs - (7 if n_chunks > 1 else 0), dtype=np.uint8)
    bufs = [base]
    for k in range(5):
        b = bufs[-1].copy()
        m = max(1, n_chunks // 10)
        for c in rng.integers(0, n_chunks, m):
            b[c * cs:(c + 1) * cs] = rng.integers(0, 256, min(cs, b.size - c * cs), dtype=np.uint8)
        if n_chunks > 4:   # shifted copies of other chunks, and a repeated pair within the checkpoint
            src, dst = rng.integers(0, n_chunks - 1, 2)
            b[dst * cs:(dst + 1) * cs] = bufs[0][src * cs:(src + 1) * cs]
            b[2 * cs:3 * cs] = b[3 * cs:4 * cs] = np.uint8(k + 1)
        bufs.append(b)
    o = O.OracleListDeduplicator(cs)
    diffs = [o.checkpoint(b, i == 0) for i, b in enumerate(bufs)]
    for i, (d, b) in enumerate(zip(diffs, bufs)):
        h, first, rows, pairs, data = split(d)
        assert h["chkpt_id"] == i and h["ref_id"] == 0 and h["datalen"] == b.size
        assert np.all(np.diff(first.astype(np.int64)) > 0)                      # chunk order
        assert np.all(np.diff(rows[:, 0].astype(np.int64)) > 0) and rows[:, 1].sum() == h["num_shift_dupl"]
        cum = np.cumsum(rows[:, 1])
        for j in range(h["num_shift_dupl"]):                                    # grouped by checkpoint
            t = rows[np.searchsorted(cum, j, side="right"), 0]
            assert t <= i
        for k, c in enumerate(first):                                           # first occurrence bytes
            chunk = b[c * cs:(c + 1) * cs]
            assert data[k * cs:k * cs + chunk.size].tobytes() == chunk.tobytes()
        out, rc = O.list_restart(diffs, i)
        assert rc == 0 and out.tobytes() == b.tobytes(), i


def test_list_baseline_resets_list_and_map():
    """a baseline starts from an all-zero digest list and an empty map (src/list_approach.cpp:865-869):
    after it, unchanged chunks of the previous series are first occurrences again"""
    rng = np.random.default_rng(5)
    a = rng.integers(0, 256, 64 * 100, dtype=np.uint8)
    o = O.OracleListDeduplicator(64)
    o.checkpoint(a, True)
    o.checkpoint(a, False)
    assert o.num_first_ocur() == 0 and o.num_shift_dupl() == 0
    o.checkpoint(a, True)
    assert o.num_first_ocur() == 100 and o.num_shift_dupl() == 0


def py_list_series(bufs, cs, baselines):
    """A second, independent reading of src/list_approach.cpp (:23-257, :843-931) in plain Python,
    for small inputs: the per-chunk rule in ascending chunk order, then the diff layout."""
    zero = bytes(16)
    digests, table, diffs = [], {}, []
    cur = base_id = 0
    for b, mb in zip(bufs, baselines):
        n = -(-len(b) // cs)
        if mb:
            digests, table = [zero] * n, {}
        digests += [zero] * (n - len(digests))
        if cur == 0 or mb:
            base_id = cur
        first, shift = [], []
        for c in range(n):
            d = O.hash_bytes(bytes(b[c * cs:(c + 1) * cs]))
            if d == digests[c]:
                continue
            if d in table:
                shift.append(c)
            else:
                table[d] = (c, cur)
                first.append(c)
            digests[c] = d
        src = {c: table[digests[c]] for c in shift}
        trees = sorted({t for _, t in src.values()})
        rows = b"".join(np.array([t, sum(1 for _, u in src.values() if u == t)], np.uint32).tobytes() for t in trees)
        pairs = b"".join(np.array([c, src[c][0]], np.uint32).tobytes()
                         for t in trees for c in shift if src[c][1] == t)
        data = b"".join(bytes(b[c * cs:(c + 1) * cs]).ljust(cs, b"\0") for c in first)
        hdr = np.array([base_id, cur], np.uint32).tobytes() + np.array([len(b)], np.uint64).tobytes() + \
            np.array([cs, len(first), len(trees), len(shift)], np.uint32).tobytes()
        diffs.append(hdr + np.array(first, np.uint32).tobytes() + rows + pairs + data)
        cur += 1
    return diffs


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_list_oracle_matches_independent_model(seed):
    """random small series with many repeated chunks, reverts and baselines mid-sequence"""
    rng = np.random.default_rng(seed)
    cs = [16, 32, 48, 64][seed]
    n = int(rng.integers(3, 200))
    size = n * cs - int(rng.integers(0, cs))
    palette = rng.integers(0, 256, (6, cs), dtype=np.uint8)
    bufs = []
    for k in range(6):
        pick = rng.integers(0, len(palette) + 2, n)
        b = np.concatenate([palette[p] if p < len(palette) else rng.integers(0, 256, cs, dtype=np.uint8)
                            for p in pick])[:size]
        bufs.append(b)
    baselines = [True, False, False, bool(rng.integers(0, 2)), False, False]
    o = O.OracleListDeduplicator(cs)
    got = [o.checkpoint(b, mb) for b, mb in zip(bufs, baselines)]
    assert got == py_list_series(bufs, cs, baselines)
