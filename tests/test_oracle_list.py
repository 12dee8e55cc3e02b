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
