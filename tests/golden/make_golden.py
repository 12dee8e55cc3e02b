"""Regenerates the committed golden fixtures in this directory.

  hash_kat.json   chunk digests from the REFERENCE's own hash headers (include/kokkos_murmur3.hpp,
                  include/kokkos_md5.hpp, compiled unmodified by oracle/Makefile into
                  oracle/_ref/libref_hash.so) and OpenSSL MD5 (hashlib), over seeded inputs
  test_cases.json the reference's known-answer tests test/test_case_01.cpp .. test_case_10.cpp:
                  two 8-byte checkpoints with chunk size 1 and the expected (first, shift) region
                  counts, transcribed from those files; plus the oracle's diff bytes for each
  series.json     sha256 of every oracle diff of small seeded checkpoint series (regression pins)
  ref_series.json sha256 of every diff the REFERENCE's own TreeDeduplicator and ListDeduplicator
                  write (src/tree_approach.cpp, src/list_approach.cpp compiled unmodified against
                  the sequential Kokkos stand-in into oracle/_ref/libref_dedup.so) for seeded
                  series -- full-size config 1 included -- and of every buffer its restarts
                  rebuild where the reference's restart is defined (power-of-two chunk counts
                  for the tree; always for the list)

Run from the repository root, where the reference source tree is available:
    make -C oracle && python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth  # noqa: E402

# test/test_case_NN.cpp: step0 / step1 contents and the expected num_first_ocur(), num_shift_dupl()
TEST_CASES = {
    "01": ("ABCDEFGH", "IJKLMNOP", 1, 0),
    "02": ("ABCDEFGH", "ABCDEFGH", 0, 0),
    "03": ("ABCDEFGH", "ABCDEIJK", 2, 0),
    "04": ("ABCDEFGH", "IJABCDEK", 2, 3),
    "05": ("ABCDEFGH", "ABCIABCJ", 2, 2),
    "06": ("ABCDEFGH", "EFGBCDIJ", 1, 4),
    "07": ("ABCDEFGH", "IJKLABIH", 1, 2),
    "08": ("MNXYOPQR", "IJXYIJAB", 2, 1),
    "09": ("MNXYOPQR", "IJXYIJIB", 2, 2),
    "10": ("MNXYOPQR", "IJXYIJJI", 1, 3),
}

KAT_LENGTHS = list(range(0, 70)) + [96, 127, 128, 129, 192, 255, 256, 257, 512, 1000, 4096, 4097]

SERIES = [
    # (name, nbytes, chunk, hash, checkpoints, generator)
    ("plain_1m_cs128", 1 << 20, 128, O.HASH_MURMUR3, 4, "plain_64m"),
    ("plain_1m_cs64", 1 << 20, 64, O.HASH_MURMUR3, 4, "plain_64m"),
    ("plain_1m_cs4096", 1 << 20, 4096, O.HASH_MURMUR3, 4, "plain_4g"),
    ("plain_1m_cs256_md5", 1 << 20, 256, O.HASH_MD5, 4, "plain_64m"),
    ("ragged_1m_cs128", (1 << 20) + 77, 128, O.HASH_MURMUR3, 4, "plain_64m"),
    ("nonpow2_96k_cs128", 96 << 10, 128, O.HASH_MURMUR3, 4, "plain_64m"),
]


# (name, approach, generator, nbytes or chunk count, chunk, checkpoints, baselines): Murmur3, the
# hash the reference is built with
REF_SERIES = [
    ("tree_plain_64m_cs128", "tree", "plain_64m", 64 << 20, 128, 5, [1, 0, 0, 0, 0]),
    ("tree_plain_1m_cs64_rebase", "tree", "plain_64m", 1 << 20, 64, 6, [1, 0, 0, 1, 0, 0]),
    ("tree_ragged_1m_cs128", "tree", "plain_64m", (1 << 20) + 77, 128, 5, [1, 0, 0, 0, 0]),
    ("tree_plain_4m_cs4096", "tree", "plain_4g", 4 << 20, 4096, 4, [1, 0, 0, 0]),
    ("tree_nonpow2_96k_cs100", "tree", "plain_64m", (96 << 10) + 13, 100, 5, [1, 0, 0, 0, 0]),
    ("tree_chain13_512k_cs128", "tree", "plain_64m", (512 << 10) + 64, 128, 13, [1] + [0] * 12),
    ("tree_dupheavy_3077x64", "tree", "dup_heavy", 3077, 64, 5, [1, 0, 0, 0, 0]),
    ("tree_tiny_cs1", "tree", "plain_64m", 3000, 1, 4, [1, 0, 0, 0]),
    ("list_plain_1m_cs128_rebase", "list", "plain_64m", 1 << 20, 128, 6, [1, 0, 0, 1, 0, 0]),
    ("list_ragged_1m_cs64", "list", "plain_64m", (1 << 20) + 77, 64, 5, [1, 0, 0, 0, 0]),
    ("list_dupheavy_3077x64", "list", "dup_heavy", 3077, 64, 5, [1, 0, 0, 0, 0]),
]


def ref_series_inputs(gen, size, cs, nck):
    """the checkpoint buffers of one REF_SERIES entry"""
    if gen == "dup_heavy":
        return synth.duplicate_heavy(size, cs, nck)
    plan = synth.plan_plain_64m if gen == "plain_64m" else synth.plan_plain_4g
    s = synth.ByteSeries(size, cs, plan, 1, size % 1000)
    return [s.next().copy() for _ in range(nck)]


def ref_series_entry(approach, gen, size, cs, nck, baselines):
    bufs = ref_series_inputs(gen, size, cs, nck)
    r = O.RefDeduplicator(cs, approach)
    diffs = [r.checkpoint(b, m) for b, m in zip(bufs, baselines)]
    r.close()
    n = (len(bufs[0]) + cs - 1) // cs
    restarts = None
    if approach == "list" or n & (n - 1) == 0:
        restarts = []
        for k in range(nck):
            out = O.ref_restart(diffs, k, approach)
            assert np.array_equal(out, bufs[k]), (approach, gen, size, k)
            restarts.append(hashlib.sha256(out.tobytes()).hexdigest())
    return {"approach": approach, "generator": gen, "size": size, "chunk_size": cs, "checkpoints": nck,
            "baselines": baselines, "sha256": [hashlib.sha256(x).hexdigest() for x in diffs],
            "sizes": [len(x) for x in diffs], "restart_sha256": restarts}


def series_diffs(name, nbytes, cs, kind, nck, gen):
    s = synth.ByteSeries(nbytes, cs, synth.plan_plain_64m if gen == "plain_64m" else synth.plan_plain_4g, 1, 0)
    d = O.OracleTreeDeduplicator(cs, kind)
    out = []
    for i in range(nck):
        buf = s.next()
        out.append(d.checkpoint(buf, i == 0))
    return out


def main():
    R = O.ref_hash_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libref_hash.so missing: run `make -C oracle` where the reference exists")
    kat = []
    for L in KAT_LENGTHS:
        data = synth.chunk_bytes_np(77, [L], max(L, 1))[0][:L].copy()
        mm = np.zeros(16, np.uint8)
        md = np.zeros(16, np.uint8)
        R.ref_murmur3(data.ctypes.data, L, mm.ctypes.data)
        R.ref_md5(data.ctypes.data, L, md.ctypes.data)
        assert hashlib.md5(data.tobytes()).digest() == md.tobytes(), "reference MD5 != OpenSSL MD5"
        kat.append({"len": L, "data": data.tobytes().hex(), "murmur3": mm.tobytes().hex(), "md5": md.tobytes().hex()})
    with open(os.path.join(HERE, "hash_kat.json"), "w") as f:
        json.dump({"source": "reference include/kokkos_murmur3.hpp + include/kokkos_md5.hpp (unmodified)", "kat": kat},
                  f, indent=0)
    cases = {}
    for k, (a, b, ef, es) in TEST_CASES.items():
        d = O.OracleTreeDeduplicator(1)
        d0 = d.checkpoint(np.frombuffer(a.encode(), np.uint8), True)
        d1 = d.checkpoint(np.frombuffer(b.encode(), np.uint8), False)
        assert (d.num_first_ocur(), d.num_shift_dupl()) == (ef, es), k
        cases[k] = {"step0": a, "step1": b, "first": ef, "shift": es, "diff0": d0.hex(), "diff1": d1.hex(),
                    "source": f"test/test_case_{k}.cpp"}
    with open(os.path.join(HERE, "test_cases.json"), "w") as f:
        json.dump(cases, f, indent=1)
    series = {}
    for name, nbytes, cs, kind, nck, gen in SERIES:
        diffs = series_diffs(name, nbytes, cs, kind, nck, gen)
        series[name] = {"nbytes": nbytes, "chunk_size": cs, "hash": kind, "checkpoints": nck, "generator": gen,
                        "sha256": [hashlib.sha256(x).hexdigest() for x in diffs], "sizes": [len(x) for x in diffs]}
    with open(os.path.join(HERE, "series.json"), "w") as f:
        json.dump(series, f, indent=1)
    if O.ref_dedup_lib() is None:
        raise SystemExit("oracle/_ref/libref_dedup.so missing: run `make -C oracle` where the reference exists")
    ref = {"source": "reference src/tree_approach.cpp, src/list_approach.cpp (unmodified) on oracle/kokkos_shim"}
    for name, approach, gen, size, cs, nck, bl in REF_SERIES:
        ref[name] = ref_series_entry(approach, gen, size, cs, nck, bl)
    with open(os.path.join(HERE, "ref_series.json"), "w") as f:
        json.dump(ref, f, indent=1)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
