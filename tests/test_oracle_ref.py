"""The oracle against the reference's own code.

`tests/golden/ref_series.json` holds the sha256 of every diff the reference's own
TreeDeduplicator and ListDeduplicator write (src/tree_approach.cpp, src/list_approach.cpp compiled
unmodified against the sequential Kokkos stand-in in oracle/kokkos_shim/) for seeded series, and
of every buffer its restarts rebuild where they are defined.  The oracle must write the same
bytes and rebuild the same buffers; where the compiled reference is present (it is built with the
oracle wherever the reference source exists), further seeded series are compared live.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "ref_series.json")) as f:
    REF = json.load(f)
NAMES = sorted(k for k in REF if k != "source")


def ref_inputs(e):
    if e["generator"] == "dup_heavy":
        return synth.duplicate_heavy(e["size"], e["chunk_size"], e["checkpoints"])
    plan = synth.plan_plain_64m if e["generator"] == "plain_64m" else synth.plan_plain_4g
    s = synth.ByteSeries(e["size"], e["chunk_size"], plan, 1, e["size"] % 1000)
    return [s.next().copy() for _ in range(e["checkpoints"])]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_fixture(name):
    e = REF[name]
    bufs = ref_inputs(e)
    cls = O.OracleListDeduplicator if e["approach"] == "list" else O.OracleTreeDeduplicator
    o = cls(e["chunk_size"], O.HASH_MURMUR3, threads=4)
    diffs = [o.checkpoint(b, bool(m)) for b, m in zip(bufs, e["baselines"])]
    assert [len(d) for d in diffs] == e["sizes"]
    assert [hashlib.sha256(d).hexdigest() for d in diffs] == e["sha256"]
    if e["restart_sha256"] is not None:
        restart = O.list_restart if e["approach"] == "list" else O.restart
        for k, want in enumerate(e["restart_sha256"]):
            out, _ = restart(diffs, k)
            assert hashlib.sha256(out.tobytes()).hexdigest() == want, k


@pytest.mark.skipif(O.ref_dedup_lib() is None, reason="compiled reference not built (reference source absent)")
@pytest.mark.parametrize("approach", ["tree", "list"])
@pytest.mark.parametrize("seed", [11, 12, 13])
def test_oracle_matches_reference_live(approach, seed):
    """random sizes, chunk sizes and baseline patterns, both approaches: identical diffs, and
    identical restarts where the reference's restart is defined"""
    rng = np.random.default_rng(seed)
    cs = int(rng.choice([1, 8, 48, 64, 128, 200, 512]))
    nbytes = int(rng.integers(1, 3000) * cs + rng.integers(0, cs))
    s = synth.ByteSeries(nbytes, cs, synth.plan_plain_64m, 1, seed)
    bufs = [s.next().copy() for _ in range(7)]
    baselines = [1] + [int(x) for x in rng.integers(0, 4, 6) == 0]
    r = O.RefDeduplicator(cs, approach)
    o = (O.OracleListDeduplicator if approach == "list" else O.OracleTreeDeduplicator)(cs)
    rd = [r.checkpoint(b, m) for b, m in zip(bufs, baselines)]
    od = [o.checkpoint(b, m) for b, m in zip(bufs, baselines)]
    assert rd == od
    n = (nbytes + cs - 1) // cs
    if approach == "list" or n & (n - 1) == 0:
        restart = O.list_restart if approach == "list" else O.restart
        for k in range(len(bufs)):
            assert np.array_equal(O.ref_restart(rd, k, approach), restart(od, k)[0]), k
