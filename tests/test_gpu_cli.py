"""The argv-compatible file tools (reference src/dedup_files.cpp, src/restart_chkpt_files.cpp).

dedup_files writes <file>.hashtree.incr_chkpt (--run-tree-chkpt) or <file>.hashlist.incr_chkpt
(--run-list-chkpt) next to each checkpoint file: byte-equal to the oracle's diffs.
restart_chkpt_files rebuilds a checkpoint from those files and prints its digest the way the
reference does: equal to the digest of the original file.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import _build, synth

pytestmark = pytest.mark.gpu


def ref_digest_str(data):
    d = O.hash_bytes(bytes(data), O.HASH_MURMUR3)
    h = d.hex().upper()
    return " ".join(h[i:i + 8] for i in range(0, 32, 8)) + " "


@pytest.mark.parametrize("mode", ["tree", "list"])
def test_dedup_and_restart_files(cuda, tmp_path, mode):
    _build.build()
    flag = f"--run-{mode}-chkpt"
    suffix = ".hashtree.incr_chkpt" if mode == "tree" else ".hashlist.incr_chkpt"
    label = "Hashtree digest:" if mode == "tree" else "Hashlist digest:"
    cs, n = 128, 4
    s = synth.ByteSeries(1 << 20, cs, lambda rng, k: synth.plan_varied(rng, k, 64), 9)
    files, bufs = [], []
    for i in range(n):
        b = s.next().copy()
        p = tmp_path / f"chkpt_{i}.dat"
        p.write_bytes(b.tobytes())
        files.append(str(p))
        bufs.append(b)
    r = subprocess.run([_build.tool_path("dedup_files"), str(cs), str(n), flag] + files,
                       capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    o = (O.OracleTreeDeduplicator if mode == "tree" else O.OracleListDeduplicator)(cs, O.HASH_MURMUR3)
    for i, b in enumerate(bufs):
        want = o.checkpoint(b, i == 0)
        assert open(files[i] + suffix, "rb").read() == want, i
    # the per-checkpoint log rows name the approach like the reference's (src/list_approach.cpp:1027)
    log = (tmp_path / f"chkpt_1.dat.chunk_size.{cs}.csv").read_text().splitlines()
    assert log[0].startswith("Approach,") and log[1].startswith("Tree," if mode == "tree" else "List,")
    for rid in (0, n - 1):
        r = subprocess.run([_build.tool_path("restart_chkpt_files"), str(rid), str(n), "2", str(cs),
                            flag] + files, capture_output=True, text=True, cwd=tmp_path)
        assert r.returncode == 0, r.stderr
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith(label)]
        assert len(lines) == 2
        assert lines[0].split(":", 1)[1].strip() == ref_digest_str(bufs[rid]).strip()

