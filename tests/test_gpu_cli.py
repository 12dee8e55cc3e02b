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



def test_checkpoint_file_overload_and_write_failure(cuda, tmp_path):
    """checkpoint(data, filename, logname, make_baseline) writes the oracle's diff bytes and one
    log row per checkpoint; a diff that cannot be written (B2D_ERR_IO) does not advance the
    checkpoint id, and the handle then takes only a baseline, which continues the id sequence"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import B2DError, TreeDeduplicator

    s = synth.ByteSeries(256 << 10, 128, synth.plan_plain_64m, 1, 21)
    bufs = [s.next().copy() for _ in range(3)]
    o = O.OracleTreeDeduplicator(128)
    want = [o.checkpoint(bufs[0], True), o.checkpoint(bufs[1], False), o.checkpoint(bufs[2], True)]
    h = TreeDeduplicator(128)
    log = str(tmp_path / "run")
    files = [tmp_path / f"c{i}.hashtree.incr_chkpt" for i in range(3)]
    dev = [torch.from_numpy(b).cuda() for b in bufs]
    assert h.checkpoint(dev[0], True, filename=files[0], logname=log) is None
    h.checkpoint(dev[1], False, filename=files[1], logname=log)
    with pytest.raises(B2DError) as e:
        h.checkpoint(dev[2], False, filename=tmp_path / "missing" / "c2", logname=log)
    assert e.value.code == -5
    with pytest.raises(B2DError) as e:
        h.checkpoint(dev[2], False, filename=files[2], logname=log)
    assert e.value.code == -10
    h.checkpoint(dev[2], True, filename=files[2], logname=log)
    assert [f.read_bytes() for f in files] == want
    with open(log + ".chunk_size.128.csv") as f:
        rows = f.read().splitlines()
    assert rows[0].startswith("Approach,Chkpt ID") and [r.split(",")[1] for r in rows[1:]] == ["0", "1", "2", "2"]
    h.close()


def test_log_writers(cuda, tmp_path):
    """write_chkpt_log(header, diff_h, logname) and write_restart_log(select_chkpt, logname)
    (include/deduplicator_interface.hpp:172-183): the rows equal the ones the log-writing
    checkpoint and restart overloads write for the same checkpoint (Chkpt ID = current_id, as in
    the reference, which calls them before current_id += 1)"""
    import torch

    from reproducibility_icpp23_scalable_gpu_deduplication_b200 import TreeDeduplicator

    s = synth.ByteSeries(256 << 10, 128, synth.plan_plain_64m, 1, 22)
    bufs = [torch.from_numpy(s.next().copy()).cuda() for _ in range(2)]
    a, b = TreeDeduplicator(128), TreeDeduplicator(128)
    la, lb = str(tmp_path / "a"), str(tmp_path / "b")
    diffs = []
    for i, x in enumerate(bufs):
        diffs.append(a.checkpoint(x, i == 0, logname=la))
        # the header_t& overload's steps: checkpoint without advancing, write the logs, advance
        b.checkpoint_device(x, i == 0, advance=False)
        d = b.copy_diff()
        assert d.tobytes() == diffs[-1]
        b.write_chkpt_log(d[:32].tobytes(), d, lb)
        b.checkpoint_device(x, i == 0)          # same diff again, now advancing the id
    for ext, fields in ((".csv", 7), (".size.csv", None), (".timing.csv", 3)):
        ra = open(la + ".chunk_size.128" + ext).read().splitlines()
        rb = open(lb + ".chunk_size.128" + ext).read().splitlines()
        assert len(ra) == len(rb) and [r.split(",")[:fields] for r in ra] == [r.split(",")[:fields] for r in rb], ext
    out = torch.zeros(len(bufs[0]), dtype=torch.uint8, device="cuda")
    ra_log, rb_log = str(tmp_path / "ra.csv"), str(tmp_path / "rb.csv")
    a.restart(out, diffs, 1, logname=ra_log)   # the host-view overload names its log after logname
    assert torch.equal(out, bufs[1])
    a.write_restart_log(1, rb_log)              # the interface method writes to logname itself
    ra = open(ra_log + ".chunk_size.128.restart_timing.csv").read()
    assert ra == open(rb_log).read() and ra.startswith("Tree,1,128,")
    a.close()
    b.close()
