"""Parity at the benchmark sizes: the CUDA path against the oracle on the full buffers the
throughput figures are quoted on.

* the 4 GiB uint8 series (1% changed in Geometric(1/32) runs capped at 1024, 0.5% shifted
  copies, Murmur3) at every chunk size of that configuration, 64 B to 4 KiB (2^26 down to 2^20
  chunks): a baseline and two incremental checkpoints;
* the 8 GiB float32 series with MD5 and 256 B chunks (2^25 chunks): a baseline and two
  incremental checkpoints.

Every diff is compared byte for byte with the oracle's (src/tree_approach.cpp:261-710), and the
last checkpoint is restarted from device-resident and from host diffs and compared with the
oracle's restart (src/tree_approach.cpp:712-1128) and with the input buffer.  The buffers are
generated on the device and copied to host memory for the oracle, which hashes with every host
thread.  Each case needs tens of GB of host memory (oracle tree and map, the buffer, the
baseline diff and a restarted copy); a case that would not fit in the host's available memory
is skipped with that reason rather than run into the out-of-memory killer.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import HASH_MD5, HASH_MURMUR3, TreeDeduplicator, synth
from reproducibility_icpp23_scalable_gpu_deduplication_b200.tree import parse_header

pytestmark = pytest.mark.gpu
GiB = 1 << 30


def host_bytes_needed(nbytes, cs):
    """Peak host memory of one case: the input copy, the baseline diff twice (ours and the
    oracle's, compared, then one dropped), the restarted buffer, and the oracle's tree (16 B per
    node) and digest map (6 slots of 25 B per node after a baseline)."""
    nodes = 2 * ((nbytes + cs - 1) // cs)
    return 4 * nbytes + nodes * (16 + 6 * 25) + 2 * GiB


def require_host_memory(need):
    import psutil

    avail = psutil.virtual_memory().available
    if avail < need:
        pytest.skip(f"needs {need / GiB:.0f} GiB of host memory, {avail / GiB:.0f} GiB available")


def run_full(series, nbytes, cs, kind, ckpts=3):
    import torch

    g = TreeDeduplicator(cs, kind)
    o = O.OracleTreeDeduplicator(cs, kind, threads=os.cpu_count() or 1)
    host_diffs, x = [], None
    for k in range(ckpts):
        x = series.next()
        n = g.checkpoint_device(x, k == 0)
        gd = g.copy_diff()
        assert gd.size == n
        od = o.checkpoint(x.view(-1).cpu().numpy(), k == 0)
        assert len(od) == n, (cs, k, parse_header(gd), parse_header(od))
        assert np.array_equal(gd, np.frombuffer(od, np.uint8)), (cs, k, parse_header(gd))
        assert (g.num_first_ocur(), g.num_shift_dupl()) == (o.num_first_ocur(), o.num_shift_dupl()), (cs, k)
        del od
        host_diffs.append(gd)
    last = ckpts - 1
    want, rc = O.restart(host_diffs, last)
    assert rc == 0
    o.close()
    xin = x.view(-1)
    # the series' chunk counts are powers of two, so the restart is exact (no straddling regions)
    assert np.array_equal(want, xin.cpu().numpy())
    out = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dev_diffs = [torch.from_numpy(d).cuda() for d in host_diffs]
    out.fill_(0xA5)
    g.restart_device(out, dev_diffs, last)
    assert torch.equal(out, xin), cs
    del dev_diffs
    out.fill_(0x5A)
    g.restart(out, host_diffs, last)
    assert torch.equal(out, xin), cs
    g.close()
    del out, host_diffs, want
    torch.cuda.empty_cache()


@pytest.mark.parametrize("cs", [64, 128, 256, 512, 4096])
def test_plain_4g_full_size(cuda, cs):
    nbytes = 4 * GiB
    require_host_memory(host_bytes_needed(nbytes, cs))
    run_full(synth.plain_4g(nbytes=nbytes, chunk_size=cs, device=cuda), nbytes, cs, HASH_MURMUR3)


def test_md5_f32_8g_full_size(cuda):
    nbytes = 8 * GiB
    require_host_memory(host_bytes_needed(nbytes, 256))
    run_full(synth.FloatSeries(nbytes=nbytes, device=cuda), nbytes, 256, HASH_MD5)
