"""b2d_restart_noalloc: the restart entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc -- a process restoring a checkpoint after
the device ran out of memory, or a runtime whose device memory all belongs to its own pool --
and keeps its scratch in one fixed device array inside the library.  These tests call it
through the C ABI and compare its output byte for byte with the regular b2d_restart on two
calls in a row (the second call reuses the array the first one left behind).
"""
import ctypes

import numpy as np
import pytest

from reproducibility_icpp23_scalable_gpu_deduplication_b200 import TreeDeduplicator, lib, synth

pytestmark = pytest.mark.gpu

B2D_ERR_UNSUPPORTED = -11


def noalloc_restart(out, dev_diffs, chkpt_id):
    import torch

    ptrs = (ctypes.c_void_p * len(dev_diffs))(*[d.data_ptr() for d in dev_diffs])
    sizes = (ctypes.c_uint64 * len(dev_diffs))(*[d.numel() for d in dev_diffs])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
    return lib().b2d_restart_noalloc(ctypes.c_void_p(out.data_ptr()), out.numel(), ptrs, sizes, len(dev_diffs),
                                     chkpt_id, stream)


def make_chain(nbytes, cs, steps, buf_id):
    import torch

    s = synth.ByteSeries(nbytes, cs, synth.plan_plain_64m, 1, buf_id)
    g = TreeDeduplicator(cs)
    diffs, bufs = [], []
    for i in range(steps):
        b = s.next().copy()
        bufs.append(b)
        diffs.append(g.checkpoint(torch.from_numpy(b).cuda(), i == 0))
    return g, diffs, bufs


@pytest.mark.parametrize("nbytes,cs", [(4 << 20, 128), (3 * (1 << 20) + 4096 + 77, 64)])
def test_noalloc_matches_regular_restart_twice(cuda, nbytes, cs):
    import torch

    g, diffs, bufs = make_chain(nbytes, cs, 5, 500 + cs)
    dev_diffs = [torch.frombuffer(bytearray(d), dtype=torch.uint8).cuda() for d in diffs]
    for chkpt_id in (3, 4):   # two calls in a row on the shared scratch array
        want = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        rc_regular = g.restart(want, diffs, chkpt_id, check_status=False)
        got = torch.full((nbytes,), 0, dtype=torch.uint8, device="cuda")
        rc = noalloc_restart(got, dev_diffs, chkpt_id)
        assert rc == rc_regular
        assert torch.equal(got.cpu(), want.cpu())
        n = (nbytes + cs - 1) // cs
        if n & (n - 1) == 0:
            assert np.array_equal(got.cpu().numpy(), bufs[chkpt_id])
    g.close()


def test_noalloc_rejects_oversize(cuda):
    import torch

    hdr = np.zeros(8, np.uint32)
    datalen = (1 << 18) * 128 + 1        # one chunk beyond the fixed scratch capacity
    hdr[1], hdr[2], hdr[3], hdr[4] = 0, datalen & 0xFFFFFFFF, datalen >> 32, 128
    d = torch.from_numpy(hdr.view(np.uint8).copy()).cuda()
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    big = torch.zeros(datalen, dtype=torch.uint8, device="cuda")
    assert noalloc_restart(big, [d], 0) == B2D_ERR_UNSUPPORTED
    assert lib().b2d_restart_noalloc(ctypes.c_void_p(out.data_ptr()), 16, None, None, 0, 0, None) == -1
