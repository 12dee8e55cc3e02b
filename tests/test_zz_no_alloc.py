"""b2d_restart_noalloc: the restart entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc -- a process restoring a checkpoint after
the device ran out of memory, or a runtime whose device memory all belongs to its own pool --
and keeps its scratch in one fixed device array inside the library.  These tests call it
through the C ABI and compare its output byte for byte with the regular b2d_restart and with
the oracle's restart, on two calls in a row (the second call reuses the array the first one
left behind), at small sizes and at the array's capacity of 2^18 chunks.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from reproducibility_icpp23_scalable_gpu_deduplication_b200 import TreeDeduplicator, lib, synth

pytestmark = pytest.mark.gpu

B2D_ERR_FORMAT = -4
B2D_ERR_UNSUPPORTED = -11
NOALLOC_MAX_CHUNKS = 1 << 18


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


def check_against_regular_and_oracle(nbytes, cs, steps, buf_id, ids):
    import torch

    g, diffs, bufs = make_chain(nbytes, cs, steps, buf_id)
    dev_diffs = [torch.frombuffer(bytearray(d), dtype=torch.uint8).cuda() for d in diffs]
    for chkpt_id in ids:   # calls in a row on the shared scratch array
        want = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        rc_regular = g.restart(want, diffs, chkpt_id, check_status=False)
        oracle_out, rc_oracle = O.restart(diffs, chkpt_id)
        # all three start from a zeroed buffer: a restart of a non-power-of-two tree leaves some
        # chunks unwritten, in the reference as here
        got = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
        rc = noalloc_restart(got, dev_diffs, chkpt_id)
        assert rc == rc_regular and (rc == 0) == (rc_oracle == 0), (rc, rc_regular, rc_oracle)
        g_host = got.cpu().numpy()
        assert np.array_equal(g_host, want.cpu().numpy()), chkpt_id
        assert np.array_equal(g_host, oracle_out), chkpt_id
        n = (nbytes + cs - 1) // cs
        if n & (n - 1) == 0:
            assert np.array_equal(g_host, bufs[chkpt_id]), chkpt_id
    g.close()


@pytest.mark.parametrize("nbytes,cs", [(4 << 20, 128), (3 * (1 << 20) + 4096 + 77, 64)])
def test_noalloc_matches_regular_restart_twice(cuda, nbytes, cs):
    check_against_regular_and_oracle(nbytes, cs, 5, 500 + cs, (3, 4))


def test_noalloc_at_capacity(cuda):
    """exactly 2^18 chunks (32 MiB at 128 B): every region of the packed scratch layout at its
    full size"""
    check_against_regular_and_oracle(NOALLOC_MAX_CHUNKS * 128, 128, 3, 611, (2, 1))


def test_noalloc_near_capacity_ragged(cuda):
    """2^18 - 3 chunks with a short last chunk: a non-power-of-two tree, so regions straddle the
    tree's two leaf depths"""
    check_against_regular_and_oracle((NOALLOC_MAX_CHUNKS - 3) * 128 - 50, 128, 3, 612, (2, 2))


def test_noalloc_rejects_oversize(cuda):
    import torch

    hdr = np.zeros(8, np.uint32)
    datalen = NOALLOC_MAX_CHUNKS * 128 + 1        # one chunk beyond the fixed scratch capacity
    hdr[1], hdr[2], hdr[3], hdr[4] = 0, datalen & 0xFFFFFFFF, datalen >> 32, 128
    d = torch.from_numpy(hdr.view(np.uint8).copy()).cuda()
    out = torch.zeros(16, dtype=torch.uint8, device="cuda")
    big = torch.zeros(datalen, dtype=torch.uint8, device="cuda")
    assert noalloc_restart(big, [d], 0) == B2D_ERR_UNSUPPORTED
    assert lib().b2d_restart_noalloc(ctypes.c_void_p(out.data_ptr()), 16, None, None, 0, 0, None) == -1


@pytest.mark.parametrize("ref_id,chkpt_id,index", [(2, 1, 1), (0, 2, 1)])
def test_inconsistent_headers_rejected(cuda, ref_id, chkpt_id, index):
    """a main diff whose baseline comes after it, or whose id is not its position in the list,
    names no chain: every restart entry point returns B2D_ERR_FORMAT and writes nothing"""
    import torch

    g, diffs, _ = make_chain(64 << 10, 128, 3, 613)
    bad = bytearray(diffs[index])
    bad[0:4] = int(ref_id).to_bytes(4, "little")
    bad[4:8] = int(chkpt_id).to_bytes(4, "little")
    diffs = list(diffs)
    diffs[index] = bytes(bad)
    dev_diffs = [torch.frombuffer(bytearray(d), dtype=torch.uint8).cuda() for d in diffs]
    out = torch.full((64 << 10,), 0x77, dtype=torch.uint8, device="cuda")
    assert noalloc_restart(out, dev_diffs, index) == B2D_ERR_FORMAT
    assert g.restart(out, diffs, index, check_status=False) == B2D_ERR_FORMAT
    assert g.restart_device(out, dev_diffs, index, check_status=False) == B2D_ERR_FORMAT
    assert bool((out == 0x77).all())
    g.close()
