"""Batched checkpoints over the C ABI (b2d_batch_*).

The reference checkpoints one buffer per call (TreeDeduplicator::checkpoint,
src/tree_approach.cpp:1705-1738).  ``CheckpointBatch.checkpoint`` takes one buffer for each of
many ``TreeDeduplicator`` handles and runs them as one CUDA graph: a persistent hashing kernel
fed by a work queue over all buffers, then each handle's Merkle-tree and diff work on parallel
graph branches.  Each handle's diff is what its own ``checkpoint_device`` would produce.
"""
import ctypes

from ._lib import check, lib
from .tree import _dev_ptr, _stream_handle

__all__ = ["CheckpointBatch"]


class CheckpointBatch:
    PARAMS = ("leaf_stages", "leaf_ctas_per_sm", "tiles_per_pop", "streams", "shared", "warp_bands",
              "map_headroom_pct", "autotune", "graph_cache", "graph", "batch_diff", "batch_forest")

    def __init__(self, autotune=False, **params):
        h = ctypes.c_void_p()
        check(lib().b2d_batch_create(ctypes.byref(h)), "b2d_batch_create")
        self._h = h
        for k, v in params.items():
            self.set_param(k, v)
        if autotune:
            self.set_param("autotune", 1)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().b2d_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_param(self, name, value):
        check(lib().b2d_batch_set_param(self._h, name.encode(), int(value)), f"b2d_batch_set_param({name})")

    def get_param(self, name):
        v = ctypes.c_int64()
        check(lib().b2d_batch_get_param(self._h, name.encode(), ctypes.byref(v)), f"b2d_batch_get_param({name})")
        return v.value

    def _args(self, dedups, buffers, make_baseline):
        n = len(dedups)
        if len(buffers) != n:
            raise ValueError("one buffer per handle")
        hs = (ctypes.c_void_p * n)(*[d._h.value for d in dedups])
        ptrs = (ctypes.c_void_p * n)()
        lens = (ctypes.c_uint64 * n)()
        for i, b in enumerate(buffers):
            p, nb = _dev_ptr(b)
            ptrs[i] = p.value
            lens[i] = nb
        mb = None
        if make_baseline is not None:
            if isinstance(make_baseline, bool):
                make_baseline = [make_baseline] * n
            mb = (ctypes.c_int * n)(*[int(bool(x)) for x in make_baseline])
        return hs, ptrs, lens, mb, n

    def checkpoint(self, dedups, buffers, make_baseline=None, check_status=True):
        """One checkpoint of buffers[i] through dedups[i] for every i.  Returns per-handle status codes
        (raises on the first failure when check_status).  Diffs are read from each handle afterwards
        (``diff_device`` / ``copy_diff``)."""
        hs, ptrs, lens, mb, n = self._args(dedups, buffers, make_baseline)
        check(lib().b2d_batch_set_stream(self._h, _stream_handle()), "b2d_batch_set_stream")
        rcs = (ctypes.c_int * n)()
        rc = lib().b2d_batch_checkpoint(self._h, hs, ptrs, lens, mb, n, rcs)
        if check_status:
            check(rc, "b2d_batch_checkpoint")
        return list(rcs)

    def launch(self, dedups, buffers, make_baseline=None, stream=None):
        """First half of ``checkpoint``: prepares and launches the batch on `stream` (a
        torch.cuda.Stream; default the current one) and returns while it runs."""
        import ctypes as C

        hs, ptrs, lens, mb, n = self._args(dedups, buffers, make_baseline)
        sh = C.c_void_p(stream.cuda_stream) if stream is not None else _stream_handle()
        check(lib().b2d_batch_set_stream(self._h, sh), "b2d_batch_set_stream")
        self._n = n
        check(lib().b2d_batch_launch(self._h, hs, ptrs, lens, mb, n, None), "b2d_batch_launch")

    def done(self):
        """True once the launched batch's device work has completed (None: nothing in flight)."""
        v = ctypes.c_int()
        check(lib().b2d_batch_query(self._h, ctypes.byref(v)), "b2d_batch_query")
        return None if v.value < 0 else bool(v.value)

    def wait(self, check_status=True):
        """Second half: completes every handle's checkpoint; returns per-handle status codes."""
        rcs = (ctypes.c_int * max(1, getattr(self, "_n", 1)))()
        rc = lib().b2d_batch_wait(self._h, rcs)
        if check_status:
            check(rc, "b2d_batch_wait")
        return list(rcs)[:getattr(self, "_n", 0)]

    def times(self):
        """(device seconds of the last batch's graph, host seconds of the whole call)."""
        a = (ctypes.c_double * 2)()
        check(lib().b2d_batch_times(self._h, a), "b2d_batch_times")
        return a[0], a[1]

    def launch_count(self):
        v = ctypes.c_uint32()
        check(lib().b2d_batch_launch_count(self._h, ctypes.byref(v)), "b2d_batch_launch_count")
        return v.value
