"""Python mirror of the reference TreeDeduplicator over the C ABI.

Method names and argument meaning follow include/tree_approach.hpp:16-205 and
include/deduplicator_interface.hpp:14-184 of the reference: ``checkpoint`` takes a device
buffer (any CUDA tensor; its bytes are deduplicated) and returns the
``.hashtree.incr_chkpt`` diff, ``restart`` rebuilds a checkpoint into a device buffer from the
list of host diffs.  torch is used only for device memory and the current CUDA stream.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import HASH_MD5, HASH_MURMUR3, check, lib

__all__ = ["TreeDeduplicator", "ListDeduplicator", "hash_chunks", "HASH_MURMUR3", "HASH_MD5", "HEADER_BYTES", "parse_header"]

HEADER_BYTES = 32


def _dev_ptr(t):
    import torch

    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return ctypes.c_void_p(t.data_ptr()), t.numel() * t.element_size()


def _stream_handle():
    import torch

    # the legacy default stream has handle 0; pass cudaStreamLegacy (1) so the library
    # orders its work after torch's, instead of falling back to its own stream
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream or 1)


def _host_bytes(c):
    """A diff as a uint8 numpy view without copying when it already is one (pinned memory stays
    pinned, so the library copies it to the device directly)."""
    if isinstance(c, np.ndarray) and c.dtype == np.uint8 and c.flags.c_contiguous:
        return c
    if isinstance(c, (bytes, bytearray, memoryview)):
        return np.frombuffer(c, dtype=np.uint8)
    return np.frombuffer(bytes(c), dtype=np.uint8)


def parse_header(diff):
    """header_t (include/utils.hpp:29-37) of a diff as a dict."""
    h = np.frombuffer(bytes(diff[:HEADER_BYTES]), dtype=np.uint32)
    return {
        "ref_id": int(h[0]), "chkpt_id": int(h[1]),
        "datalen": int(h[2]) | (int(h[3]) << 32), "chunk_size": int(h[4]),
        "num_first_ocur": int(h[5]), "num_prior_chkpts": int(h[6]), "num_shift_dupl": int(h[7]),
    }


class TreeDeduplicator:
    """One deduplicated buffer: TreeDeduplicator(uint32_t bytes_per_chunk) (src/tree_approach.cpp:5-9)."""

    _create = "b2d_create"

    def __init__(self, chunk_size, hash_kind=HASH_MURMUR3):
        h = ctypes.c_void_p()
        check(getattr(lib(), self._create)(int(chunk_size), int(hash_kind), ctypes.byref(h)), self._create)
        self._h = h
        self.chunk_size = int(chunk_size)
        self.hash_kind = int(hash_kind)

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().b2d_destroy(self._h)
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
        """Tuning knob of the C ABI (b2d_set_param); output bytes never depend on it."""
        check(lib().b2d_set_param(self._h, name.encode(), int(value)), f"b2d_set_param({name})")

    def _sync_stream(self):
        check(lib().b2d_set_stream(self._h, _stream_handle()), "b2d_set_stream")

    # -- checkpoint overloads (src/tree_approach.cpp:1577-1776)
    def checkpoint_device(self, data, make_baseline=False, advance=True):
        """Dedup the device buffer; the diff stays on the device.  Returns its length."""
        self._sync_stream()
        p, n = _dev_ptr(data)
        out = ctypes.c_uint64(0)
        check(lib().b2d_checkpoint_device(self._h, p, n, int(bool(make_baseline)), int(bool(advance)),
                                          ctypes.byref(out)), "b2d_checkpoint_device")
        return out.value

    def diff_device(self):
        p, n = ctypes.c_void_p(), ctypes.c_uint64()
        check(lib().b2d_diff_device(self._h, ctypes.byref(p), ctypes.byref(n)), "b2d_diff_device")
        return p.value, n.value

    def copy_diff(self, out=None):
        _, n = self.diff_device()
        buf = np.empty(n, np.uint8) if out is None else out
        check(lib().b2d_copy_diff(self._h, ctypes.c_void_p(buf.ctypes.data), buf.nbytes), "b2d_copy_diff")
        return buf[:n]

    def copy_diff_async(self, out, stream=None):
        """Enqueue the copy of the last diff into `out` (a pinned uint8 tensor or array) on `stream`
        (a torch.cuda.Stream; default the handle's) and return the diff length; the bytes are
        there once that stream reaches the copy."""
        _, n = self.diff_device()
        if hasattr(out, "data_ptr"):
            ptr, cap = out.data_ptr(), out.numel() * out.element_size()
        else:
            ptr, cap = out.ctypes.data, out.nbytes
        sh = ctypes.c_void_p(stream.cuda_stream if stream is not None else None)
        check(lib().b2d_copy_diff_async(self._h, ctypes.c_void_p(ptr), cap, sh), "b2d_copy_diff_async")
        return n

    def checkpoint(self, data, make_baseline=False, filename=None, logname=None, copy=True):
        """checkpoint(data_ptr, len, diff_h[, logname], make_baseline) / (.., filename, logname, ..).

        Returns the diff as bytes (None for the file overload, which writes `filename`).  With
        ``copy=False`` it returns a read-only uint8 numpy view of the library's pinned host copy
        of the diff instead: no host-side copy, valid until this deduplicator's next call."""
        self._sync_stream()
        p, n = _dev_ptr(data)
        if filename is not None:
            check(lib().b2d_checkpoint_file(self._h, p, n, str(filename).encode(), str(logname or "/dev/null").encode(),
                                            int(bool(make_baseline))), "b2d_checkpoint_file")
            return None
        dptr = ctypes.POINTER(ctypes.c_uint8)()
        dlen = ctypes.c_uint64(0)
        if logname is not None:
            check(lib().b2d_checkpoint_log(self._h, p, n, str(logname).encode(), int(bool(make_baseline)),
                                           ctypes.byref(dptr), ctypes.byref(dlen)), "b2d_checkpoint_log")
        else:
            check(lib().b2d_checkpoint(self._h, p, n, int(bool(make_baseline)), ctypes.byref(dptr),
                                       ctypes.byref(dlen)), "b2d_checkpoint")
        view = np.ctypeslib.as_array(dptr, shape=(dlen.value,)) if dlen.value else np.empty(0, np.uint8)
        if copy:
            # not ctypes.string_at: its length is a C int, which cuts diffs of 2 GiB and more
            return view.tobytes()
        view.flags.writeable = False
        return view

    # -- restart overloads (src/tree_approach.cpp:1786-1838)
    def restart(self, out, chkpts, chkpt_id, logname=None, check_status=True):
        self._sync_stream()
        p, n = _dev_ptr(out)
        bufs = [_host_bytes(c) for c in chkpts]
        ptrs = (ctypes.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
        sizes = (ctypes.c_uint64 * len(bufs))(*[b.size for b in bufs])
        rc = lib().b2d_restart(self._h, p, n, ptrs, sizes, len(bufs), int(chkpt_id),
                               None if logname is None else str(logname).encode())
        if check_status:
            check(rc, "b2d_restart")
        return rc

    def restart_device(self, out, chkpts, chkpt_id, check_status=True):
        """restart from diffs already in device memory (CUDA uint8 tensors, e.g. diffs copied
        with diff_device or kept on the GPU); same result as ``restart``."""
        self._sync_stream()
        p, n = _dev_ptr(out)
        ds = [_dev_ptr(c) for c in chkpts]
        ptrs = (ctypes.c_void_p * len(ds))(*[q.value for q, _ in ds])
        sizes = (ctypes.c_uint64 * len(ds))(*[m for _, m in ds])
        rc = lib().b2d_restart_device(self._h, p, n, ptrs, sizes, len(ds), int(chkpt_id))
        if check_status:
            check(rc, "b2d_restart_device")
        return rc

    def restart_files(self, out, filenames, chkpt_id, logname=None, check_status=True):
        self._sync_stream()
        p, n = _dev_ptr(out)
        names = (ctypes.c_char_p * len(filenames))(*[str(f).encode() for f in filenames])
        rc = lib().b2d_restart_files(self._h, p, n, names, len(filenames), int(chkpt_id),
                                     None if logname is None else str(logname).encode())
        if check_status:
            check(rc, "b2d_restart_files")
        return rc

    # -- logs (include/deduplicator_interface.hpp:172-183)
    def write_chkpt_log(self, header, diff, logname):
        """write_chkpt_log(header_t&, HostMirror& diff_h, std::string& logname): the three CSV
        logs; `header` is the diff's 32-byte header (bytes, or None to take the diff's own)."""
        d = _host_bytes(diff)
        hb = np.frombuffer(bytes(d[:HEADER_BYTES]) if header is None else bytes(header), dtype=np.uint8)
        check(lib().b2d_write_chkpt_log_host(self._h, ctypes.c_void_p(hb.ctypes.data), ctypes.c_void_p(d.ctypes.data),
                                             d.size, str(logname).encode()), "b2d_write_chkpt_log_host")

    def write_restart_log(self, select_chkpt, logname):
        """write_restart_log(uint32_t select_chkpt, std::string& logname)"""
        check(lib().b2d_write_restart_log(self._h, int(select_chkpt), str(logname).encode()), "b2d_write_restart_log")

    # -- state (include/tree_approach.hpp:53-59, include/deduplicator_interface.hpp:16-23)
    def _u64(self, fn):
        v = ctypes.c_uint64()
        check(fn(self._h, ctypes.byref(v)), fn.__name__)
        return v.value

    def num_first_ocur(self):
        return self._u64(lib().b2d_num_first_ocur)

    def num_shift_dupl(self):
        return self._u64(lib().b2d_num_shift_dupl)

    @property
    def current_id(self):
        v = ctypes.c_uint32()
        check(lib().b2d_current_id(self._h, ctypes.byref(v)), "b2d_current_id")
        return v.value

    @property
    def baseline_id(self):
        v = ctypes.c_uint32()
        check(lib().b2d_baseline_id(self._h, ctypes.byref(v)), "b2d_baseline_id")
        return v.value

    @property
    def timers(self):
        a = (ctypes.c_double * 4)()
        check(lib().b2d_timers(self._h, a), "b2d_timers")
        return list(a)

    @property
    def restart_timers(self):
        a = (ctypes.c_double * 2)()
        check(lib().b2d_restart_timers(self._h, a), "b2d_restart_timers")
        return list(a)

    @property
    def datasizes(self):
        a = (ctypes.c_uint64 * 2)()
        check(lib().b2d_datasizes(self._h, a), "b2d_datasizes")
        return a[0], a[1]

    def phase_times(self):
        """(leaf, forest, gather) device seconds of the last checkpoint, and the leaf path (1 = TMA)."""
        a = (ctypes.c_double * 3)()
        p = ctypes.c_int()
        check(lib().b2d_phase_times(self._h, a, ctypes.byref(p)), "b2d_phase_times")
        return list(a), p.value

    def last_launch_count(self):
        v = ctypes.c_uint32()
        check(lib().b2d_last_launch_count(self._h, ctypes.byref(v)), "b2d_last_launch_count")
        return v.value

    def memory(self):
        """Device bytes this handle holds."""
        v = ctypes.c_uint64()
        check(lib().b2d_memory(self._h, ctypes.byref(v)), "b2d_memory")
        return v.value

    def map_stats(self):
        """(slots, entries, growths, seconds spent growing, of which allocating) of the digest map."""
        a = (ctypes.c_double * 5)()
        check(lib().b2d_map_stats(self._h, a), "b2d_map_stats")
        return int(a[0]), int(a[1]), int(a[2]), a[3], a[4]

    def diff_checksum(self, block=4096):
        """MD5 (hex) of the Murmur3 digests of the device diff's `block`-byte blocks: a cheap identity
        check of a large diff without copying it to the host."""
        import hashlib

        import torch

        p, n = self.diff_device()
        nblk = (n + block - 1) // block
        out = torch.empty((nblk, 16), dtype=torch.uint8, device="cuda")
        check(lib().b2d_hash_chunks(HASH_MURMUR3, ctypes.c_void_p(p), n, int(block), ctypes.c_void_p(out.data_ptr()),
                                    _stream_handle()), "b2d_hash_chunks")
        return hashlib.md5(out.cpu().numpy().tobytes() + n.to_bytes(8, "little")).hexdigest()

    def debug_tree(self, nodes):
        out = np.empty((nodes, 16), np.uint8)
        check(lib().b2d_debug_tree(self._h, ctypes.c_void_p(out.ctypes.data), nodes), "b2d_debug_tree")
        return out

    def debug_labels(self, leaves):
        out = np.empty(leaves, np.uint8)
        check(lib().b2d_debug_labels(self._h, ctypes.c_void_p(out.ctypes.data), leaves), "b2d_debug_labels")
        return out


def reserve_map_memory(nbytes):
    """Keep `nbytes` of device memory mapped for digest maps (see b2d_pool_reserve)."""
    check(lib().b2d_pool_reserve(int(nbytes)), "b2d_pool_reserve")


def estimate_memory(nbytes, chunk_size, map_max_load_pct=0):
    """Device bytes a handle will hold for checkpoints of an `nbytes` buffer."""
    v = ctypes.c_uint64()
    check(lib().b2d_estimate_memory(int(nbytes), int(chunk_size), int(map_max_load_pct), ctypes.byref(v)),
          "b2d_estimate_memory")
    return v.value



class ListDeduplicator(TreeDeduplicator):
    """The list approach: ListDeduplicator(uint32_t bytes_per_chunk) (src/list_approach.cpp:5-9).

    Same methods and argument meaning as ``TreeDeduplicator`` (include/list_approach.hpp): one
    digest per chunk, a changed chunk is a first occurrence or a shifted duplicate of an earlier
    one, and the diff names chunk indices (src/list_approach.cpp:23-257).  Restarts take list
    diffs (:259-586).  ``CheckpointBatch`` takes list handles beside tree handles."""

    _create = "b2d_create_list"


def hash_chunks(data, chunk_size, hash_kind=HASH_MURMUR3):
    """Digest of every chunk of a device buffer (the reference's hash(), one per chunk)."""
    import torch

    p, n = _dev_ptr(data)
    nchunks = (n + chunk_size - 1) // chunk_size
    out = torch.empty((nchunks, 16), dtype=torch.uint8, device=data.device)
    check(lib().b2d_hash_chunks(int(hash_kind), p, n, int(chunk_size), ctypes.c_void_p(out.data_ptr()),
                                _stream_handle()), "b2d_hash_chunks")
    return out
