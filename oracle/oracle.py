"""ctypes bindings for the CPU oracle (oracle/tree_oracle.c, oracle/list_oracle.c).

TEST INFRASTRUCTURE ONLY -- imported by tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU baseline.  The oracle restates the reference tree approach (src/tree_approach.cpp:13-1128)
and list approach (src/list_approach.cpp:23-586) of
TauferLab/Reproducibility_ICPP23_Scalable_GPU_Deduplication sequentially.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HASH_PATH = os.path.join(HERE, "_ref", "libref_hash.so")
REF_DEDUP_PATH = os.path.join(HERE, "_ref", "libref_dedup.so")

HASH_MURMUR3 = 0
HASH_MD5 = 1
_lib = None


def build(force=False):
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, os.path.join(HERE, "liboracle.so")], check=True,
                       stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        vp, u8p, u64, u32 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8), ctypes.c_uint64, ctypes.c_uint32
        L.oracle_create.restype = vp
        L.oracle_create.argtypes = [u32, ctypes.c_int]
        L.oracle_destroy.argtypes = [vp]
        L.oracle_set_threads.argtypes = [vp, ctypes.c_int]
        L.oracle_checkpoint.restype = ctypes.c_int
        L.oracle_checkpoint.argtypes = [vp, vp, u64, ctypes.c_int, ctypes.POINTER(u8p), ctypes.POINTER(u64)]
        L.oracle_free.argtypes = [vp]
        L.oracle_num_first_ocur.restype = u64
        L.oracle_num_first_ocur.argtypes = [vp]
        L.oracle_num_shift_dupl.restype = u64
        L.oracle_num_shift_dupl.argtypes = [vp]
        L.oracle_current_id.restype = u32
        L.oracle_current_id.argtypes = [vp]
        L.oracle_datasizes.argtypes = [vp, ctypes.POINTER(u64)]
        L.oracle_tree.restype = u8p
        L.oracle_tree.argtypes = [vp, ctypes.POINTER(u64)]
        L.oracle_labels.restype = u8p
        L.oracle_labels.argtypes = [vp]
        L.oracle_map_lookup.restype = ctypes.c_int
        L.oracle_map_lookup.argtypes = [vp, vp, ctypes.POINTER(u32)]
        L.oracle_map_size.restype = u64
        L.oracle_map_size.argtypes = [vp]
        L.oracle_restart.restype = ctypes.c_int
        L.oracle_restart.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(u64), u32, u32, vp, u64]
        L.oracle_hash.argtypes = [ctypes.c_int, vp, u64, vp]
        L.oracle_num_leaf_descendents.restype = u32
        L.oracle_num_leaf_descendents.argtypes = [u32, u32]
        L.oracle_leftmost_leaf.restype = u32
        L.oracle_leftmost_leaf.argtypes = [u32, u32]
        L.oracle_list_create.restype = vp
        L.oracle_list_create.argtypes = [u32, ctypes.c_int]
        L.oracle_list_destroy.argtypes = [vp]
        L.oracle_list_set_threads.argtypes = [vp, ctypes.c_int]
        L.oracle_list_checkpoint.restype = ctypes.c_int
        L.oracle_list_checkpoint.argtypes = [vp, vp, u64, ctypes.c_int, ctypes.POINTER(u8p), ctypes.POINTER(u64)]
        L.oracle_list_num_first_ocur.restype = u64
        L.oracle_list_num_first_ocur.argtypes = [vp]
        L.oracle_list_num_shift_dupl.restype = u64
        L.oracle_list_num_shift_dupl.argtypes = [vp]
        L.oracle_list_current_id.restype = u32
        L.oracle_list_current_id.argtypes = [vp]
        L.oracle_list_datasizes.argtypes = [vp, ctypes.POINTER(u64)]
        L.oracle_list_restart.restype = ctypes.c_int
        L.oracle_list_restart.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(u64), u32, u32, vp, u64]
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a.size else ctypes.c_void_p(0)


def _take_bytes(p, n):
    """`n` bytes at `p` as bytes (ctypes.string_at takes a C int length: 4 GiB diffs would be cut
    to their size modulo 2^32), then the oracle's buffer is freed"""
    out = np.ctypeslib.as_array(p, shape=(n,)).tobytes() if n else b""
    lib().oracle_free(p)
    return out


def hash_bytes(data, kind=HASH_MURMUR3):
    a = np.ascontiguousarray(np.frombuffer(bytes(data), dtype=np.uint8)) if not isinstance(data, np.ndarray) else np.ascontiguousarray(data, dtype=np.uint8)
    out = np.zeros(16, np.uint8)
    lib().oracle_hash(kind, _ptr(a), a.size, _ptr(out))
    return out.tobytes()


def num_leaf_descendents(node, num_nodes):
    return lib().oracle_num_leaf_descendents(node, num_nodes)


def leftmost_leaf(node, num_nodes):
    return lib().oracle_leftmost_leaf(node, num_nodes)


class OracleTreeDeduplicator:
    """Sequential restatement of the reference ``TreeDeduplicator`` (host buffers)."""

    def __init__(self, chunk_size, hash_kind=HASH_MURMUR3, threads=1):
        L = lib()
        self._h = L.oracle_create(chunk_size, hash_kind)
        if not self._h:
            raise ValueError("bad chunk size")
        L.oracle_set_threads(self._h, threads)
        self.chunk_size = chunk_size
        self.hash_kind = hash_kind

    def close(self):
        if self._h:
            lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def checkpoint(self, data, make_baseline=False):
        a = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_uint64(0)
        rc = lib().oracle_checkpoint(self._h, _ptr(a), a.size, int(bool(make_baseline)), ctypes.byref(out), ctypes.byref(n))
        if rc < 0:
            raise RuntimeError(f"oracle checkpoint failed: {rc}")
        diff = _take_bytes(out, n.value)
        self.last_rc = rc
        return diff

    def num_first_ocur(self):
        return lib().oracle_num_first_ocur(self._h)

    def num_shift_dupl(self):
        return lib().oracle_num_shift_dupl(self._h)

    @property
    def current_id(self):
        return lib().oracle_current_id(self._h)

    def datasizes(self):
        out = (ctypes.c_uint64 * 2)()
        lib().oracle_datasizes(self._h, out)
        return out[0], out[1]

    def tree(self):
        n = ctypes.c_uint64(0)
        p = lib().oracle_tree(self._h, ctypes.byref(n))
        return np.ctypeslib.as_array(p, shape=(n.value * 16,)).copy().reshape(-1, 16)

    def labels(self, num_nodes):
        p = lib().oracle_labels(self._h)
        return np.ctypeslib.as_array(p, shape=(num_nodes,)).copy()

    def map_lookup(self, digest):
        k = np.frombuffer(bytes(digest), np.uint8).copy()
        out = (ctypes.c_uint32 * 2)()
        ok = lib().oracle_map_lookup(self._h, _ptr(k), out)
        return (out[0], out[1]) if ok else None

    def map_size(self):
        return lib().oracle_map_size(self._h)


class OracleListDeduplicator:
    """Sequential restatement of the reference ``ListDeduplicator`` (host buffers)."""

    def __init__(self, chunk_size, hash_kind=HASH_MURMUR3, threads=1):
        L = lib()
        self._h = L.oracle_list_create(chunk_size, hash_kind)
        if not self._h:
            raise ValueError("bad chunk size")
        L.oracle_list_set_threads(self._h, threads)
        self.chunk_size = chunk_size
        self.hash_kind = hash_kind

    def close(self):
        if self._h:
            lib().oracle_list_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def checkpoint(self, data, make_baseline=False):
        a = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_uint64(0)
        rc = lib().oracle_list_checkpoint(self._h, _ptr(a), a.size, int(bool(make_baseline)), ctypes.byref(out),
                                          ctypes.byref(n))
        if rc < 0:
            raise RuntimeError(f"oracle list checkpoint failed: {rc}")
        diff = _take_bytes(out, n.value)
        self.last_rc = rc
        return diff

    def num_first_ocur(self):
        return lib().oracle_list_num_first_ocur(self._h)

    def num_shift_dupl(self):
        return lib().oracle_list_num_shift_dupl(self._h)

    @property
    def current_id(self):
        return lib().oracle_list_current_id(self._h)

    def datasizes(self):
        out = (ctypes.c_uint64 * 2)()
        lib().oracle_list_datasizes(self._h, out)
        return out[0], out[1]


def _as_u8(d):
    """a diff as a contiguous uint8 array, without a copy when it already is one (the oracle only
    reads it; full-size diffs are gigabytes)"""
    if isinstance(d, np.ndarray) and d.dtype == np.uint8 and d.flags.c_contiguous:
        return d.reshape(-1)
    if isinstance(d, (bytes, bytearray)):
        return np.frombuffer(d, dtype=np.uint8)
    return np.frombuffer(bytes(d), dtype=np.uint8)


def _restart(fn, diffs, chkpt_idx, out_len, init):
    bufs = [_as_u8(d) for d in diffs]
    if out_len is None:
        out_len = int(np.frombuffer(bufs[chkpt_idx][8:16].tobytes(), np.uint64)[0])
    out = np.zeros(out_len, np.uint8) if init is None else np.array(init, dtype=np.uint8).copy()
    ptrs = (ctypes.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
    sizes = (ctypes.c_uint64 * len(bufs))(*[b.size for b in bufs])
    rc = fn(ptrs, sizes, len(bufs), chkpt_idx, _ptr(out), out_len)
    if rc < 0:
        raise RuntimeError(f"oracle restart failed: {rc}")
    return out, rc


def list_restart(diffs, chkpt_idx, out_len=None, init=None):
    """List host-view restart (src/list_approach.cpp:259-586). Returns (buffer, rc)."""
    return _restart(lib().oracle_list_restart, diffs, chkpt_idx, out_len, init)


def restart(diffs, chkpt_idx, out_len=None, init=None):
    """Host-view restart (src/tree_approach.cpp:712-1128). Returns (buffer, rc)."""
    return _restart(lib().oracle_restart, diffs, chkpt_idx, out_len, init)


def ref_hash_lib():
    """The reference's own hash headers compiled in place (only where the source exists)."""
    if not os.path.exists(REF_HASH_PATH):
        return None
    L = ctypes.CDLL(REF_HASH_PATH)
    for f in (L.ref_murmur3, L.ref_md5):
        f.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    return L


_ref_dedup = None


def ref_dedup_lib():
    """The reference's own tree and list deduplicators compiled in place against the sequential
    Kokkos stand-in (oracle/kokkos_shim), or None where the reference source was not present."""
    global _ref_dedup
    if _ref_dedup is None and os.path.exists(REF_DEDUP_PATH):
        L = ctypes.CDLL(REF_DEDUP_PATH)
        vp, u8pp, u64 = ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)), ctypes.c_uint64
        for a in ("tree", "list"):
            getattr(L, f"ref_{a}_create").restype = vp
            getattr(L, f"ref_{a}_create").argtypes = [ctypes.c_uint32]
            getattr(L, f"ref_{a}_destroy").argtypes = [vp]
            getattr(L, f"ref_{a}_checkpoint").restype = ctypes.c_int
            getattr(L, f"ref_{a}_checkpoint").argtypes = [vp, vp, u64, ctypes.c_int, u8pp, ctypes.POINTER(u64)]
            getattr(L, f"ref_{a}_restart").restype = ctypes.c_int
            getattr(L, f"ref_{a}_restart").argtypes = [ctypes.c_uint32, ctypes.POINTER(vp), ctypes.POINTER(u64),
                                                       ctypes.c_uint32, ctypes.c_uint32, vp, u64]
        L.ref_tree_num_first_ocur.restype = u64
        L.ref_tree_num_first_ocur.argtypes = [vp]
        L.ref_tree_num_shift_dupl.restype = u64
        L.ref_tree_num_shift_dupl.argtypes = [vp]
        L.ref_free.argtypes = [vp]
        _ref_dedup = L
    return _ref_dedup


class RefDeduplicator:
    """The reference's own TreeDeduplicator / ListDeduplicator (approach "tree" / "list"),
    compiled from its source (Murmur3, the hash it is built with); checkpoint() is the host-view
    overload (src/tree_approach.cpp:1740-1748, src/list_approach.cpp)."""

    def __init__(self, chunk_size, approach="tree"):
        self.L = ref_dedup_lib()
        if self.L is None:
            raise RuntimeError("the compiled reference (oracle/_ref/libref_dedup.so) is not built")
        self.approach = approach
        self._h = getattr(self.L, f"ref_{approach}_create")(chunk_size)

    def checkpoint(self, data, make_baseline=False):
        a = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_uint64(0)
        rc = getattr(self.L, f"ref_{self.approach}_checkpoint")(self._h, _ptr(a), a.size, int(bool(make_baseline)),
                                                                ctypes.byref(out), ctypes.byref(n))
        if rc != 0:
            raise RuntimeError("reference checkpoint failed")
        diff = np.ctypeslib.as_array(out, shape=(n.value,)).tobytes() if n.value else b""
        self.L.ref_free(out)
        return diff

    def close(self):
        if self._h:
            getattr(self.L, f"ref_{self.approach}_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_restart(diffs, chkpt_idx, approach="tree", out_len=None, init=None):
    """The reference's own host-view restart of checkpoint `chkpt_idx` (src/tree_approach.cpp:
    1786-1817; src/list_approach.cpp), into a buffer that starts as `init` (zeros by default)."""
    L = ref_dedup_lib()
    if L is None:
        raise RuntimeError("the compiled reference (oracle/_ref/libref_dedup.so) is not built")
    bufs = [_as_u8(d) for d in diffs]
    hdr = np.frombuffer(bufs[chkpt_idx][:32].tobytes(), np.uint32)
    if out_len is None:
        out_len = int(hdr[2]) | (int(hdr[3]) << 32)
    out = np.zeros(out_len, np.uint8) if init is None else np.array(init, dtype=np.uint8).copy()
    ptrs = (ctypes.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
    sizes = (ctypes.c_uint64 * len(bufs))(*[b.size for b in bufs])
    getattr(L, f"ref_{approach}_restart")(int(hdr[4]), ptrs, sizes, len(bufs), chkpt_idx, _ptr(out), out_len)
    return out
