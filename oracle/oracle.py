"""ctypes wrapper of the CPU oracle (dcore_oracle.c) -- TEST INFRASTRUCTURE.

Used only by the tests, the smoke check and the benchmark's CPU-baseline leg
to check or time the engine; never by the engine itself.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None

u32p = ctypes.POINTER(ctypes.c_uint32)
i32p = ctypes.POINTER(ctypes.c_int32)
i64p = ctypes.POINTER(ctypes.c_int64)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b  # noqa: F401  (package import when available)
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.or_peel_levels.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_int, ctypes.c_int32, i32p]
        _lib.or_peel_levels.restype = ctypes.c_int32
        _lib.or_kmax.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, i32p]
        _lib.or_kmax.restype = ctypes.c_int32
        _lib.or_bz_row.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, i32p, ctypes.c_int32, i32p]
        _lib.or_bz_row.restype = ctypes.c_int32
        _lib.or_dcore.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_int, i32p, i32p,
                                  ctypes.c_uint64, i32p, i32p]
        _lib.or_dcore.restype = ctypes.c_int
        _lib.or_kedge_batches.argtypes = [ctypes.c_uint32, i32p, ctypes.c_uint64, u32p, u32p, i64p]
        _lib.or_kedge_batches.restype = ctypes.c_int64
        _lib.og_gen_er.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, u32p, u32p]
        _lib.og_gen_er.restype = ctypes.c_int
        _lib.og_gen_rmat.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, u32p, u32p,
                                     ctypes.POINTER(ctypes.c_uint64)]
        _lib.og_gen_rmat.restype = ctypes.c_int
    return _lib


def _u32(a):
    return np.ascontiguousarray(a, np.uint32)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def peel_levels(V, src, dst, swap, k):
    """Literal restatement of one reference pass; returns (last level, core[V])."""
    src, dst = _u32(src), _u32(dst)
    core = np.empty(max(V, 1), np.int32)
    lvl = lib().or_peel_levels(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), int(swap), k, _ptr(core, i32p))
    return lvl, core[:V]


def dcore_levels(V, src, dst):
    """dcore() with the literal level-loop pass for every row (small graphs)."""
    kmax, kmaxes = peel_levels(V, dst, src, 0, 0)  # swapped k = 0 pass
    kmax = max(kmax, 0)
    rows = []
    lmax = 0
    for k in range(kmax + 1):
        l, row = peel_levels(V, src, dst, 0, k)
        lmax = max(lmax, l)
        rows.append(row)
    return kmax, lmax, kmaxes, np.stack(rows) if rows else np.zeros((1, V), np.int32)


def dcore(V, src, dst, threads=0):
    """Bucket-queue decomposition: (kmax, lmax, kmaxes[V], rows[kmax+1, V])."""
    src, dst = _u32(src), _u32(dst)
    kmaxes = np.empty(max(V, 1), np.int32)
    km = ctypes.c_int32(0)
    lm = ctypes.c_int32(0)
    rc = lib().or_dcore(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), threads, _ptr(kmaxes, i32p), None, 0,
                        ctypes.byref(km), ctypes.byref(lm))
    if rc not in (0, -5):
        raise RuntimeError(f"oracle or_dcore failed: {rc}")
    rows = np.empty((km.value + 1, max(V, 1)), np.int32)
    rc = lib().or_dcore(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), threads, _ptr(kmaxes, i32p),
                        _ptr(rows, i32p), km.value + 1, ctypes.byref(km), ctypes.byref(lm))
    if rc != 0:
        raise RuntimeError(f"oracle or_dcore failed: {rc}")
    return km.value, lm.value, kmaxes[:V], rows[:, :V]


def dcore_timed(V, src, dst, threads=0, rows=None):
    """One full decomposition timed from the built CSR/CSC to the last row:
    (kmax, lmax, kmaxes[V], rows[kmax+1, V], seconds, threads used).  rows
    may be a preallocated int32 array of at least (kmax+1) * V values, so
    that repeated calls do not allocate; it is sized by a kmax pass when
    None or too small."""
    L = lib()
    L.or_dcore_timed.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_int, i32p, i32p,
                                 ctypes.c_uint64, i32p, i32p, ctypes.POINTER(ctypes.c_double)]
    L.or_dcore_timed.restype = ctypes.c_int
    src, dst = _u32(src), _u32(dst)
    kmaxes = np.empty(max(V, 1), np.int32)
    km = ctypes.c_int32(0)
    lm = ctypes.c_int32(0)
    secs = ctypes.c_double(0)
    nt = threads if threads > 0 else max_threads()
    cap = 0 if rows is None else rows.size // max(V, 1)
    if rows is None or cap == 0:
        _, kmaxes_ = kmax(V, src, dst)
        cap = int(kmaxes_.max()) + 1 if V else 1
        rows = np.empty(cap * max(V, 1), np.int32)
    rc = L.or_dcore_timed(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), nt, _ptr(kmaxes, i32p),
                          rows.ctypes.data_as(i32p), cap, ctypes.byref(km), ctypes.byref(lm), ctypes.byref(secs))
    if rc == -5:  # the preallocated rows were too small: size them and run again
        rows = np.empty((km.value + 1) * max(V, 1), np.int32)
        return dcore_timed(V, src, dst, threads, rows)
    if rc != 0:
        raise RuntimeError(f"oracle or_dcore_timed failed: {rc}")
    K = km.value
    out = rows[:(K + 1) * max(V, 1)].reshape(K + 1, max(V, 1))[:, :V]
    return K, lm.value, kmaxes[:V], out, secs.value, nt


class BuiltGraph:
    """The oracle's CSR/CSC of one graph, built once, for checking a large
    decomposition a chunk of rows at a time (or_graph_new / or_graph_rows)."""

    def __init__(self, V, src, dst):
        L = lib()
        L.or_graph_new.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p]
        L.or_graph_new.restype = ctypes.c_void_p
        L.or_graph_delete.argtypes = [ctypes.c_void_p]
        L.or_graph_delete.restype = None
        L.or_graph_kmax.argtypes = [ctypes.c_void_p, i32p]
        L.or_graph_kmax.restype = ctypes.c_int32
        L.or_graph_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, i32p, ctypes.c_int32, ctypes.c_int32, i32p]
        L.or_graph_rows.restype = ctypes.c_int
        src, dst = _u32(src), _u32(dst)
        self.V = V
        self._g = L.or_graph_new(V, len(src), _ptr(src, u32p), _ptr(dst, u32p))
        if not self._g:
            raise RuntimeError("oracle or_graph_new failed")

    def kmax(self):
        out = np.empty(max(self.V, 1), np.int32)
        km = lib().or_graph_kmax(self._g, _ptr(out, i32p))
        return km, out[:self.V]

    def rows(self, kmaxes, k0, k1, threads=0, out=None):
        """Rows k0..k1-1 as an array [(k1 - k0), V]."""
        kmaxes = np.ascontiguousarray(kmaxes, np.int32)
        n = max(k1 - k0, 0)
        if out is None or out.size < n * max(self.V, 1):
            out = np.empty(n * max(self.V, 1), np.int32)
        rc = lib().or_graph_rows(self._g, threads, _ptr(kmaxes, i32p), k0, k1, out.ctypes.data_as(i32p))
        if rc:
            raise RuntimeError(f"oracle or_graph_rows failed: {rc}")
        return out[:n * max(self.V, 1)].reshape(n, max(self.V, 1))[:, :self.V]

    def close(self):
        if self._g:
            lib().or_graph_delete(self._g)
            self._g = None

    def __del__(self):
        self.close()


def kmax(V, src, dst):
    src, dst = _u32(src), _u32(dst)
    out = np.empty(max(V, 1), np.int32)
    km = lib().or_kmax(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), _ptr(out, i32p))
    return km, out[:V]


def row(V, src, dst, kmaxes, k):
    src, dst = _u32(src), _u32(dst)
    kmaxes = np.ascontiguousarray(kmaxes, np.int32)
    out = np.empty(max(V, 1), np.int32)
    l = lib().or_bz_row(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), _ptr(kmaxes, i32p), k, _ptr(out, i32p))
    return l, out[:V]


def kedge_batches(V, kmaxes, frm, to):
    """getKmaxEdgeBatches (KEDGE_BATCHING): sub-batch index of every edge."""
    frm, to = _u32(frm), _u32(to)
    kmaxes = np.ascontiguousarray(kmaxes, np.int32)
    out = np.empty(max(len(frm), 1), np.int64)
    nb = lib().or_kedge_batches(V, _ptr(kmaxes, i32p), len(frm), _ptr(frm, u32p), _ptr(to, u32p), _ptr(out, i64p))
    return nb, out[:len(frm)]


def rows_sample(V, src, dst, kmaxes, kmax, stride, threads=0):
    """Computes rows 0, stride, ... <= kmax in parallel; returns (rows
    computed, summed per-row seconds)."""
    L = lib()
    L.or_rows_sample.argtypes = [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_int, i32p, ctypes.c_int32,
                                 ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    L.or_rows_sample.restype = ctypes.c_int64
    src, dst = _u32(src), _u32(dst)
    kmaxes = np.ascontiguousarray(kmaxes, np.int32)
    secs = ctypes.c_double(0)
    n = L.or_rows_sample(V, len(src), _ptr(src, u32p), _ptr(dst, u32p), threads, _ptr(kmaxes, i32p), kmax, stride,
                         ctypes.byref(secs))
    if n < 0:
        raise RuntimeError(f"oracle or_rows_sample failed: {n}")
    return n, secs.value


def gen_er(n, m, seed):
    """Seeded directed G(n, m), sorted by (src, dst): the engine's dc_gen_er
    restated (gen_oracle.c)."""
    src = np.empty(max(m, 1), np.uint32)
    dst = np.empty(max(m, 1), np.uint32)
    rc = lib().og_gen_er(n, m, seed, _ptr(src, u32p), _ptr(dst, u32p))
    if rc:
        raise RuntimeError(f"oracle og_gen_er failed: {rc}")
    return src[:m], dst[:m]


def gen_rmat(scale, edge_factor, seed, a=0.57, b=0.19, c=0.19, permute=True):
    """Seeded R-MAT (self-loops and duplicates removed, labels permuted), the
    engine's dc_gen_rmat restated (gen_oracle.c): (V, src, dst)."""
    cap = edge_factor << scale
    src = np.empty(max(cap, 1), np.uint32)
    dst = np.empty(max(cap, 1), np.uint32)
    n = ctypes.c_uint64(0)
    rc = lib().og_gen_rmat(scale, edge_factor, a, b, c, seed, int(permute), cap, _ptr(src, u32p), _ptr(dst, u32p),
                           ctypes.byref(n))
    if rc:
        raise RuntimeError(f"oracle og_gen_rmat failed: {rc}")
    return 1 << scale, src[:n.value], dst[:n.value]


def max_threads():
    L = lib()
    L.or_max_threads.restype = ctypes.c_int
    return L.or_max_threads()
