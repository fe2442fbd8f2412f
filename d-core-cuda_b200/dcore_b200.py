"""Python binding of the d-core-b200 C ABI (include/dcore_b200.h).

A thin ctypes layer over libdcore_b200.so: numpy arrays in, numpy arrays out.
It mirrors the reference's host interface for the load -> decompose ->
maintain path (Graph, dcore, maintenanceFast in llysdal/d-core-cuda) so that
tests and the benchmark read like the reference's own driver.  There is no
CPU fallback: compute calls fail with DCoreError when the library or a CUDA
device is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdcore_b200.so")

DC_OK = 0
ERR_NAMES = {
    -1: "DC_ERR_INVALID", -2: "DC_ERR_CUDA", -3: "DC_ERR_NOMEM", -4: "DC_ERR_IO", -5: "DC_ERR_CAPACITY",
    -6: "DC_ERR_TIMEOUT", -7: "DC_ERR_NOT_FOUND", -8: "DC_ERR_STATE", -9: "DC_ERR_NO_DEVICE",
}
METHOD_INCREMENTAL = 0
METHOD_PEEL = 1


class DCoreError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None

u32p = ctypes.POINTER(ctypes.c_uint32)
i32p = ctypes.POINTER(ctypes.c_int32)
u64p = ctypes.POINTER(ctypes.c_uint64)
i64p = ctypes.POINTER(ctypes.c_int64)
u8p = ctypes.POINTER(ctypes.c_uint8)
f32p = ctypes.POINTER(ctypes.c_float)
vp = ctypes.c_void_p


class GraphOpts(ctypes.Structure):
    _fields_ = [("gap_min", ctypes.c_uint32), ("gap_div", ctypes.c_uint32), ("device", ctypes.c_int32)]


class DecompInfo(ctypes.Structure):
    _fields_ = [("kmax", ctypes.c_int32), ("lmax", ctypes.c_int32), ("n_corners", ctypes.c_uint64),
                ("kmax_ms", ctypes.c_float), ("row0_ms", ctypes.c_float), ("rows_ms", ctypes.c_float),
                ("skyline_ms", ctypes.c_float), ("expand_ms", ctypes.c_float),
                ("evals", ctypes.c_uint64), ("drops", ctypes.c_uint64), ("entries", ctypes.c_uint64)]


class MaintStats(ctypes.Structure):
    _fields_ = [("inserted", ctypes.c_uint64), ("deleted", ctypes.c_uint64), ("kmax", ctypes.c_int32),
                ("lmax", ctypes.c_int32), ("rows_recomputed", ctypes.c_int32), ("method", ctypes.c_int32),
                ("rebuilt", ctypes.c_uint32), ("rows_local", ctypes.c_uint32), ("region", ctypes.c_uint64),
                ("apply_ms", ctypes.c_float), ("core_ms", ctypes.c_float), ("rows_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("del_repair_ms", ctypes.c_float), ("ins_repair_ms", ctypes.c_float),
                ("ins_scanned", ctypes.c_uint64), ("captured", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


MAINT_AUTO, MAINT_LOCAL, MAINT_REPEEL = 0, 1, 2


class Tuning(ctypes.Structure):
    _fields_ = [("peel_blocks_per_sm", ctypes.c_int32), ("rows_blocks_per_sm", ctypes.c_int32),
                ("peel_chunk", ctypes.c_int32), ("rows_split_permille", ctypes.c_int32 * 7)]

    def as_dict(self):
        return {"peel_blocks_per_sm": self.peel_blocks_per_sm, "rows_blocks_per_sm": self.rows_blocks_per_sm,
                "peel_chunk": self.peel_chunk, "rows_split_permille": list(self.rows_split_permille)}


class ServerInfo(ctypes.Structure):
    _fields_ = [("budget_bytes", ctypes.c_uint64), ("used_bytes", ctypes.c_uint64), ("peak_bytes", ctypes.c_uint64),
                ("admissions", ctypes.c_uint64), ("evictions", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("measured_bytes", ctypes.c_uint64),
                ("graphs", ctypes.c_uint32),
                ("resident", ctypes.c_uint32)]

# name -> argtypes; every function returns int status unless listed in _VOID / _STR
SIGNATURES = {
    "dc_gen_er": [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64, u32p, u32p],
    "dc_gen_rmat": [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                    ctypes.c_uint64, ctypes.c_int, ctypes.c_uint64, u32p, u32p, u64p],
    "dc_kmax_edge_batches": [ctypes.c_uint32, i32p, ctypes.c_uint64, u32p, u32p, i64p, i64p],
    "dc_gen_updates": [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_uint64, ctypes.c_double,
                       ctypes.c_uint64, u32p, u32p, u8p],
    "dc_gen_updates_hot": [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_uint64, ctypes.c_double,
                           ctypes.c_uint64, u32p, ctypes.c_uint32, u8p, u32p, u32p, u8p],
    "dc_text_read_edges": [ctypes.c_char_p, ctypes.c_int, u32p, u64p, u32p, u32p, ctypes.c_uint64],
    "dc_binary_read_edges": [ctypes.c_char_p, u32p, u64p, u32p, u32p, ctypes.c_uint64],
    "dc_binary_write_edges": [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.c_uint32],
    "dc_decomp_file_write": [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_int32, ctypes.c_int32, i32p, i32p],
    "dc_decomp_file_read": [ctypes.c_char_p, ctypes.c_uint32, i32p, i32p, i32p, i32p, ctypes.c_uint64],
    "dc_decomp_cpu_file_write": [ctypes.c_char_p, ctypes.c_uint32, i32p, i32p],
    "dc_graph_opts_default": [ctypes.POINTER(GraphOpts)],
    "dc_device_count": [ctypes.POINTER(ctypes.c_int)],
    "dc_graph_create": [ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, ctypes.POINTER(GraphOpts), ctypes.POINTER(vp)],
    "dc_graph_create_device": [ctypes.c_uint32, ctypes.c_uint64, vp, vp, ctypes.POINTER(GraphOpts),
                               ctypes.POINTER(vp)],
    "dc_graph_load": [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(GraphOpts), ctypes.POINTER(vp)],
    "dc_graph_free": [vp],
    "dc_graph_info": [vp, u32p, u64p],
    "dc_graph_degrees": [vp, i32p, i32p],
    "dc_graph_get_edges": [vp, u32p, u32p, ctypes.c_uint64, u64p],
    "dc_graph_write_binary": [vp, ctypes.c_char_p, ctypes.c_uint32],
    "dc_decompose": [vp, ctypes.c_int, i32p, i32p],
    "dc_decompose_rows": [vp, ctypes.c_uint32, ctypes.c_uint32, i32p, i32p],
    "dc_row_weights": [vp, u64p, ctypes.c_uint64],
    "dc_set_row_repair": [vp, ctypes.c_int],
    "dc_set_captured_batches": [vp, ctypes.c_int],
    "dc_reserve_device_memory": [ctypes.c_int, ctypes.c_uint64],
    "dc_maintain": [vp, u32p, u8p, ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(MaintStats)],
    "dc_decomp_info_get": [vp, ctypes.POINTER(DecompInfo)],
    "dc_get_kmaxes": [vp, i32p],
    "dc_get_lmax_rows": [vp, ctypes.c_uint32, ctypes.c_uint32, i32p],
    "dc_get_lmax_rows_device": [vp, ctypes.c_uint32, ctypes.c_uint32, vp],
    "dc_materialize_rows": [vp],
    "dc_release_rows": [vp],
    "dc_get_skyline": [vp, u32p, i32p, i32p, ctypes.c_uint64, u64p],
    "dc_write_decomp": [vp, ctypes.c_char_p],
    "dc_write_decomp_cpu": [vp, ctypes.c_char_p],
    "dc_host_alloc": [ctypes.c_uint64, ctypes.POINTER(vp)],
    "dc_host_free": [vp],
    "dc_synchronize": [vp],
    "dc_graph_stream": [vp, ctypes.POINTER(vp)],
    "dc_set_trace": [vp, ctypes.c_uint32, vp, vp],
    "dc_set_launch": [vp, ctypes.c_int],
    "dc_get_tuning": [vp, ctypes.POINTER(Tuning)],
    "dc_set_tuning": [vp, ctypes.POINTER(Tuning)],
    "dc_autotune": [vp, ctypes.POINTER(Tuning), ctypes.POINTER(ctypes.c_float)],
    "dc_sched_create": [ctypes.c_uint64, ctypes.POINTER(vp)],
    "dc_sched_free": [vp],
    "dc_sched_param_count": [],
    "dc_sched_get_params": [vp, ctypes.POINTER(ctypes.c_float)],
    "dc_sched_set_params": [vp, ctypes.POINTER(ctypes.c_float)],
    "dc_sched_set_norm": [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "dc_sched_predict": [vp, ctypes.POINTER(ctypes.c_float), ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)],
    "dc_sched_grad": [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), u8p, ctypes.c_uint64,
                      ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "dc_sched_train": [vp, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), u8p, ctypes.c_uint64,
                       ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_float)],
    "dc_graph_set_scheduler": [vp, vp],
    "dc_maint_log_enable": [vp, ctypes.c_int],
    "dc_maint_log_get": [vp, ctypes.POINTER(ctypes.c_float), i32p, ctypes.POINTER(ctypes.c_float), ctypes.c_uint64,
                         u64p],
    "dc_graph_device_bytes": [vp, u64p],
    "dc_server_create": [ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)],
    "dc_server_add_graph": [vp, ctypes.c_uint32, ctypes.c_uint64, u32p, u32p, u32p],
    "dc_server_submit": [vp, ctypes.c_uint32, u32p, u8p, ctypes.c_uint64, u64p],
    "dc_server_drain": [vp, ctypes.c_uint64],
    "dc_server_completions": [vp, u64p, u32p, ctypes.POINTER(ctypes.c_double), u32p, u64p, i32p, ctypes.c_uint64,
                              u64p],
    "dc_server_info_get": [vp, ctypes.POINTER(ServerInfo)],
    "dc_server_graph_result": [vp, ctypes.c_uint32, i32p, i32p, ctypes.c_uint64, i32p],
    "dc_server_free": [vp],
    "dc_server_set_row_repair": [vp, ctypes.c_int],
    "dc_set_wait_limit": [vp, ctypes.c_uint64],
    "dc_test_withhold_barrier": [vp, ctypes.c_int32],
    "dc_graph_kmax_edge_batches": [vp, ctypes.c_uint64, vp, vp, vp, ctypes.POINTER(ctypes.c_int64)],
    "dc_graph_load_text_device": [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(GraphOpts), ctypes.POINTER(vp)],
    "dc_write_decomp_cpu_device": [vp, ctypes.c_char_p],
    "dc_kmax_noalloc": [ctypes.c_uint32, ctypes.c_uint64, vp, vp, vp, vp, i32p, vp],
    "dc_plan_row_cuts": [i32p, f32p, ctypes.c_int32, ctypes.c_float, ctypes.c_int32, i32p, f32p],
    "dc_launch_count": [u64p],
    "dc_last_error": [],
    "dc_version": [],
}
_VOID = {"dc_graph_opts_default"}
_STR = {"dc_last_error", "dc_version"}


def lib():
    """Loads libdcore_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise DCoreError(-9, f"{LIB_PATH} is not built; run d-core-cuda_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        if not hasattr(L, name):
            continue
        f = getattr(L, name)
        f.argtypes = args
        f.restype = None if name in _VOID else (ctypes.c_char_p if name in _STR else ctypes.c_int)
    _lib = L
    return L


def _check(rc):
    if rc != DC_OK:
        raise DCoreError(rc, lib().dc_last_error().decode())


def _p(a, t):
    return a.ctypes.data_as(t)


def last_error():
    return lib().dc_last_error().decode()


def launch_count():
    n = ctypes.c_uint64(0)
    _check(lib().dc_launch_count(ctypes.byref(n)))
    return n.value


def plan_row_cuts(grid, cost, total, ncut):
    """dc_plan_row_cuts: the ncut grid values (per mille of kmax) whose
    segments' largest predicted cost is smallest; returns (cuts, that cost)."""
    g = np.ascontiguousarray(grid, np.int32)
    c = np.ascontiguousarray(cost, np.float32)
    out = np.zeros(max(int(ncut), 1), np.int32)
    lo = ctypes.c_float(0)
    _check(lib().dc_plan_row_cuts(_p(g, i32p), _p(c, f32p), len(g), float(total), int(ncut), _p(out, i32p),
                                  ctypes.byref(lo)))
    return out[:ncut].tolist(), lo.value


def device_count():
    n = ctypes.c_int(0)
    _check(lib().dc_device_count(ctypes.byref(n)))
    return n.value


def reserve_device_memory(device, nbytes):
    """Grow the device's memory pool (which the engine allocates from) to at
    least nbytes, so later calls map no new memory."""
    _check(lib().dc_reserve_device_memory(int(device), int(nbytes)))


# ---------------------------------------------------------------- pinned host memory
_PINNED = {}


def pinned_array(n, dtype):
    """numpy array of n elements in pinned host memory (dc_host_alloc); it
    stays allocated until free_pinned(arr) or process exit."""
    dt = np.dtype(dtype)
    nbytes = max(int(n) * dt.itemsize, 1)
    p = vp()
    _check(lib().dc_host_alloc(nbytes, ctypes.byref(p)))
    buf = (ctypes.c_uint8 * nbytes).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dt, count=int(n))
    _PINNED[arr.ctypes.data] = (p.value, buf)
    return arr


def free_pinned(arr):
    ent = _PINNED.pop(arr.ctypes.data, None)
    if ent:
        lib().dc_host_free(vp(ent[0]))


# ---------------------------------------------------------------- generators
def gen_er(n, m, seed):
    """Seeded directed G(n, m), sorted by (src, dst)."""
    src = np.empty(max(m, 1), np.uint32)
    dst = np.empty(max(m, 1), np.uint32)
    _check(lib().dc_gen_er(n, m, seed, _p(src, u32p), _p(dst, u32p)))
    return src[:m], dst[:m]


def gen_rmat(scale, edge_factor, seed, a=0.57, b=0.19, c=0.19, permute=True):
    """Seeded R-MAT graph, self-loops and duplicates removed, sorted by (src, dst)."""
    cap = edge_factor << scale
    src = np.empty(max(cap, 1), np.uint32)
    dst = np.empty(max(cap, 1), np.uint32)
    n = ctypes.c_uint64(0)
    _check(lib().dc_gen_rmat(scale, edge_factor, a, b, c, seed, int(permute), cap, _p(src, u32p), _p(dst, u32p),
                             ctypes.byref(n)))
    return 1 << scale, src[:n.value], dst[:n.value]


def gen_updates(V, src, dst, n_ops, insert_frac, seed):
    """Seeded valid-in-sequence update stream: (u, v, is_delete) arrays."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    u = np.empty(max(n_ops, 1), np.uint32)
    v = np.empty(max(n_ops, 1), np.uint32)
    dl = np.empty(max(n_ops, 1), np.uint8)
    _check(lib().dc_gen_updates(V, len(src), _p(src, u32p), _p(dst, u32p), n_ops, insert_frac, seed, _p(u, u32p),
                                _p(v, u32p), _p(dl, u8p)))
    return u[:n_ops], v[:n_ops], dl[:n_ops]


def gen_updates_hot(V, src, dst, n_ops, insert_frac, seed, hot, op_hot):
    """gen_updates where operations marked in op_hot have their source among
    the vertices `hot`."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    hot = np.ascontiguousarray(hot, np.uint32)
    op_hot = np.ascontiguousarray(op_hot, np.uint8)
    assert len(op_hot) == n_ops
    u = np.empty(max(n_ops, 1), np.uint32)
    v = np.empty(max(n_ops, 1), np.uint32)
    dl = np.empty(max(n_ops, 1), np.uint8)
    _check(lib().dc_gen_updates_hot(V, len(src), _p(src, u32p), _p(dst, u32p), n_ops, insert_frac, seed,
                                    _p(hot, u32p), len(hot), _p(op_hot, u8p), _p(u, u32p), _p(v, u32p),
                                    _p(dl, u8p)))
    return u[:n_ops], v[:n_ops], dl[:n_ops]


def kmax_edge_batches(kmaxes, frm, to):
    """getKmaxEdgeBatches (KEDGE_BATCHING): (number of sub-batches, sub-batch of every edge)."""
    kmaxes = np.ascontiguousarray(kmaxes, np.int32)
    frm = np.ascontiguousarray(frm, np.uint32)
    to = np.ascontiguousarray(to, np.uint32)
    out = np.empty(max(len(frm), 1), np.int64)
    nb = ctypes.c_int64(0)
    _check(lib().dc_kmax_edge_batches(len(kmaxes), _p(kmaxes, i32p), len(frm), _p(frm, u32p), _p(to, u32p),
                                      _p(out, i64p), ctypes.byref(nb)))
    return nb.value, out[:len(frm)]


# ---------------------------------------------------------------- file formats
def read_text_edges(path, prune=True):
    V = ctypes.c_uint32(0)
    E = ctypes.c_uint64(0)
    _check(lib().dc_text_read_edges(path.encode(), int(prune), ctypes.byref(V), ctypes.byref(E), None, None, 0))
    src = np.empty(max(E.value, 1), np.uint32)
    dst = np.empty(max(E.value, 1), np.uint32)
    _check(lib().dc_text_read_edges(path.encode(), int(prune), ctypes.byref(V), ctypes.byref(E), _p(src, u32p),
                                    _p(dst, u32p), E.value))
    return V.value, src[:E.value], dst[:E.value]


def read_binary_edges(path):
    V = ctypes.c_uint32(0)
    E = ctypes.c_uint64(0)
    _check(lib().dc_binary_read_edges(path.encode(), ctypes.byref(V), ctypes.byref(E), None, None, 0))
    src = np.empty(max(E.value, 1), np.uint32)
    dst = np.empty(max(E.value, 1), np.uint32)
    _check(lib().dc_binary_read_edges(path.encode(), ctypes.byref(V), ctypes.byref(E), _p(src, u32p),
                                      _p(dst, u32p), E.value))
    return V.value, src[:E.value], dst[:E.value]


def write_binary_edges(path, V, src, dst, gap=1):
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    _check(lib().dc_binary_write_edges(path.encode(), V, len(src), _p(src, u32p), _p(dst, u32p), gap))


def write_decomp_file(path, kmax, lmax, kmaxes, rows):
    kmaxes = np.ascontiguousarray(kmaxes, np.int32)
    rows = np.ascontiguousarray(rows, np.int32)
    _check(lib().dc_decomp_file_write(path.encode(), len(kmaxes), kmax, lmax, _p(kmaxes, i32p), _p(rows, i32p)))


def read_decomp_file(path, V):
    km = ctypes.c_int32(0)
    lm = ctypes.c_int32(0)
    _check(lib().dc_decomp_file_read(path.encode(), V, ctypes.byref(km), ctypes.byref(lm), None, None, 0))
    kmaxes = np.empty(max(V, 1), np.int32)
    rows = np.empty(max((km.value + 1) * V, 1), np.int32)
    _check(lib().dc_decomp_file_read(path.encode(), V, ctypes.byref(km), ctypes.byref(lm), _p(kmaxes, i32p),
                                     _p(rows, i32p), rows.size))
    return km.value, lm.value, kmaxes[:V], rows[:(km.value + 1) * V].reshape(km.value + 1, V)


def write_decomp_cpu_file(path, kmaxes, rows):
    kmaxes = np.ascontiguousarray(kmaxes, np.int32)
    rows = np.ascontiguousarray(rows, np.int32)
    _check(lib().dc_decomp_cpu_file_write(path.encode(), len(kmaxes), _p(kmaxes, i32p), _p(rows, i32p)))


# ---------------------------------------------------------------- graphs
class Graph:
    """A device-resident graph handle (Graph / GraphGPU in the reference)."""

    def __init__(self, handle):
        self._h = vp(handle)

    @staticmethod
    def _opts(gap_min=1, gap_div=0, device=-1):
        o = GraphOpts()
        lib().dc_graph_opts_default(ctypes.byref(o))
        o.gap_min, o.gap_div, o.device = gap_min, gap_div, device
        return o

    @classmethod
    def from_edges(cls, V, src, dst, gap_min=1, gap_div=0, device=-1):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        h = vp()
        o = cls._opts(gap_min, gap_div, device)
        _check(lib().dc_graph_create(V, len(src), _p(src, u32p), _p(dst, u32p), ctypes.byref(o), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def from_device_edges(cls, V, E, d_src_ptr, d_dst_ptr, gap_min=1, gap_div=0, device=-1):
        h = vp()
        o = cls._opts(gap_min, gap_div, device)
        _check(lib().dc_graph_create_device(V, E, vp(d_src_ptr), vp(d_dst_ptr), ctypes.byref(o), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def load_text_device(cls, path, prune=True, gap_min=1, gap_div=0, device=-1):
        """Text graph parsed on the GPU (dc_graph_load_text_device)."""
        h = vp()
        o = cls._opts(gap_min, gap_div, device)
        _check(lib().dc_graph_load_text_device(path.encode(), int(prune), ctypes.byref(o), ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def load(cls, path, prune=True, gap_min=1, gap_div=0, device=-1):
        h = vp()
        o = cls._opts(gap_min, gap_div, device)
        _check(lib().dc_graph_load(path.encode(), int(prune), ctypes.byref(o), ctypes.byref(h)))
        return cls(h.value)

    def free(self):
        if self._h and self._h.value:
            lib().dc_graph_free(self._h)
            self._h = vp()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    @property
    def handle(self):
        return self._h

    def info(self):
        V = ctypes.c_uint32(0)
        E = ctypes.c_uint64(0)
        _check(lib().dc_graph_info(self._h, ctypes.byref(V), ctypes.byref(E)))
        return V.value, E.value

    @property
    def V(self):
        return self.info()[0]

    def degrees(self):
        V = self.V
        i = np.empty(max(V, 1), np.int32)
        o = np.empty(max(V, 1), np.int32)
        _check(lib().dc_graph_degrees(self._h, _p(i, i32p), _p(o, i32p)))
        return i[:V], o[:V]

    def edges(self):
        n = ctypes.c_uint64(0)
        _check(lib().dc_graph_get_edges(self._h, None, None, 0, ctypes.byref(n)))
        s = np.empty(max(n.value, 1), np.uint32)
        d = np.empty(max(n.value, 1), np.uint32)
        _check(lib().dc_graph_get_edges(self._h, _p(s, u32p), _p(d, u32p), n.value, ctypes.byref(n)))
        return s[:n.value], d[:n.value]

    def write_binary(self, path, gap=1):
        _check(lib().dc_graph_write_binary(self._h, path.encode(), gap))

    # ---- decomposition
    def device_bytes(self):
        n = ctypes.c_uint64(0)
        _check(lib().dc_graph_device_bytes(self._h, ctypes.byref(n)))
        return n.value

    def decompose(self, method=METHOD_INCREMENTAL):
        km = ctypes.c_int32(0)
        lm = ctypes.c_int32(0)
        _check(lib().dc_decompose(self._h, method, ctypes.byref(km), ctypes.byref(lm)))
        return km.value, lm.value

    def decompose_rows(self, k_first, k_last):
        """kmax, row 0 and rows max(k_first, 1)..k_last only (row sharding);
        k_first = 0 recomputes kmax and row 0 even when current; an empty
        range computes (or keeps) kmax and row 0 alone."""
        km = ctypes.c_int32(0)
        lm = ctypes.c_int32(0)
        k_last = max(k_last, 0)
        _check(lib().dc_decompose_rows(self._h, k_first, k_last, ctypes.byref(km), ctypes.byref(lm)))
        return km.value, lm.value

    def row_weights(self):
        """weights[k] = total degree of the vertices with kmax >= k."""
        K = self.decomp_info()["kmax"]
        w = np.zeros(K + 1, np.uint64)
        _check(lib().dc_row_weights(self._h, _p(w, u64p), K + 1))
        return w

    def maintain(self, src, dst, is_delete=None, method=MAINT_AUTO):
        """maintenanceFast: applies the update batch; returns the stats dict."""
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        pairs = np.empty(2 * len(src), np.uint32)
        pairs[0::2] = src
        pairs[1::2] = dst
        dl = None
        if is_delete is not None:
            dl = np.ascontiguousarray(is_delete, np.uint8)
        st = MaintStats()
        _check(lib().dc_maintain(self._h, _p(pairs, u32p), None if dl is None else _p(dl, u8p), len(src), method,
                                 ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in MaintStats._fields_}

    def set_captured_batches(self, on):
        """Run eligible maintenance batches as one captured CUDA graph (default on)."""
        _check(lib().dc_set_captured_batches(self._h, 1 if on else 0))

    def set_row_repair(self, mode):
        """0 recompute rows, 1 repair deletions in place when worthwhile, 2 always when they fit."""
        _check(lib().dc_set_row_repair(self._h, int(mode)))

    def set_scheduler(self, sched):
        _check(lib().dc_graph_set_scheduler(self._h, sched.handle if sched is not None else None))
        self._sched_ref = sched

    def maint_log(self, enable=None):
        """With enable=True/False switches logging; returns (features[n,16], methods[n], times_ms[n,3])."""
        if enable is not None:
            _check(lib().dc_maint_log_enable(self._h, int(enable)))
        n = ctypes.c_uint64(0)
        _check(lib().dc_maint_log_get(self._h, None, None, None, 0, ctypes.byref(n)))
        f = np.empty((max(n.value, 1), 16), np.float32)
        m = np.empty(max(n.value, 1), np.int32)
        t = np.empty((max(n.value, 1), 3), np.float32)
        _check(lib().dc_maint_log_get(self._h, _p(f, f32p), _p(m, i32p), _p(t, f32p), n.value, ctypes.byref(n)))
        return f[:n.value], m[:n.value], t[:n.value]

    def decomp_info(self):
        info = DecompInfo()
        _check(lib().dc_decomp_info_get(self._h, ctypes.byref(info)))
        return {f: getattr(info, f) for f, _ in DecompInfo._fields_}

    def kmaxes(self, out=None):
        V = self.V
        if out is None:
            out = np.empty(max(V, 1), np.int32)
        _check(lib().dc_get_kmaxes(self._h, _p(out, i32p)))
        return out[:V]

    def rows(self, k0=0, n=None, out=None):
        """Dense rows k0..k0+n-1 of lmaxes as an (n, V) int32 array."""
        V = self.V
        if n is None:
            n = self.decomp_info()["kmax"] + 1 - k0
        if out is None:
            out = np.empty((n, V), np.int32)
        if n and V:
            _check(lib().dc_get_lmax_rows(self._h, k0, n, _p(out, i32p)))
        return out

    def rows_to_device(self, k0, n, d_ptr):
        _check(lib().dc_get_lmax_rows_device(self._h, k0, n, vp(d_ptr)))

    def materialize_rows(self):
        _check(lib().dc_materialize_rows(self._h))

    def release_rows(self):
        _check(lib().dc_release_rows(self._h))

    def skyline(self):
        n = ctypes.c_uint64(0)
        _check(lib().dc_get_skyline(self._h, None, None, None, 0, ctypes.byref(n)))
        V = self.V
        off = np.empty(V + 1, np.uint32)
        ks = np.empty(max(n.value, 1), np.int32)
        ls = np.empty(max(n.value, 1), np.int32)
        _check(lib().dc_get_skyline(self._h, _p(off, u32p), _p(ks, i32p), _p(ls, i32p), n.value, ctypes.byref(n)))
        return off, ks[:n.value], ls[:n.value]

    def write_decomp(self, path):
        _check(lib().dc_write_decomp(self._h, path.encode()))

    def write_decomp_cpu(self, path):
        _check(lib().dc_write_decomp_cpu(self._h, path.encode()))

    def set_trace(self, max_steps, callback):
        """callback(phase, records[steps, 4] uint64) after each persistent kernel."""
        if callback is None:
            _check(lib().dc_set_trace(self._h, 0, None, None))
            self._trace_cb = None
            return
        CB = ctypes.CFUNCTYPE(None, ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint, ctypes.c_void_p)

        def _cb(phase, rec, steps, user):
            arr = np.ctypeslib.as_array(rec, shape=(max_steps * 8,)).reshape(max_steps, 8)[:steps].copy()
            callback(phase.decode(), arr)
        self._trace_cb = CB(_cb)
        _check(lib().dc_set_trace(self._h, max_steps, ctypes.cast(self._trace_cb, vp), None))

    def tuning(self):
        t = Tuning()
        _check(lib().dc_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, peel_blocks_per_sm=2, rows_blocks_per_sm=2, peel_chunk=64, rows_split_permille=()):
        """rows_split_permille: up to seven ascending cuts (per mille of kmax)
        splitting a full run of rows into concurrent launches; () = none."""
        cuts = [rows_split_permille] if isinstance(rows_split_permille, int) else list(rows_split_permille)
        if len(cuts) > 7:
            raise DCoreError(-1, "at most seven row cuts")
        t = Tuning(peel_blocks_per_sm, rows_blocks_per_sm, peel_chunk, (ctypes.c_int32 * 7)(*(cuts + [0] * (7 - len(cuts)))))
        _check(lib().dc_set_tuning(self._h, ctypes.byref(t)))

    def autotune(self):
        """Picks the fastest launch shapes for this graph (dc_autotune);
        returns (setting, its peel + rows device ms)."""
        t = Tuning()
        ms = ctypes.c_float(0)
        _check(lib().dc_autotune(self._h, ctypes.byref(t), ctypes.byref(ms)))
        return t.as_dict(), ms.value

    def set_launch(self, blocks_per_sm):
        _check(lib().dc_set_launch(self._h, blocks_per_sm))

    def kmax_edge_batches_device(self, d_from_ptr, d_to_ptr, B, d_batch_of_ptr):
        """getKmaxEdgeBatches (KEDGE_BATCHING) on the GPU by the graph's
        current kmax: device arrays in and out; returns the number of
        sub-batches."""
        n = ctypes.c_int64(0)
        _check(lib().dc_graph_kmax_edge_batches(self._h, int(B), vp(d_from_ptr), vp(d_to_ptr), vp(d_batch_of_ptr),
                                                ctypes.byref(n)))
        return n.value

    def write_decomp_cpu_device(self, path):
        _check(lib().dc_write_decomp_cpu_device(self._h, path.encode()))

    def set_wait_limit(self, ns):
        """Limit of every bounded device wait (ns; 0 = the 4 s default)."""
        _check(lib().dc_set_wait_limit(self._h, int(ns)))

    def withhold_barrier(self, block=0):
        """Failure-detection tests: block `block` of the next persistent
        launch leaves at its first grid barrier without arriving (-1
        cancels)."""
        _check(lib().dc_test_withhold_barrier(self._h, int(block)))

    def synchronize(self):
        _check(lib().dc_synchronize(self._h))

    def stream(self):
        s = vp()
        _check(lib().dc_graph_stream(self._h, ctypes.byref(s)))
        return s.value or 0


class Scheduler:
    """The learned maintenance scheduler (BF16 MLP 16-64-64-2 on the GPU)."""

    def __init__(self, seed=0):
        h = vp()
        _check(lib().dc_sched_create(seed, ctypes.byref(h)))
        self._h = h
        self.nparams = lib().dc_sched_param_count()

    @property
    def handle(self):
        return self._h

    def free(self):
        if self._h and self._h.value:
            lib().dc_sched_free(self._h)
            self._h = vp()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def params(self):
        p = np.empty(self.nparams, np.float32)
        _check(lib().dc_sched_get_params(self._h, _p(p, f32p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(lib().dc_sched_set_params(self._h, _p(p, f32p)))

    def set_norm(self, mean, scale):
        mean = np.ascontiguousarray(mean, np.float32)
        scale = np.ascontiguousarray(scale, np.float32)
        _check(lib().dc_sched_set_norm(self._h, _p(mean, f32p), _p(scale, f32p)))

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, 16)
        Y = np.empty((len(X), 2), np.float32)
        _check(lib().dc_sched_predict(self._h, _p(X, f32p), len(X), _p(Y, f32p)))
        return Y

    def grad(self, X, T, M):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, 16)
        T = np.ascontiguousarray(T, np.float32).reshape(-1, 2)
        M = np.ascontiguousarray(M, np.uint8).reshape(-1, 2)
        g = np.empty(self.nparams, np.float32)
        loss = ctypes.c_float(0)
        _check(lib().dc_sched_grad(self._h, _p(X, f32p), _p(T, f32p), _p(M, u8p), len(X), _p(g, f32p),
                                   ctypes.byref(loss)))
        return g, loss.value

    def train(self, X, T, M, epochs=200, lr=3e-3):
        X = np.ascontiguousarray(X, np.float32).reshape(-1, 16)
        T = np.ascontiguousarray(T, np.float32).reshape(-1, 2)
        M = np.ascontiguousarray(M, np.uint8).reshape(-1, 2)
        loss = ctypes.c_float(0)
        _check(lib().dc_sched_train(self._h, _p(X, f32p), _p(T, f32p), _p(M, u8p), len(X), epochs, lr,
                                    ctypes.byref(loss)))
        return loss.value


class Server:
    """Serving loop over many device-resident graphs (dc_server_*): requests
    are queued per graph, coalesced into one maintenance batch per graph when
    a worker picks it, and run on per-graph streams under an HBM budget."""

    def __init__(self, hbm_budget_bytes, max_concurrent=4, method=MAINT_AUTO, device=0):
        h = vp()
        _check(lib().dc_server_create(int(hbm_budget_bytes), max_concurrent, method, device, ctypes.byref(h)))
        self._h = h

    def free(self):
        if getattr(self, "_h", None):
            lib().dc_server_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()

    def set_row_repair(self, on):
        _check(lib().dc_server_set_row_repair(self._h, 1 if on else 0))

    def add_graph(self, V, src, dst):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        gid = ctypes.c_uint32(0)
        _check(lib().dc_server_add_graph(self._h, V, len(src), _p(src, u32p), _p(dst, u32p), ctypes.byref(gid)))
        return gid.value

    def submit(self, graph_id, src, dst, is_delete=None):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        pairs = np.empty(2 * len(src), np.uint32)
        pairs[0::2] = src
        pairs[1::2] = dst
        dl = None if is_delete is None else np.ascontiguousarray(is_delete, np.uint8)
        rid = ctypes.c_uint64(0)
        _check(lib().dc_server_submit(self._h, graph_id, _p(pairs, u32p), None if dl is None else _p(dl, u8p),
                                      len(src), ctypes.byref(rid)))
        return rid.value

    def drain(self, timeout_ms=600000):
        _check(lib().dc_server_drain(self._h, timeout_ms))

    def completions(self):
        """Completed requests since the last call as a dict of arrays."""
        n = ctypes.c_uint64(0)
        _check(lib().dc_server_completions(self._h, None, None, None, None, None, None, 0, ctypes.byref(n)))
        m = n.value
        out = {"id": np.zeros(m, np.uint64), "graph": np.zeros(m, np.uint32), "latency_ms": np.zeros(m, np.float64),
               "batch_requests": np.zeros(m, np.uint32), "batch_updates": np.zeros(m, np.uint64),
               "status": np.zeros(m, np.int32)}
        if m:
            _check(lib().dc_server_completions(
                self._h, _p(out["id"], u64p), _p(out["graph"], u32p),
                out["latency_ms"].ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _p(out["batch_requests"], u32p),
                _p(out["batch_updates"], u64p), _p(out["status"], i32p), m, ctypes.byref(n)))
            for k in out:
                out[k] = out[k][:n.value]
        return out

    def info(self):
        st = ServerInfo()
        _check(lib().dc_server_info_get(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in ServerInfo._fields_}

    def result(self, graph_id, V, rows=True):
        """(kmaxes, rows or None) of a graph after all its queued requests."""
        km = np.zeros(V, np.int32)
        kmax = ctypes.c_int32(0)
        _check(lib().dc_server_graph_result(self._h, graph_id, _p(km, i32p), None, 0, ctypes.byref(kmax)))
        if not rows:
            return km, None
        R = np.zeros((kmax.value + 1) * V, np.int32)
        _check(lib().dc_server_graph_result(self._h, graph_id, _p(km, i32p), _p(R, i32p), R.size,
                                            ctypes.byref(kmax)))
        return km, R.reshape(kmax.value + 1, V)


def exported_symbols():
    """Names the header declares that the loaded library exports."""
    L = lib()
    return sorted(n for n in SIGNATURES if hasattr(L, n))
