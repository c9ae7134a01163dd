"""ctypes binding of the B200 Louvain engine's C ABI (include/louvain_b200.h).

The engine is the CUDA library lib/liblouvain_b200.so; this module only
marshals arguments.  There is no CPU fallback: if the library cannot be
loaded, or no CUDA device is usable, the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "liblouvain_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(PKG_DIR), "include", "louvain_b200.h")

RULE_PY = 0
RULE_CUDA = 1
RULES = {"py": RULE_PY, "cuda": RULE_CUDA}
GAINS = {"fp32": 0, "fp64": 1}  # lv_gain

STATUS = {
    0: "LV_OK", 1: "LV_ERR_ARG", 2: "LV_ERR_IO", 3: "LV_ERR_PARSE",
    4: "LV_ERR_NOMEM", 5: "LV_ERR_CUDA", 6: "LV_ERR_STATE", 7: "LV_ERR_LIMIT",
    8: "LV_ERR_TIMEOUT",
}


class LouvainError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int),
        ("rule", ctypes.c_int),
        ("max_passes", ctypes.c_uint32),
        ("max_levels", ctypes.c_uint32),
        ("use_graphs", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("gain", ctypes.c_int),
        ("level_kernel", ctypes.c_int),
        ("contract_sort", ctypes.c_int),
        ("apply_launch", ctypes.c_int),
        ("modularity_full", ctypes.c_int),
    ]


class LevelInfo(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_uint32),
        ("n_entries", ctypes.c_uint64),
        ("passes", ctypes.c_uint32),
        ("moved", ctypes.c_uint32),
        ("q_start", ctypes.c_double),
        ("q_end", ctypes.c_double),
        ("move_ms", ctypes.c_float),
        ("aggregate_ms", ctypes.c_float),
        ("prepare_ms", ctypes.c_float),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("modularity", ctypes.c_double),
        ("n_vertices", ctypes.c_uint32),
        ("n_communities", ctypes.c_uint32),
        ("n_levels", ctypes.c_uint32),
        ("edges_processed", ctypes.c_uint64),
        ("alg_ms", ctypes.c_float),
        ("copy_ms", ctypes.c_float),
    ]


class KernelStat(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_uint64),
        ("total_ms", ctypes.c_double),
        ("bytes", ctypes.c_double),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [("bucket_kernel", ctypes.c_uint8 * 8), ("bucket_ms", ctypes.c_float * 8)]


KERNELS = ["lanes4", "lanes8", "lanes16", "lanes32", "warp128", "warp512", "block"]
KERNEL_MAX_DEGREE = [4, 8, 16, 32, 84, 319, 2048]
BUCKET_MAX_DEGREE = [0, 4, 8, 16, 32, 84, 319, 2048]


class ServeConfig(ctypes.Structure):
    _fields_ = [("min_gain", ctypes.c_float), ("budget_bytes", ctypes.c_uint64),
                ("max_graphs", ctypes.c_uint32), ("n_lanes", ctypes.c_uint32),
                ("lane_max_entries", ctypes.c_uint64 * 4), ("lane_share", ctypes.c_float * 4),
                ("background", ctypes.c_int), ("lane_solo", ctypes.c_uint32)]


class ServeResult(ctypes.Structure):
    _fields_ = [("ticket", ctypes.c_uint64), ("modularity", ctypes.c_double),
                ("n_vertices", ctypes.c_uint32), ("n_communities", ctypes.c_uint32),
                ("levels", ctypes.c_uint32), ("lane", ctypes.c_uint32),
                ("submit_ms", ctypes.c_double), ("admit_ms", ctypes.c_double),
                ("done_ms", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [("queued", ctypes.c_uint32), ("resident", ctypes.c_uint32),
                ("finished", ctypes.c_uint32), ("slot_cap", ctypes.c_uint32),
                ("n_lanes", ctypes.c_uint32),
                ("resident_vertices", ctypes.c_uint64), ("resident_entries", ctypes.c_uint64),
                ("cap_vertices", ctypes.c_uint64), ("cap_entries", ctypes.c_uint64),
                ("budget_bytes", ctypes.c_uint64), ("steps", ctypes.c_uint64),
                ("admitted", ctypes.c_uint64), ("completed", ctypes.c_uint64)]


# symbol -> (restype, argtypes)
_VP = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_SIGS = {
    "lv_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "lv_last_error": (ctypes.c_char_p, []),
    "lv_abi_version": (ctypes.c_int, []),
    "lv_config_default": (None, [ctypes.POINTER(Config)]),
    "lv_graph_load_mtx": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
    "lv_graph_from_edges": (ctypes.c_int, [_U32, _U64, _VP, _VP, _VP, ctypes.POINTER(_VP)]),
    "lv_graph_from_csr": (ctypes.c_int, [_U32, _VP, _VP, _VP, ctypes.POINTER(_VP)]),
    "lv_graph_view": (ctypes.c_int, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U64),
                                     ctypes.POINTER(_VP), ctypes.POINTER(_VP),
                                     ctypes.POINTER(_VP), ctypes.POINTER(_U32)]),
    "lv_graph_destroy": (None, [_VP]),
    "lv_graph_save": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "lv_graph_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_VP)]),
    "lv_engine_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(_VP)]),
    "lv_engine_destroy": (None, [_VP]),
    "lv_engine_load": (ctypes.c_int, [_VP, _VP]),
    "lv_engine_load_device": (ctypes.c_int, [_VP, _U32, _U64, _VP, _VP, _VP]),
    "lv_phase_move": (ctypes.c_int, [_VP, ctypes.c_float, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_double)]),
    "lv_phase_aggregate": (ctypes.c_int, [_VP]),
    "lv_run": (ctypes.c_int, [_VP, _VP, ctypes.c_float, ctypes.POINTER(Result)]),
    "lv_run_device": (ctypes.c_int, [_VP, _U32, _U64, _VP, _VP, _VP, ctypes.c_float, _VP,
                                     ctypes.POINTER(Result)]),
    "lv_get_assignment": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t]),
    "lv_get_levels": (ctypes.c_int, [_VP, ctypes.POINTER(LevelInfo), _U32,
                                     ctypes.POINTER(_U32)]),
    "lv_get_level_size": (ctypes.c_int, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U64)]),
    "lv_get_level_state": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "lv_get_level_csr": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "lv_set_level_comm": (ctypes.c_int, [_VP, _VP]),
    "lv_modularity_fp64": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(ctypes.c_double)]),
    "lv_get_buckets": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t]),
    "lv_set_profiling": (ctypes.c_int, [_VP, ctypes.c_int]),
    "lv_get_kernel_stats": (ctypes.c_int, [_VP, ctypes.POINTER(KernelStat), _U32,
                                           ctypes.POINTER(_U32)]),
    "lv_reset_kernel_stats": (ctypes.c_int, [_VP]),
    "lv_get_launch_count": (ctypes.c_int, [ctypes.POINTER(_U64)]),
    "lv_debug_fail_device_alloc": (ctypes.c_int, [_U64]),
    "lv_get_sync_count": (ctypes.c_int, [ctypes.POINTER(_U64)]),
    "lv_engine_load_edges": (ctypes.c_int, [_VP, _U32, _U64, _VP, _VP, _VP]),
    "lv_engine_load_mtx": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "lv_csr_from_edges_device": (ctypes.c_int, [_U32, _U64, _VP, _VP, _VP, _VP, _VP, _VP,
                                                ctypes.POINTER(_U64), _VP]),
    "lv_get_communities": (ctypes.c_int, [_VP, _VP, ctypes.c_size_t,
                                          ctypes.POINTER(_U32)]),
    "lv_modularity_noalloc": (ctypes.c_int, [_U32, _VP, _VP, _VP, _VP, _VP,
                                             ctypes.POINTER(ctypes.c_double), _VP]),
    "lv_batch_run_device": (ctypes.c_int, [_VP, _U32, _VP, _U32, _U64, _VP, _VP, _VP,
                                           ctypes.c_float, _VP, _VP, _VP,
                                           ctypes.POINTER(Result)]),
    "lv_batch_run": (ctypes.c_int, [_VP, _U32, _VP, ctypes.c_float, _VP, _VP, _VP,
                                    ctypes.POINTER(Result)]),
    "lv_serve_config_default": (None, [ctypes.POINTER(ServeConfig)]),
    "lv_autotune": (ctypes.c_int, [_VP, _U32, ctypes.POINTER(Tuning)]),
    "lv_set_tuning": (ctypes.c_int, [_VP, ctypes.POINTER(Tuning)]),
    "lv_get_tuning": (ctypes.c_int, [_VP, ctypes.POINTER(Tuning)]),
    "lv_serve_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(ServeConfig),
                                       ctypes.POINTER(_VP)]),
    "lv_serve_wait": (ctypes.c_int, [_VP, _U32, ctypes.POINTER(ctypes.c_int)]),
    "lv_serve_submit": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(_U64)]),
    "lv_serve_step": (ctypes.c_int, [_VP, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "lv_serve_poll": (ctypes.c_int, [_VP, ctypes.POINTER(ServeResult), _VP, ctypes.c_size_t,
                                     ctypes.POINTER(ctypes.c_int)]),
    "lv_serve_get_stats": (ctypes.c_int, [_VP, ctypes.POINTER(ServeStats)]),
    "lv_serve_destroy": (None, [_VP]),
    "lv_serve_engine": (ctypes.c_int, [_VP, _U32, ctypes.POINTER(_VP)]),
}

NOALLOC_MAX_VERTICES = 1 << 20


def modularity_noalloc(n: int, d_off: int, d_col: int, d_w: int, d_part: int,
                       d_q: int, stream: int = 0) -> float:
    """FP64 modularity of a partition kept in device memory, computed
    without any allocation (fixed scratch inside the library).  Returns Q
    and also leaves it at d_q."""
    q = ctypes.c_double()
    _check(lib().lv_modularity_noalloc(n, d_off, d_col, d_w, d_part, d_q,
                                       ctypes.byref(q), stream or None))
    return q.value

def pack_graphs(csrs):
    """Block-diagonal union of CSR graphs [(n, off, col, w), ...], the input
    layout of lv_batch_run_device.  Returns (graph_offsets u64[G+1],
    off u64[N+1], col u32[E], w f32[E]): graph g's vertices are renumbered
    by graph_offsets[g] and its entries keep their order."""
    G = len(csrs)
    goff = np.zeros(G + 1, dtype=np.uint64)
    eoff = np.zeros(G + 1, dtype=np.uint64)
    for g, (n, off, col, w) in enumerate(csrs):
        goff[g + 1] = goff[g] + np.uint64(n)
        eoff[g + 1] = eoff[g] + np.uint64(len(col))
    N, E = int(goff[G]), int(eoff[G])
    off = np.empty(N + 1, dtype=np.uint64)
    col = np.empty(E, dtype=np.uint32)
    w = np.empty(E, dtype=np.float32)
    for g, (n, o, c, x) in enumerate(csrs):
        vb, eb = int(goff[g]), int(eoff[g])
        off[vb:vb + n] = np.asarray(o[:n], dtype=np.uint64) + np.uint64(eb)
        col[eb:eb + len(c)] = np.asarray(c, dtype=np.uint64) + np.uint64(vb)
        w[eb:eb + len(c)] = x
    off[N] = E
    return goff, off, col, w


_lib = None


def header_symbols() -> list[str]:
    """Function names declared in include/louvain_b200.h."""
    import re

    text = open(HEADER_PATH).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(lv_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with "
                          "`python -c 'import __graft_entry__ as g; g.build()'`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def sync_count() -> int:
    """Host waits on a stream the library has made so far (process-wide)."""
    c = _U64()
    _check(lib().lv_get_sync_count(ctypes.byref(c)))
    return int(c.value)


def fail_device_alloc(n: int):
    """Fault injection for tests: the nth device allocation from now on
    fails as out-of-memory (0 switches it off)."""
    _check(lib().lv_debug_fail_device_alloc(n))


def launch_count() -> int:
    """Kernels the library has launched in this process."""
    c = _U64()
    _check(lib().lv_get_launch_count(ctypes.byref(c)))
    return c.value


def _check(status: int):
    if status != 0:
        raise LouvainError(status, lib().lv_last_error().decode(errors="replace"))


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Graph:
    """Host CSR graph owned by the library."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def load_mtx(cls, path: str) -> "Graph":
        h = ctypes.c_void_p()
        _check(lib().lv_graph_load_mtx(path.encode(), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_edges(cls, n: int, src, dst, w=None) -> "Graph":
        src = np.ascontiguousarray(src, dtype=np.uint32)
        dst = np.ascontiguousarray(dst, dtype=np.uint32)
        wp = None
        if w is not None:
            w = np.ascontiguousarray(w, dtype=np.float32)
            wp = _p(w)
        h = ctypes.c_void_p()
        _check(lib().lv_graph_from_edges(n, len(src), _p(src), _p(dst), wp,
                                         ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, n: int, off, col, w) -> "Graph":
        off = np.ascontiguousarray(off, dtype=np.uint64)
        col = np.ascontiguousarray(col, dtype=np.uint32)
        w = np.ascontiguousarray(w, dtype=np.float32)
        h = ctypes.c_void_p()
        _check(lib().lv_graph_from_csr(n, _p(off), _p(col), _p(w), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def load(cls, path: str) -> "Graph":
        """A graph saved with save() (binary CSR)."""
        h = ctypes.c_void_p()
        _check(lib().lv_graph_load(path.encode(), ctypes.byref(h)))
        return cls(h)

    def save(self, path: str):
        _check(lib().lv_graph_save(self._h, path.encode()))

    def csr(self):
        n = _U32()
        e = _U64()
        po, pc, pw = _VP(), _VP(), _VP()
        md = _U32()
        _check(lib().lv_graph_view(self._h, ctypes.byref(n), ctypes.byref(e),
                                   ctypes.byref(po), ctypes.byref(pc),
                                   ctypes.byref(pw), ctypes.byref(md)))
        N, E = n.value, e.value
        off = np.ctypeslib.as_array(ctypes.cast(po, ctypes.POINTER(_U64)),
                                    shape=(N + 1,)).copy()
        if E:
            col = np.ctypeslib.as_array(ctypes.cast(pc, ctypes.POINTER(_U32)),
                                        shape=(E,)).copy()
            w = np.ctypeslib.as_array(ctypes.cast(pw, ctypes.POINTER(ctypes.c_float)),
                                      shape=(E,)).copy()
        else:
            col = np.zeros(0, np.uint32)
            w = np.zeros(0, np.float32)
        return N, off, col, w, md.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lv_graph_destroy(self._h)
            self._h = None


@dataclass
class RunResult:
    modularity: float
    assignment: np.ndarray
    n_communities: int
    levels: list
    edges_processed: int
    alg_ms: float
    copy_ms: float


class Engine:
    def __init__(self, device: int = 0, rule: str = "py", max_passes: int = 0,
                 max_levels: int = 0, use_graphs: bool = True, stream: int = 0,
                 gain: str = "fp32", level_kernel: bool = False,
                 contract_sort: bool = False, apply_launch: bool = False,
                 modularity_full: bool = False):
        cfg = Config()
        lib().lv_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.rule = RULES[rule]
        cfg.gain = GAINS[gain]
        cfg.level_kernel = int(level_kernel)
        cfg.contract_sort = int(contract_sort)
        cfg.apply_launch = int(apply_launch)
        cfg.modularity_full = int(modularity_full)
        cfg.max_passes = max_passes
        cfg.max_levels = max_levels
        cfg.use_graphs = int(use_graphs)
        cfg.stream = stream or None
        h = ctypes.c_void_p()
        _check(lib().lv_engine_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self.n0 = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().lv_engine_destroy(self._h)
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

    # -- loading ---------------------------------------------------------
    def load(self, g: Graph):
        _check(lib().lv_engine_load(self._h, g._h))
        self.n0 = self._level_size()[0]

    def load_edges(self, n: int, src, dst, w=None):
        """Edge lines (host) -> the reference reader's CSR built on the device."""
        src = np.ascontiguousarray(src, dtype=np.uint32)
        dst = np.ascontiguousarray(dst, dtype=np.uint32)
        wp = None
        if w is not None:
            w = np.ascontiguousarray(w, dtype=np.float32)
            wp = _p(w)
        _check(lib().lv_engine_load_edges(self._h, n, len(src), _p(src), _p(dst), wp))
        self.n0 = n

    def load_mtx(self, path: str):
        """Matrix Market file -> host parse -> CSR built on the device."""
        _check(lib().lv_engine_load_mtx(self._h, path.encode()))
        self.n0 = self._level_size()[0]  # level 0 = the input graph

    def communities(self):
        """(offsets, members) of the final partition, grouped on the device."""
        c = _U32()
        _check(lib().lv_get_communities(self._h, None, 0, ctypes.byref(c)))
        out = np.zeros(int(c.value) + 1 + self.n0, dtype=np.uint32)
        _check(lib().lv_get_communities(self._h, _p(out), out.size, ctypes.byref(c)))
        k = int(c.value)
        return out[:k + 1].copy(), out[k + 1:].copy()

    def load_device(self, n: int, nnz: int, d_off: int, d_col: int, d_w: int):
        _check(lib().lv_engine_load_device(self._h, n, nnz, d_off, d_col, d_w))
        self.n0 = n

    # -- phases ----------------------------------------------------------
    def phase_move(self, min_gain: float):
        more = ctypes.c_int()
        q = ctypes.c_double()
        _check(lib().lv_phase_move(self._h, min_gain, ctypes.byref(more), ctypes.byref(q)))
        return bool(more.value), q.value

    def phase_aggregate(self):
        _check(lib().lv_phase_aggregate(self._h))

    def run(self, g: Graph, min_gain: float) -> RunResult:
        r = Result()
        _check(lib().lv_run(self._h, g._h, min_gain, ctypes.byref(r)))
        self.n0 = r.n_vertices
        return self._result(r)

    def run_device(self, n: int, nnz: int, d_off: int, d_col: int, d_w: int,
                   min_gain: float, d_assignment: int = 0) -> Result:
        r = Result()
        _check(lib().lv_run_device(self._h, n, nnz, d_off, d_col, d_w, min_gain,
                                   d_assignment or None, ctypes.byref(r)))
        self.n0 = n
        return r

    # -- autotuning ------------------------------------------------------
    def autotune(self, reps: int = 5) -> dict:
        """Times every fitting kernel variant of every bucket on the loaded
        graph's current level and keeps the fastest.  Returns {bucket:
        (kernel name, ms per launch)} for the non-empty buckets."""
        t = Tuning()
        _check(lib().lv_autotune(self._h, reps, ctypes.byref(t)))
        return {b: (KERNELS[t.bucket_kernel[b]], t.bucket_ms[b])
                for b in range(1, 8) if t.bucket_ms[b] > 0}

    def set_tuning(self, kernels):
        """kernels: 7 names or ids, buckets 1..7."""
        t = Tuning()
        for b, k in enumerate(kernels, start=1):
            t.bucket_kernel[b] = KERNELS.index(k) if isinstance(k, str) else int(k)
        _check(lib().lv_set_tuning(self._h, ctypes.byref(t)))

    def tuning(self) -> list:
        t = Tuning()
        _check(lib().lv_get_tuning(self._h, ctypes.byref(t)))
        return [KERNELS[t.bucket_kernel[b]] for b in range(1, 8)]

    def batch_run(self, graphs, min_gain: float):
        """Runs every graph of `graphs` (Graph objects) in one batched run.
        Returns (list of per-graph local assignments, modularity array,
        levels array, Result)."""
        G = len(graphs)
        arr = (_VP * max(G, 1))(*[g._h for g in graphs])
        sizes = [g.csr()[0] for g in graphs]
        out = np.zeros(max(sum(sizes), 1), dtype=np.uint32)
        q = np.zeros(max(G, 1), dtype=np.float64)
        lv = np.zeros(max(G, 1), dtype=np.uint32)
        r = Result()
        _check(lib().lv_batch_run(self._h, G, arr, min_gain, _p(out), _p(q), _p(lv),
                                  ctypes.byref(r)))
        parts, s = [], 0
        for n in sizes:
            parts.append(out[s:s + n].copy())
            s += n
        return parts, q[:G].copy(), lv[:G].copy(), r

    def batch_run_device(self, graph_offsets, n: int, nnz: int, d_off: int, d_col: int,
                         d_w: int, min_gain: float, d_assignment: int):
        """Batched run over a block-diagonal union CSR in device memory;
        graph g owns vertices [graph_offsets[g], graph_offsets[g+1]).
        Returns (modularity array, levels array, Result)."""
        goff = np.ascontiguousarray(graph_offsets, dtype=np.uint64)
        G = len(goff) - 1
        q = np.zeros(max(G, 1), dtype=np.float64)
        lv = np.zeros(max(G, 1), dtype=np.uint32)
        r = Result()
        _check(lib().lv_batch_run_device(self._h, G, _p(goff), n, nnz, d_off, d_col, d_w,
                                         min_gain, d_assignment, _p(q), _p(lv),
                                         ctypes.byref(r)))
        return q[:G].copy(), lv[:G].copy(), r

    def _result(self, r: Result) -> RunResult:
        return RunResult(r.modularity, self.assignment(), r.n_communities,
                         self.levels(), r.edges_processed, r.alg_ms, r.copy_ms)

    # -- introspection ---------------------------------------------------
    def assignment(self) -> np.ndarray:
        out = np.zeros(max(self.n0, 1), dtype=np.uint32)
        _check(lib().lv_get_assignment(self._h, _p(out), self.n0))
        return out[: self.n0]

    def levels(self) -> list:
        cnt = _U32()
        _check(lib().lv_get_levels(self._h, None, 0, ctypes.byref(cnt)))
        arr = (LevelInfo * max(cnt.value, 1))()
        _check(lib().lv_get_levels(self._h, arr, cnt.value, ctypes.byref(cnt)))
        return [
            dict(n_vertices=a.n_vertices, n_entries=a.n_entries, passes=a.passes,
                 moved=bool(a.moved), q_start=a.q_start, q_end=a.q_end,
                 move_ms=a.move_ms, aggregate_ms=a.aggregate_ms,
                 prepare_ms=a.prepare_ms)
            for a in arr[: cnt.value]
        ]

    def _level_size(self):
        n = _U32()
        e = _U64()
        _check(lib().lv_get_level_size(self._h, ctypes.byref(n), ctypes.byref(e)))
        return n.value, e.value

    def level_size(self):
        return self._level_size()

    def level_state(self):
        n, _ = self._level_size()
        comm = np.zeros(max(n, 1), np.uint32)
        sz = np.zeros(max(n, 1), np.uint32)
        k = np.zeros(max(n, 1), np.float32)
        _check(lib().lv_get_level_state(self._h, _p(comm), _p(sz), _p(k)))
        return comm[:n], sz[:n], k[:n]

    def level_csr(self):
        n, e = self._level_size()
        off = np.zeros(n + 1, np.uint64)
        col = np.zeros(max(e, 1), np.uint32)
        w = np.zeros(max(e, 1), np.float32)
        _check(lib().lv_get_level_csr(self._h, _p(off), _p(col), _p(w)))
        return n, off, col[:e], w[:e]

    def set_level_comm(self, comm):
        comm = np.ascontiguousarray(comm, dtype=np.uint32)
        _check(lib().lv_set_level_comm(self._h, _p(comm)))

    def modularity(self, partition) -> float:
        part = np.ascontiguousarray(partition, dtype=np.uint32)
        q = ctypes.c_double()
        _check(lib().lv_modularity_fp64(self._h, _p(part), ctypes.byref(q)))
        return q.value

    def buckets(self) -> np.ndarray:
        n, _ = self._level_size()
        out = np.zeros(max(n, 1), np.uint8)
        _check(lib().lv_get_buckets(self._h, _p(out), n))
        return out[:n]

    # -- kernel timing ---------------------------------------------------
    def set_profiling(self, on: bool = True):
        _check(lib().lv_set_profiling(self._h, int(on)))

    def reset_kernel_stats(self):
        _check(lib().lv_reset_kernel_stats(self._h))

    def kernel_stats(self) -> dict:
        arr = (KernelStat * 32)()
        cnt = _U32()
        _check(lib().lv_get_kernel_stats(self._h, arr, 32, ctypes.byref(cnt)))
        return {a.name.decode(): dict(launches=a.launches, total_ms=a.total_ms,
                                      bytes=a.bytes)
                for a in arr[: cnt.value]}


@dataclass
class ServedGraph:
    ticket: int
    modularity: float
    assignment: np.ndarray
    n_communities: int
    levels: int
    lane: int
    submit_ms: float
    admit_ms: float
    done_ms: float


class Server:
    """Continuous-batching server (lv_serve_*).  submit() queues a graph;
    without background workers step() admits what fits and runs one level
    of every lane; poll() returns finished requests; drain() runs until
    everything submitted is finished.  lanes > 1 routes requests by entry
    count (lane_max_entries) to separate unions with their own budget share;
    background=True steps every lane on its own worker thread."""

    def __init__(self, min_gain: float, budget_bytes: int, max_graphs: int = 0,
                 lanes: int = 1, background: bool = False, lane_max_entries=None,
                 lane_share=None, device: int = 0, rule: str = "py", max_passes: int = 0,
                 max_levels: int = 0, use_graphs: bool = True, gain: str = "fp32",
                 lane_solo: int | None = None):
        cfg = Config()
        lib().lv_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.rule = RULES[rule]
        cfg.gain = GAINS[gain]
        cfg.max_passes = max_passes
        cfg.max_levels = max_levels
        cfg.use_graphs = int(use_graphs)
        sc = ServeConfig()
        lib().lv_serve_config_default(ctypes.byref(sc))
        sc.min_gain = min_gain
        sc.budget_bytes = budget_bytes
        sc.max_graphs = max_graphs
        sc.n_lanes = lanes
        sc.background = int(background)
        if lanes == 1:
            sc.lane_share[0] = 1.0
        if lane_max_entries is not None:
            for i, x in enumerate(lane_max_entries):
                sc.lane_max_entries[i] = x
        if lane_share is not None:
            for i, x in enumerate(lane_share):
                sc.lane_share[i] = x
        if lane_solo is not None:
            sc.lane_solo = lane_solo
        elif lanes == 1:
            sc.lane_solo = 0
        h = ctypes.c_void_p()
        _check(lib().lv_serve_create(ctypes.byref(cfg), ctypes.byref(sc), ctypes.byref(h)))
        self._h = h
        self.background = background
        self.lanes = lanes
        self._sizes = {}
        self._graphs = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().lv_serve_destroy(self._h)
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

    def submit(self, g: Graph, n_vertices: int | None = None) -> int:
        """Queues g; returns its ticket.  n_vertices (if known) saves a
        look-up of the graph's size."""
        t = _U64()
        _check(lib().lv_serve_submit(self._h, g._h, ctypes.byref(t)))
        self._sizes[t.value] = g.csr()[0] if n_vertices is None else n_vertices
        self._graphs[t.value] = g  # the server reads it until the result is polled
        return t.value

    def step(self):
        """One scheduling step of every lane (nothing with background
        workers); returns (resident, queued) graph counts."""
        r, q = _U32(), _U32()
        _check(lib().lv_serve_step(self._h, ctypes.byref(r), ctypes.byref(q)))
        return r.value, q.value

    def wait(self, timeout_ms: int = 50) -> bool:
        """Background mode: blocks until a result is ready, the server is
        idle or the timeout passes; returns True when idle."""
        idle = ctypes.c_int()
        _check(lib().lv_serve_wait(self._h, timeout_ms, ctypes.byref(idle)))
        return bool(idle.value)

    def poll(self):
        """The oldest finished request as a ServedGraph, or None."""
        cap = max(self._sizes.values(), default=0)
        buf = np.zeros(max(cap, 1), dtype=np.uint32)
        res = ServeResult()
        got = ctypes.c_int()
        _check(lib().lv_serve_poll(self._h, ctypes.byref(res), _p(buf), buf.size,
                                   ctypes.byref(got)))
        if not got.value:
            return None
        self._sizes.pop(res.ticket, None)
        self._graphs.pop(res.ticket, None)
        return ServedGraph(res.ticket, res.modularity, buf[: res.n_vertices].copy(),
                           res.n_communities, res.levels, res.lane, res.submit_ms,
                           res.admit_ms, res.done_ms)

    def drain(self):
        """Runs until nothing is queued or resident; returns the finished
        requests by ticket."""
        out = {}
        while True:
            if self.background:
                idle = self.wait(50)
                r = q = 0 if idle else 1
            else:
                r, q = self.step()
            while (x := self.poll()) is not None:
                out[x.ticket] = x
            if r == 0 and q == 0:
                break
        while (x := self.poll()) is not None:
            out[x.ticket] = x
        return out

    def set_profiling(self, on: bool = True, lane: int = 0):
        _check(lib().lv_set_profiling(self._engine(lane), int(on)))

    def kernel_stats(self, lane: int = 0) -> dict:
        arr = (KernelStat * 32)()
        cnt = _U32()
        _check(lib().lv_get_kernel_stats(self._engine(lane), arr, 32, ctypes.byref(cnt)))
        return {a.name.decode(): dict(launches=a.launches, total_ms=a.total_ms, bytes=a.bytes)
                for a in arr[: cnt.value]}

    def _engine(self, lane: int = 0):
        e = ctypes.c_void_p()
        _check(lib().lv_serve_engine(self._h, lane, ctypes.byref(e)))
        return e

    def stats(self) -> dict:
        st = ServeStats()
        _check(lib().lv_serve_get_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}
