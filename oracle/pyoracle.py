"""ctypes binding of the CPU oracle (liblvoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke()
(as the checker) and by bench.py's CPU-baseline leg.  The product never
imports it.  The C sources (louvain_oracle.c) cite the reference file:line
each step restates.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblvoracle.so")

RULES = {"cuda": 0, "py": 1}
PRECS = {"fp64": 0, "fp32": 1}
ROWS = {"first_seen": 0, "sorted": 1}
BUCKET_HI = (0, 4, 8, 16, 32, 84, 319)


class _LevelStat(ctypes.Structure):
    _fields_ = [
        ("n_vertices", ctypes.c_uint32),
        ("n_entries", ctypes.c_uint64),
        ("passes", ctypes.c_uint32),
        ("moved", ctypes.c_uint32),
        ("q_start", ctypes.c_double),
        ("q_end", ctypes.c_double),
    ]


_lib = None


def build() -> None:
    """Compile liblvoracle.so with the oracle's own Makefile."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        f64p = ctypes.POINTER(ctypes.c_double)
        L.orc_read_mtx.argtypes = [
            ctypes.c_char_p, ctypes.c_int, u32p, u64p,
            ctypes.POINTER(u64p), ctypes.POINTER(u32p), ctypes.POINTER(f64p),
            u32p, ctypes.c_char_p, ctypes.c_int,
        ]
        L.orc_read_mtx.restype = ctypes.c_int
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_buckets.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_move_phase.argtypes = [
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_uint32,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, u32p, f64p, f64p,
        ]
        L.orc_move_phase.restype = ctypes.c_int
        L.orc_contract.argtypes = [
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, u32p, u64p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ]
        L.orc_contract.restype = ctypes.c_int
        L.orc_louvain.argtypes = [
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, f64p,
            ctypes.POINTER(_LevelStat), ctypes.c_uint32, u32p,
        ]
        L.orc_louvain.restype = ctypes.c_int
        L.orc_modularity.argtypes = [
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p,
        ]
        L.orc_modularity.restype = ctypes.c_double
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def set_threads(t: int):
    """Host threads of the oracle's move decisions and intra-weight sum
    (1: the sequential restatement in louvian.py's summation order)."""
    lib().orc_set_threads(int(t))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class CSR:
    n: int
    off: np.ndarray  # uint64[n+1]
    col: np.ndarray  # uint32[E]
    w: np.ndarray  # float64[E] (FP32 values when read as float)
    max_deg: int = 0

    @property
    def nnz(self) -> int:
        return int(self.off[-1]) if self.n or len(self.off) else 0

    def normalized(self) -> "CSR":
        return CSR(
            self.n,
            np.ascontiguousarray(self.off, dtype=np.uint64),
            np.ascontiguousarray(self.col, dtype=np.uint32),
            np.ascontiguousarray(self.w, dtype=np.float64),
            self.max_deg,
        )


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"oracle error {code}: {msg}")
        self.code = code


def read_mtx(path: str, as_float: bool = True) -> CSR:
    L = lib()
    n = ctypes.c_uint32()
    nnz = ctypes.c_uint64()
    off = ctypes.POINTER(ctypes.c_uint64)()
    col = ctypes.POINTER(ctypes.c_uint32)()
    w = ctypes.POINTER(ctypes.c_double)()
    md = ctypes.c_uint32()
    err = ctypes.create_string_buffer(256)
    rc = L.orc_read_mtx(path.encode(), int(as_float), ctypes.byref(n),
                        ctypes.byref(nnz), ctypes.byref(off), ctypes.byref(col),
                        ctypes.byref(w), ctypes.byref(md), err, 256)
    if rc != 0:
        raise OracleError(rc, err.value.decode())
    N, E = n.value, nnz.value
    o = np.ctypeslib.as_array(off, shape=(N + 1,)).copy()
    c = np.ctypeslib.as_array(col, shape=(max(E, 1),))[:E].copy()
    ww = np.ctypeslib.as_array(w, shape=(max(E, 1),))[:E].copy()
    L.orc_free(ctypes.cast(off, ctypes.c_void_p))
    L.orc_free(ctypes.cast(col, ctypes.c_void_p))
    L.orc_free(ctypes.cast(w, ctypes.c_void_p))
    return CSR(N, o, c, ww, md.value)


def buckets(g: CSR) -> np.ndarray:
    g = g.normalized()
    out = np.zeros(max(g.n, 1), dtype=np.uint8)
    lib().orc_buckets(g.n, _p(g.off), _p(out))
    return out[: g.n]


@dataclass
class Level:
    n_vertices: int
    n_entries: int
    passes: int
    moved: bool
    q_start: float
    q_end: float


@dataclass
class Result:
    assignment: np.ndarray
    q: float
    levels: list = field(default_factory=list)


def louvain(g: CSR, threshold: float, rule: str = "cuda", prec: str = "fp32",
            rows: str = "sorted", max_passes: int = 100000,
            max_levels: int = 0) -> Result:
    g = g.normalized()
    L = lib()
    asg = np.zeros(max(g.n, 1), dtype=np.uint32)
    q = ctypes.c_double()
    stats = (_LevelStat * 256)()
    nl = ctypes.c_uint32()
    rc = L.orc_louvain(g.n, _p(g.off), _p(g.col), _p(g.w), float(threshold),
                       RULES[rule], PRECS[prec], ROWS[rows], max_passes,
                       max_levels, _p(asg), ctypes.byref(q), stats, 256,
                       ctypes.byref(nl))
    if rc != 0:
        raise OracleError(rc, "louvain failed")
    levels = [
        Level(s.n_vertices, s.n_entries, s.passes, bool(s.moved), s.q_start,
              s.q_end)
        for s in stats[: min(nl.value, 256)]
    ]
    return Result(asg[: g.n], q.value, levels)


def move_phase(g: CSR, threshold: float, rule: str = "cuda",
               prec: str = "fp32", max_passes: int = 100000):
    """Returns (progressed, comm, q_trace, q_start, q_end)."""
    g = g.normalized()
    comm = np.zeros(max(g.n, 1), dtype=np.uint32)
    trace = np.zeros(max_passes if max_passes < 100000 else 4096,
                     dtype=np.float64)
    passes = ctypes.c_uint32()
    qs = ctypes.c_double()
    qe = ctypes.c_double()
    r = lib().orc_move_phase(g.n, _p(g.off), _p(g.col), _p(g.w),
                             float(threshold), RULES[rule], PRECS[prec],
                             max_passes, _p(comm), _p(trace), len(trace),
                             ctypes.byref(passes), ctypes.byref(qs),
                             ctypes.byref(qe))
    if r < 0:
        raise OracleError(-r, "move phase failed")
    return bool(r), comm[: g.n], trace[: min(passes.value, len(trace))], \
        qs.value, qe.value


def contract(g: CSR, comm: np.ndarray, rows: str = "sorted",
             prec: str = "fp32"):
    """Returns (new CSR, new_id)."""
    g = g.normalized()
    comm = np.ascontiguousarray(comm, dtype=np.uint32)
    noff = np.zeros(g.n + 1, dtype=np.uint64)
    ncol = np.zeros(max(g.nnz, 1), dtype=np.uint32)
    nw = np.zeros(max(g.nnz, 1), dtype=np.float64)
    nid = np.zeros(max(g.n, 1), dtype=np.uint32)
    nn = ctypes.c_uint32()
    ne = ctypes.c_uint64()
    rc = lib().orc_contract(g.n, _p(g.off), _p(g.col), _p(g.w), _p(comm),
                            ROWS[rows], PRECS[prec], ctypes.byref(nn),
                            ctypes.byref(ne), _p(noff), _p(ncol), _p(nw),
                            _p(nid))
    if rc != 0:
        raise OracleError(rc, "contract failed")
    N, E = nn.value, ne.value
    return CSR(N, noff[: N + 1].copy(), ncol[:E].copy(), nw[:E].copy()), \
        nid[: g.n]


def modularity(g: CSR, part: np.ndarray) -> float:
    g = g.normalized()
    part = np.ascontiguousarray(part, dtype=np.uint32)
    return float(lib().orc_modularity(g.n, _p(g.off), _p(g.col), _p(g.w),
                                      _p(part)))
