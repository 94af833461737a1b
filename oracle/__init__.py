"""CPU checkers for the n_queens_b200 GPU path (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline / reference legs
of bench.py import this package.  The product library never calls it.

Two ctypes libraries are exposed:

* :data:`lib` -- ``liboracle_nq.so``, the plain-C restatement in
  ``nq_oracle.c`` (count, node count and expander, each citing the reference
  line it restates) and ``dihedral_oracle.c`` (the 8-fold decomposition of the
  library's dihedral entries, pinned by the reference's totals);
* :func:`ref` -- ``_ref/libnq_ref.so``, the reference's own
  ``src/n_queens.cpp`` compiled unchanged behind ``ref_shim.cpp``.  It exists
  only where the reference sources were available at build time (the golden
  fixtures in tests/golden/ carry its outputs elsewhere).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(HERE, "liboracle_nq.so")
_REF_SO = os.path.join(HERE, "_ref", "libnq_ref.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build() -> None:
    """Compile the checkers (make in this directory)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load_oracle():
    if not os.path.exists(_ORACLE_SO):
        build()
    L = ctypes.CDLL(_ORACLE_SO)
    L.nq_oracle_count_task.restype = ctypes.c_uint64
    L.nq_oracle_count_task.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    L.nq_oracle_nodes_task.restype = ctypes.c_uint64
    L.nq_oracle_nodes_task.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    L.nq_oracle_expand.restype = ctypes.c_int64
    L.nq_oracle_expand.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_int64]
    L.nq_oracle_count_tasks.restype = None
    L.nq_oracle_count_tasks.argtypes = [ctypes.c_int, ctypes.c_int64, _u32p, _u32p, _u32p, _u64p, _u64p,
                                        ctypes.c_int]
    L.nq_oracle_total.restype = ctypes.c_int64
    L.nq_oracle_total.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u64p]
    return L


lib = _load_oracle()


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def count_task(N: int, cur: int, left: int, right: int) -> int:
    """Completions of one partial board (restates src/n_queens.cpp:8-21)."""
    return int(lib.nq_oracle_count_task(N, cur & 0xFFFFFFFF, left & 0xFFFFFFFF, right & 0xFFFFFFFF))


def nodes_task(N: int, cur: int, left: int, right: int) -> int:
    """DFS nodes of one task (placements into rows popc(cur)..N-2)."""
    return int(lib.nq_oracle_nodes_task(N, cur & 0xFFFFFFFF, left & 0xFFFFFFFF, right & 0xFFFFFFFF))


def expand(N: int, rows: int):
    """Prefix tasks as three uint32 arrays (restates src/n_queens.cpp:74-113)."""
    n = lib.nq_oracle_expand(N, rows, None, None, None, 0)
    if n < 0:
        raise ValueError(f"bad (N, rows) = ({N}, {rows})")
    c = np.empty(n, np.uint32)
    l = np.empty(n, np.uint32)
    r = np.empty(n, np.uint32)
    lib.nq_oracle_expand(N, rows, _p(c, _u32p), _p(l, _u32p), _p(r, _u32p), n)
    return c, l, r


def count_tasks(N: int, cols, ld, rd, nodes: bool = False, threads: int = 0):
    """Per-task counts (and optionally nodes) of a task list, OpenMP."""
    cols = np.ascontiguousarray(cols, np.uint32)
    ld = np.ascontiguousarray(ld, np.uint32)
    rd = np.ascontiguousarray(rd, np.uint32)
    n = cols.size
    cnt = np.empty(n, np.uint64)
    nd = np.empty(n, np.uint64) if nodes else None
    lib.nq_oracle_count_tasks(N, n, _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p), _p(cnt, _u64p),
                              _p(nd, _u64p), threads)
    return (cnt, nd) if nodes else cnt


def total(N: int, rows: int, threads: int = 0, with_nodes: bool = False):
    """Whole-board count (x2 over the half-board prefixes), optionally with nodes."""
    nd = ctypes.c_uint64(0)
    s = lib.nq_oracle_total(N, rows, threads, ctypes.byref(nd) if with_nodes else None)
    return (int(s), int(nd.value)) if with_nodes else int(s)


class DihClass(ctypes.Structure):
    _fields_ = [("side_row", ctypes.c_int32), ("last_mask", ctypes.c_uint32), ("tie_bit", ctypes.c_uint32),
                ("w", ctypes.c_uint32), ("w_tie", ctypes.c_uint32)]


lib.nq_oracle_dihedral_expand.restype = ctypes.c_int64
lib.nq_oracle_dihedral_expand.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p,
                                          ctypes.POINTER(ctypes.c_uint8), ctypes.c_int64, ctypes.POINTER(DihClass),
                                          ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
lib.nq_oracle_dihedral_count_tasks.restype = None
lib.nq_oracle_dihedral_count_tasks.argtypes = [ctypes.c_int, ctypes.c_int64, _u32p, _u32p, _u32p,
                                               ctypes.POINTER(ctypes.c_uint8), ctypes.POINTER(DihClass), _u64p,
                                               ctypes.c_int]
lib.nq_oracle_dihedral_total.restype = ctypes.c_int64
lib.nq_oracle_dihedral_total.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]


def dihedral_expand(N: int, rows: int):
    """Dihedral decomposition tasks (dihedral_oracle.c): (cols, ld, rd, cls, classes as tuples)."""
    ncls = ctypes.c_int(0)
    n = lib.nq_oracle_dihedral_expand(N, rows, None, None, None, None, 0, None, 0, ctypes.byref(ncls))
    if n < 0:
        raise ValueError(f"bad (N, rows) = ({N}, {rows})")
    c, l, r = (np.empty(n, np.uint32) for _ in range(3))
    k = np.empty(n, np.uint8)
    tab = (DihClass * 64)()
    lib.nq_oracle_dihedral_expand(N, rows, _p(c, _u32p), _p(l, _u32p), _p(r, _u32p),
                                  k.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n, tab, 64, ctypes.byref(ncls))
    classes = [(t.side_row, t.last_mask, t.tie_bit, t.w, t.w_tie) for t in tab[:ncls.value]]
    return c, l, r, k, classes


def dihedral_count_tasks(N: int, rows: int, cols, ld, rd, cls, threads: int = 0) -> np.ndarray:
    """Weighted count of each dihedral task under its class's rules (OpenMP)."""
    ncls = ctypes.c_int(0)
    tab = (DihClass * 64)()
    lib.nq_oracle_dihedral_expand(N, rows, None, None, None, None, 0, tab, 64, ctypes.byref(ncls))
    cols = np.ascontiguousarray(cols, np.uint32)
    ld = np.ascontiguousarray(ld, np.uint32)
    rd = np.ascontiguousarray(rd, np.uint32)
    cls = np.ascontiguousarray(cls, np.uint8)
    if cls.size and int(cls.max()) >= ncls.value:
        raise ValueError("class index out of range")
    out = np.empty(cols.size, np.uint64)
    lib.nq_oracle_dihedral_count_tasks(N, cols.size, _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p),
                                       cls.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), tab, _p(out, _u64p),
                                       threads)
    return out


def dihedral_total(N: int, rows: int, threads: int = 0) -> int:
    """Whole-board total through the dihedral decomposition."""
    return int(lib.nq_oracle_dihedral_total(N, rows, threads))


_ref_lib = None


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref():
    """ctypes handle on the reference's own CPU code (oracle/_ref/libnq_ref.so)."""
    global _ref_lib
    if _ref_lib is None:
        if not os.path.exists(_REF_SO):
            raise FileNotFoundError(_REF_SO + " is not built (the reference sources were not available)")
        L = ctypes.CDLL(_REF_SO)
        L.nqref_n_queens.restype = ctypes.c_longlong
        L.nqref_n_queens.argtypes = [ctypes.c_int] * 4
        L.nqref_expand.restype = ctypes.c_longlong
        L.nqref_expand.argtypes = [ctypes.c_int, ctypes.c_int, _i32p, ctypes.c_longlong]
        L.nqref_serial.restype = ctypes.c_longlong
        L.nqref_serial.argtypes = [ctypes.c_int, ctypes.c_int]
        L.nqref_parallel.restype = ctypes.c_longlong
        L.nqref_parallel.argtypes = [ctypes.c_int, ctypes.c_int]
        L.nqref_count_tasks.restype = ctypes.c_longlong
        L.nqref_count_tasks.argtypes = [ctypes.c_int, ctypes.c_longlong, _i32p, _i64p, ctypes.c_int]
        _ref_lib = L
    return _ref_lib


def ref_expand_aos(N: int, rows: int) -> np.ndarray:
    """The reference expander's vector<int> (AoS c,l,r triples) as int32[n, 3]."""
    L = ref()
    n = L.nqref_expand(N, rows, None, 0)
    out = np.empty((n, 3), np.int32)
    L.nqref_expand(N, rows, _p(out, _i32p), n)
    return out


def ref_count_tasks(N: int, aos: np.ndarray, threads: int = 0, per_task: bool = False):
    """Reference n_queens() over a task list; returns the x2 sum (and per-task counts)."""
    L = ref()
    aos = np.ascontiguousarray(aos, np.int32).reshape(-1, 3)
    out = np.empty(aos.shape[0], np.int64) if per_task else None
    s = L.nqref_count_tasks(N, aos.shape[0], _p(aos, _i32p), _p(out, _i64p), threads)
    return (int(s), out) if per_task else int(s)
