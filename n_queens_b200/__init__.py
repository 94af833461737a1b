"""n_queens_b200 -- B200-native N-Queens solution counter (Python host mirror).

Thin ctypes layer over ``libnqueens_b200.so`` (the C ABI declared in
``include/n_queens_b200.h``).  Every count runs on the GPU; there is no CPU
path in this package.  If the shared library is missing the import fails
loudly -- build it with ``make -C n_queens_b200`` (``__graft_entry__.build()``).

Reference interface this mirrors (ygch/n_queens, ``src/n_queens.h``):

* :func:`cuda_n_queens` -- ``long long cuda_n_queens(int N, int rows)``
  (``src/n_queens_cuda.cu:84-186``): whole-board count, 2 x the sum over the
  half-board prefixes;
* :func:`partial_n_queens` -- the prefix expander (``src/n_queens.cpp:74-113``);
* :func:`n_queens` -- per-board completion count (``src/n_queens.cpp:8-21``),
  here counted on the GPU.

and adds the library's own entries: :func:`count`, :func:`count_tasks`,
:func:`count_tasks_device`, :func:`count_batch`, and (``n_queens_b200.learned``)
the learned subtree-cost scheduler.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnqueens_b200.so")
CLI_PATH = os.path.join(HERE, "n_queens")

NQ_OK = 0
NQ_ERR_ARG = -1
NQ_ERR_NO_DEVICE = -2
NQ_ERR_CUDA = -3
NQ_ERR_OOM = -4
NQ_ERR_DEPTH = -5
NQ_ERR_TIMEOUT = -6
NQ_ERR_NO_KERNEL = -7

NQ_ORDER_PLAIN = 0
NQ_ORDER_GIVEN = 1
NQ_MAX_N = 31
NQ_MAX_INNER_STEPS = 1 << 20
NQ_MAX_STACK_LEVELS = 32


class NQError(RuntimeError):
    """A non-zero nq_status from the library."""

    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {status_string(status)} ({status})" + (f": {detail}" if detail else ""))


class Config(ctypes.Structure):
    """Mirror of ``nq_config``; zero fields mean "default"."""

    _fields_ = [
        ("block_threads", ctypes.c_int),
        ("blocks_per_sm", ctypes.c_int),
        ("stack_levels", ctypes.c_int),
        ("steal", ctypes.c_int),
        ("inner_steps", ctypes.c_int),
        ("order_kind", ctypes.c_int),
        ("order", ctypes.c_void_p),
        ("time_limit_ms", ctypes.c_uint32),
        ("device", ctypes.c_int),
        ("timing", ctypes.c_int),
        ("layout", ctypes.c_int),
        ("device_expand", ctypes.c_int),
        ("queue_len", ctypes.c_uint32),
        ("reserved", ctypes.c_int * 2),
    ]


class Stats(ctypes.Structure):
    """Mirror of ``nq_stats``."""

    _fields_ = [
        ("expand_ms", ctypes.c_double),
        ("h2d_ms", ctypes.c_double),
        ("kernel_ms", ctypes.c_double),
        ("d2h_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("tasks", ctypes.c_int64),
        ("nodes", ctypes.c_uint64),
        ("grid", ctypes.c_int),
        ("block_threads", ctypes.c_int),
        ("stack_levels", ctypes.c_int),
        ("smem_bytes", ctypes.c_int),
        ("reserved", ctypes.c_int * 5),
        ("makespan_ms", ctypes.c_double),
        ("cta_busy_mean_ms", ctypes.c_double),
        ("tail_idle_frac", ctypes.c_double),
        ("schedule_ms", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class TuneEntry(ctypes.Structure):
    """Mirror of ``nq_tune_entry``."""

    _fields_ = [("split_rows", ctypes.c_int), ("block_threads", ctypes.c_int), ("layout", ctypes.c_int),
                ("inner_steps", ctypes.c_int), ("ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class DihedralClass(ctypes.Structure):
    """``nq_dihedral_class``: the search rules and weights of one dihedral class."""
    _fields_ = [("side_row", ctypes.c_int32), ("last_mask", ctypes.c_uint32), ("tie_bit", ctypes.c_uint32),
                ("weight", ctypes.c_uint32), ("weight_tie", ctypes.c_uint32)]


class Instance(ctypes.Structure):
    """Mirror of ``nq_instance``: one partial board."""

    _fields_ = [("N", ctypes.c_int32), ("cols", ctypes.c_uint32), ("ld", ctypes.c_uint32), ("rd", ctypes.c_uint32)]


_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_cfgp = ctypes.POINTER(Config)
_stp = ctypes.POINTER(Stats)


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: the CUDA library must be built (make -C {HERE}); "
            "n_queens_b200 has no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    L.nq_abi_version.restype = ctypes.c_int
    L.nq_status_string.restype = ctypes.c_char_p
    L.nq_status_string.argtypes = [ctypes.c_int]
    L.nq_last_error.restype = ctypes.c_char_p
    L.nq_device_count.restype = ctypes.c_int
    L.nq_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
    L.nq_stack_levels.restype = ctypes.c_int
    L.nq_stack_levels.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.nq_expand.restype = ctypes.c_int
    L.nq_expand.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_int64, _i64p, ctypes.c_int]
    L.nq_expand_device.restype = ctypes.c_int
    L.nq_expand_device.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_int64, _i64p, ctypes.c_int, ctypes.c_void_p]
    L.nq_count.restype = ctypes.c_int
    L.nq_count.argtypes = [ctypes.c_int, ctypes.c_int, _cfgp, _u64p, _u64p, _stp]
    L.nq_count_resumable.restype = ctypes.c_int
    L.nq_count_resumable.argtypes = [ctypes.c_int, ctypes.c_int, _cfgp, ctypes.c_char_p, _u64p,
                                     ctypes.POINTER(ctypes.c_int), _stp]
    L.nq_count_tasks.restype = ctypes.c_int
    L.nq_count_tasks.argtypes = [ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_int64, _u64p, _u64p, _u64p, _cfgp,
                                 _stp]
    L.nq_count_tasks_device.restype = ctypes.c_int
    L.nq_count_tasks_device.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _cfgp,
                                        ctypes.c_void_p]
    L.nq_count_tasks_device_noalloc.restype = ctypes.c_int
    L.nq_count_tasks_device_noalloc.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_int64, ctypes.c_void_p, _cfgp, ctypes.c_void_p]
    L.nq_batch_create.restype = ctypes.c_int
    L.nq_batch_create.argtypes = [ctypes.POINTER(Instance), ctypes.c_int64, ctypes.c_int, _cfgp,
                                  ctypes.POINTER(ctypes.c_void_p)]
    L.nq_batch_run.restype = ctypes.c_int
    L.nq_batch_run.argtypes = [ctypes.c_void_p, _u64p, _stp]
    L.nq_batch_destroy.restype = ctypes.c_int
    L.nq_batch_destroy.argtypes = [ctypes.c_void_p]
    L.nq_batch_autotune.restype = ctypes.c_int
    L.nq_batch_autotune.argtypes = [ctypes.POINTER(Instance), ctypes.c_int64, ctypes.c_int, _cfgp,
                                    ctypes.POINTER(TuneEntry), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(TuneEntry)]
    L.nq_count_batch.restype = ctypes.c_int
    L.nq_count_batch.argtypes = [ctypes.POINTER(Instance), ctypes.c_int64, ctypes.c_int, _u64p, _cfgp, _stp]
    L.nq_dihedral_expand.restype = ctypes.c_int
    L.nq_dihedral_expand.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, _u8p, ctypes.c_int64, _i64p,
                                     ctypes.POINTER(DihedralClass), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.nq_count_dihedral.restype = ctypes.c_int
    L.nq_count_dihedral.argtypes = [ctypes.c_int, ctypes.c_int, _cfgp, _u64p, _stp]
    L.nq_count_dihedral_resumable.restype = ctypes.c_int
    L.nq_count_dihedral_resumable.argtypes = [ctypes.c_int, ctypes.c_int, _cfgp, ctypes.c_char_p, _u64p,
                                              ctypes.POINTER(ctypes.c_int), _stp]
    L.nq_count_dihedral_tasks.restype = ctypes.c_int
    L.nq_count_dihedral_tasks.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, _u32p, _u8p, ctypes.c_int64,
                                          _u64p, _u64p, _cfgp, _stp]
    return L


lib = _load()

# Every symbol the C header declares (checked by the CPU test suite).
EXPORTS = ("nq_abi_version", "nq_status_string", "nq_last_error", "nq_device_count", "nq_stack_levels", "nq_expand",
           "nq_expand_device", "nq_count",
           "nq_count_resumable",
           "nq_count_tasks", "nq_count_tasks_device", "nq_count_tasks_device_noalloc", "nq_count_batch",
           "nq_batch_create", "nq_batch_run", "nq_batch_destroy", "nq_batch_autotune",
           "nq_mlp_num_params", "nq_mlp_create", "nq_mlp_destroy", "nq_mlp_get_params", "nq_mlp_set_params",
           "nq_mlp_predict", "nq_mlp_predict_tensor", "nq_mlp_grad", "nq_mlp_train", "nq_schedule_device",
           "nq_schedule_device_last", "nq_count_learned", "nq_count_learned_reuse",
           "nq_dihedral_expand", "nq_count_dihedral", "nq_count_dihedral_tasks",
           "nq_count_dihedral_resumable")


def status_string(status: int) -> str:
    return lib.nq_status_string(status).decode()


def last_error() -> str:
    return lib.nq_last_error().decode()


def _check(rc: int, where: str) -> None:
    if rc != NQ_OK:
        raise NQError(rc, where, last_error())


def _cfg(config) -> ctypes.POINTER(Config) | None:
    if config is None:
        return None
    if isinstance(config, Config):
        return ctypes.pointer(config)
    c = Config()
    for k, v in dict(config).items():
        setattr(c, k, v)
    return ctypes.pointer(c)


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def stack_levels(N: int, rows: int, nodes: bool = False) -> int:
    """Stack slots per lane that a count of (N, rows) prefixes needs (nq_stack_levels)."""
    v = lib.nq_stack_levels(N, rows, 1 if nodes else 0)
    if v < 0:
        raise NQError(v, "nq_stack_levels")
    return v


def device_count() -> int:
    n = ctypes.c_int(0)
    _check(lib.nq_device_count(ctypes.byref(n)), "nq_device_count")
    return n.value


def expand(N: int, rows: int, threads: int = 0):
    """Half-board prefixes as SoA uint32 (cols, ld, rd), reference order."""
    n = ctypes.c_int64(0)
    _check(lib.nq_expand(N, rows, None, None, None, 0, ctypes.byref(n), threads), "nq_expand")
    c = np.empty(n.value, np.uint32)
    l = np.empty(n.value, np.uint32)
    r = np.empty(n.value, np.uint32)
    _check(lib.nq_expand(N, rows, _p(c, _u32p), _p(l, _u32p), _p(r, _u32p), n.value, ctypes.byref(n), threads),
           "nq_expand")
    return c, l, r


def partial_n_queens(N: int, rows: int) -> np.ndarray:
    """The reference expander's output (``vector<int>`` of c,l,r triples) as int32[n, 3]."""
    c, l, r = expand(N, rows)
    return np.stack([c, l, r], axis=1).view(np.int32)


@dataclass
class CountResult:
    total: int
    nodes: int | None
    stats: dict


def count(N: int, rows: int, config=None, nodes: bool = False) -> CountResult:
    """Whole-board count on the GPU (``nq_count``): 2 x the sum over prefixes."""
    tot = ctypes.c_uint64(0)
    nd = ctypes.c_uint64(0)
    st = Stats()
    rc = lib.nq_count(N, rows, _cfg(config), ctypes.byref(tot), ctypes.byref(nd) if nodes else None,
                      ctypes.byref(st))
    _check(rc, "nq_count")
    return CountResult(int(tot.value), int(nd.value) if nodes else None, st.as_dict())


def dihedral_expand(N: int, rows: int):
    """Dihedral (8-fold) task list of (N, rows) (``nq_dihedral_expand``).

    Returns ``(cols, ld, rd, cls, classes)``: uint32 arrays, the uint8 class
    index per task, and the class table as a list of dicts.
    """
    n = ctypes.c_int64(0)
    ncls = ctypes.c_int(0)
    _check(lib.nq_dihedral_expand(N, rows, None, None, None, None, 0, ctypes.byref(n), None, 0, ctypes.byref(ncls)),
           "nq_dihedral_expand")
    c, l, r = (np.empty(n.value, np.uint32) for _ in range(3))
    k = np.empty(n.value, np.uint8)
    tab = (DihedralClass * max(ncls.value, 1))()
    _check(lib.nq_dihedral_expand(N, rows, _p(c, _u32p), _p(l, _u32p), _p(r, _u32p), _p(k, _u8p), n.value,
                                  ctypes.byref(n), tab, ncls.value, ctypes.byref(ncls)), "nq_dihedral_expand")
    classes = [{f: getattr(tab[i], f) for f, _ in DihedralClass._fields_} for i in range(ncls.value)]
    return c, l, r, k, classes


def count_dihedral(N: int, rows: int, config=None) -> CountResult:
    """Whole-board count through the dihedral decomposition (``nq_count_dihedral``)."""
    tot = ctypes.c_uint64(0)
    st = Stats()
    rc = lib.nq_count_dihedral(N, rows, _cfg(config), ctypes.byref(tot), ctypes.byref(st))
    _check(rc, "nq_count_dihedral")
    return CountResult(int(tot.value), None, st.as_dict())


def count_dihedral_tasks(N: int, rows: int, cols, ld, rd, cls, per_task: bool = False, config=None) -> dict:
    """Weighted counts of dihedral tasks (``nq_count_dihedral_tasks``)."""
    cols = np.ascontiguousarray(cols, np.uint32)
    ld = np.ascontiguousarray(ld, np.uint32)
    rd = np.ascontiguousarray(rd, np.uint32)
    cls = np.ascontiguousarray(cls, np.uint8)
    n = cols.size
    if ld.size != n or rd.size != n or cls.size != n:
        raise ValueError("cols, ld, rd and cls must have the same length")
    pt = np.empty(n, np.uint64) if per_task else None
    s = ctypes.c_uint64(0)
    st = Stats()
    rc = lib.nq_count_dihedral_tasks(N, rows, _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p), _p(cls, _u8p), n,
                                     _p(pt, _u64p), ctypes.byref(s), _cfg(config), ctypes.byref(st))
    _check(rc, "nq_count_dihedral_tasks")
    return {"sum": int(s.value), "per_task": pt, "stats": st.as_dict()}


def count_resumable(N: int, rows: int, checkpoint: str, slice_ms: int = 0, config=None, dihedral: bool = False):
    """One slice of a resumable whole-board count (``nq_count_resumable``, or
    ``nq_count_dihedral_resumable`` with ``dihedral=True``).

    Returns (done, total, stats); total is valid once done.  Call again with
    the same checkpoint path until done.
    """
    c = Config()
    if config is not None:
        for k, v in (config.items() if isinstance(config, dict) else []):
            setattr(c, k, v)
        if isinstance(config, Config):
            c = config
    c.time_limit_ms = slice_ms
    tot = ctypes.c_uint64(0)
    done = ctypes.c_int(0)
    st = Stats()
    fn = lib.nq_count_dihedral_resumable if dihedral else lib.nq_count_resumable
    rc = fn(N, rows, ctypes.byref(c), os.fsencode(checkpoint), ctypes.byref(tot), ctypes.byref(done),
            ctypes.byref(st))
    _check(rc, "nq_count_dihedral_resumable" if dihedral else "nq_count_resumable")
    return bool(done.value), int(tot.value), st.as_dict()


def cuda_n_queens(N: int, rows: int) -> int:
    """Same value as the reference's ``cuda_n_queens`` (-1 when there is no GPU)."""
    tot = ctypes.c_uint64(0)
    rc = lib.nq_count(N, rows, None, ctypes.byref(tot), None, None)
    if rc == NQ_ERR_NO_DEVICE:
        return -1
    _check(rc, "nq_count")
    return int(tot.value)


def count_tasks(N: int, cols, ld, rd, per_task: bool = False, nodes: bool = False, config=None) -> dict:
    """Counts over a host task list (``nq_count_tasks``).

    Returns ``{"sum", "per_task" (uint64[n] or None), "nodes" (uint64[n] or None), "stats"}``.
    """
    cols = np.ascontiguousarray(cols, np.uint32)
    ld = np.ascontiguousarray(ld, np.uint32)
    rd = np.ascontiguousarray(rd, np.uint32)
    n = cols.size
    if ld.size != n or rd.size != n:
        raise ValueError("cols, ld and rd must have the same length")
    pt = np.empty(n, np.uint64) if per_task else None
    nd = np.empty(n, np.uint64) if nodes else None
    s = ctypes.c_uint64(0)
    st = Stats()
    rc = lib.nq_count_tasks(N, _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p), n, _p(pt, _u64p), _p(nd, _u64p),
                            ctypes.byref(s), _cfg(config), ctypes.byref(st))
    _check(rc, "nq_count_tasks")
    return {"sum": int(s.value), "per_task": pt, "nodes": nd, "stats": st.as_dict()}


def count_tasks_device(N: int, cols, ld, rd, sum_out, per_task=None, nodes=None, config=None, stream=None) -> None:
    """Enqueues a count over device-resident tasks (torch CUDA tensors).

    ``sum_out`` is a CUDA int64 tensor of 2 elements: [0] the sum, [1] status
    bits (1 = a task was too deep, 2 = time limit).  Nothing is synchronised.
    """
    n = cols.numel()
    ptr = lambda t: None if t is None else t.data_ptr()
    s = stream.cuda_stream if stream is not None else None
    rc = lib.nq_count_tasks_device(N, ptr(cols), ptr(ld), ptr(rd), n, ptr(per_task), ptr(nodes), ptr(sum_out),
                                   _cfg(config), s)
    _check(rc, "nq_count_tasks_device")


def count_batch(instances, split_rows: int = 0, config=None, return_stats: bool = False):
    """Completions of many independent partial boards in one launch.

    ``instances`` is a sequence of (N, cols, ld, rd) tuples.
    """
    n = len(instances)
    arr = (Instance * max(n, 1))()
    for i, (N, c, l, r) in enumerate(instances):
        arr[i] = Instance(int(N), int(c) & 0xFFFFFFFF, int(l) & 0xFFFFFFFF, int(r) & 0xFFFFFFFF)
    out = np.zeros(n, np.uint64)
    st = Stats()
    rc = lib.nq_count_batch(arr, n, split_rows, _p(out, _u64p), _cfg(config), ctypes.byref(st))
    _check(rc, "nq_count_batch")
    return (out, st.as_dict()) if return_stats else out


def _instances(instances):
    n = len(instances)
    arr = (Instance * max(n, 1))()
    for i, (N, c, l, r) in enumerate(instances):
        arr[i] = Instance(int(N), int(c) & 0xFFFFFFFF, int(l) & 0xFFFFFFFF, int(r) & 0xFFFFFFFF)
    return arr, n


class BatchPlan:
    """A reusable, graph-captured batch (``nq_batch_create`` / ``nq_batch_run``)."""

    def __init__(self, instances, split_rows: int = 0, config=None):
        arr, self.n = _instances(instances)
        self._h = ctypes.c_void_p()
        _check(lib.nq_batch_create(arr, self.n, split_rows, _cfg(config), ctypes.byref(self._h)), "nq_batch_create")

    def run(self, return_stats: bool = False):
        out = np.zeros(self.n, np.uint64)
        st = Stats()
        _check(lib.nq_batch_run(self._h, _p(out, _u64p), ctypes.byref(st)), "nq_batch_run")
        return (out, st.as_dict()) if return_stats else out

    def close(self):
        if self._h:
            lib.nq_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune_batch(instances, repeats: int = 2, config=None):
    """Sweeps split depth, CTA size, stack layout and queue chunking; returns (best, table)."""
    arr, n = _instances(instances)
    table = (TuneEntry * 64)()
    cnt = ctypes.c_int(0)
    best = TuneEntry()
    _check(lib.nq_batch_autotune(arr, n, repeats, _cfg(config), table, 64, ctypes.byref(cnt), ctypes.byref(best)),
           "nq_batch_autotune")
    return best.as_dict(), [table[i].as_dict() for i in range(min(cnt.value, 64))]


def n_queens(N: int, cur: int, left: int, right: int) -> int:
    """Completions of one partial board (reference ``n_queens``, no x2), on the GPU."""
    return int(count_batch([(N, cur, left, right)])[0])
