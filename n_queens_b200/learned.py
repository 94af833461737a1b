"""Learned subtree-cost scheduling (host side).

The learned scheduling pipeline, on top of the C ABI in mlp.cu/capi.cu:

1. the solver logs per-prefix DFS node counts at small N (``solver_labels``:
   nq_count_tasks with per-task nodes), target = log2(1 + nodes);
2. an MLP (96 -> 128 -> 128 -> 1, BF16 weights, FP32 accumulation, Adam) is
   trained on N = 16, 17, 18 by the library's own GPU kernels and fine-tuned
   on a seeded sample of the target board's prefixes (``build_cost_model``);
3. the model orders the target's task queue longest-first on the device and
   the count runs with that order (``count_learned`` -> nq_count_learned).

The order never changes a count; it only decides which lane runs which task
and when, which shows up in the makespan and the tail idle time.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np

from . import (NQError, Stats, _cfg, _check, _p, _u32p, _u64p, count_tasks, expand, lib, CountResult)

_f32p = ctypes.POINTER(ctypes.c_float)
_u8p = ctypes.POINTER(ctypes.c_uint8)


class _Mlp(ctypes.Structure):
    pass


_mlpp = ctypes.POINTER(_Mlp)


def _declare():
    L = lib
    L.nq_mlp_num_params.restype = ctypes.c_int
    L.nq_mlp_create.restype = ctypes.c_int
    L.nq_mlp_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(_mlpp)]
    L.nq_mlp_destroy.restype = ctypes.c_int
    L.nq_mlp_destroy.argtypes = [_mlpp]
    L.nq_mlp_get_params.restype = ctypes.c_int
    L.nq_mlp_get_params.argtypes = [_mlpp, _f32p]
    L.nq_mlp_set_params.restype = ctypes.c_int
    L.nq_mlp_set_params.argtypes = [_mlpp, _f32p]
    L.nq_mlp_predict.restype = ctypes.c_int
    L.nq_mlp_predict.argtypes = [_mlpp, ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_int64, _f32p]
    L.nq_mlp_predict_tensor.restype = ctypes.c_int
    L.nq_mlp_predict_tensor.argtypes = [_mlpp, ctypes.c_int, _u32p, _u32p, _u32p, ctypes.c_int64, _f32p]
    L.nq_mlp_grad.restype = ctypes.c_int
    L.nq_mlp_grad.argtypes = [_mlpp, _u8p, _u32p, _u32p, _u32p, _f32p, ctypes.c_int64, _f32p, _f32p]
    L.nq_mlp_train.restype = ctypes.c_int
    L.nq_mlp_train.argtypes = [_mlpp, _u8p, _u32p, _u32p, _u32p, _f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                               ctypes.c_float, ctypes.c_uint64, _f32p]
    L.nq_schedule_device.restype = ctypes.c_int
    L.nq_schedule_device.argtypes = [_mlpp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.nq_schedule_device_last.restype = ctypes.c_int
    L.nq_schedule_device_last.argtypes = [_mlpp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]
    L.nq_count_learned.restype = ctypes.c_int
    L.nq_count_learned.argtypes = [ctypes.c_int, ctypes.c_int, _mlpp, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.POINTER(Stats)]
    L.nq_count_learned_reuse.restype = ctypes.c_int
    L.nq_count_learned_reuse.argtypes = [ctypes.c_int, ctypes.c_int, _mlpp, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.c_int64, ctypes.c_uint64, ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(Stats)]


_declare()
NUM_PARAMS = lib.nq_mlp_num_params()


def _u32(a):
    return np.ascontiguousarray(a, np.uint32)


class CostModel:
    """A device-resident cost model (wraps nq_mlp)."""

    def __init__(self, seed: int = 0, device: int = 0):
        self._m = _mlpp()
        _check(lib.nq_mlp_create(device, seed, ctypes.byref(self._m)), "nq_mlp_create")
        self.device = device

    def close(self):
        if self._m:
            lib.nq_mlp_destroy(self._m)
            self._m = _mlpp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        out = np.empty(NUM_PARAMS, np.float32)
        _check(lib.nq_mlp_get_params(self._m, _p(out, _f32p)), "nq_mlp_get_params")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == NUM_PARAMS
        _check(lib.nq_mlp_set_params(self._m, _p(p, _f32p)), "nq_mlp_set_params")

    def predict(self, N: int, cols, ld, rd) -> np.ndarray:
        cols, ld, rd = _u32(cols), _u32(ld), _u32(rd)
        out = np.empty(cols.size, np.float32)
        _check(lib.nq_mlp_predict(self._m, N, _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p), cols.size,
                                  _p(out, _f32p)), "nq_mlp_predict")
        return out

    def predict_tensor(self, N: int, cols, ld, rd) -> np.ndarray:
        """Forward on the tensor cores (tcgen05), as the scheduler runs it."""
        cols, ld, rd = _u32(cols), _u32(ld), _u32(rd)
        out = np.empty(cols.size, np.float32)
        _check(lib.nq_mlp_predict_tensor(self._m, N, _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p), cols.size,
                                         _p(out, _f32p)), "nq_mlp_predict_tensor")
        return out

    def grad(self, task_n, cols, ld, rd, target):
        task_n = np.ascontiguousarray(task_n, np.uint8)
        cols, ld, rd = _u32(cols), _u32(ld), _u32(rd)
        target = np.ascontiguousarray(target, np.float32)
        g = np.empty(NUM_PARAMS, np.float32)
        loss = ctypes.c_float(0)
        _check(lib.nq_mlp_grad(self._m, _p(task_n, _u8p), _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p),
                               _p(target, _f32p), cols.size, _p(g, _f32p), ctypes.byref(loss)), "nq_mlp_grad")
        return g, loss.value

    def train(self, task_n, cols, ld, rd, target, epochs: int, batch: int = 4096, lr: float = 2e-3,
              seed: int = 0) -> np.ndarray:
        task_n = np.ascontiguousarray(task_n, np.uint8)
        cols, ld, rd = _u32(cols), _u32(ld), _u32(rd)
        target = np.ascontiguousarray(target, np.float32)
        losses = np.zeros(max(epochs, 1), np.float32)
        _check(lib.nq_mlp_train(self._m, _p(task_n, _u8p), _p(cols, _u32p), _p(ld, _u32p), _p(rd, _u32p),
                                _p(target, _f32p), cols.size, epochs, batch, lr, seed, _p(losses, _f32p)),
               "nq_mlp_train")
        return losses[:epochs]


def solver_labels(N: int, k: int, index=None, config=None):
    """Prefix tasks of (N, k) (optionally a subset) with the solver's own node counts.

    Returns (cols, ld, rd, target, nodes, counts) with target = log2(1 + nodes).
    """
    cols, ld, rd = expand(N, k)
    if index is not None:
        cols, ld, rd = cols[index], ld[index], rd[index]
    res = count_tasks(N, cols, ld, rd, per_task=True, nodes=True,
                      config=config if config is not None else dict(stack_levels=N - 1 - k))
    nodes = res["nodes"]
    target = np.log2(nodes.astype(np.float64) + 1.0).astype(np.float32)
    return cols, ld, rd, target, nodes, res["per_task"]


def spearman(a, b) -> float:
    ra = np.argsort(np.argsort(a, kind="stable"), kind="stable").astype(np.float64)
    rb = np.argsort(np.argsort(b, kind="stable"), kind="stable").astype(np.float64)
    return float(np.corrcoef(ra, rb)[0, 1])


@dataclass
class BuildReport:
    label_s: float = 0.0
    pretrain_s: float = 0.0
    finetune_label_s: float = 0.0
    finetune_s: float = 0.0
    pretrain_losses: list = field(default_factory=list)
    finetune_losses: list = field(default_factory=list)
    holdout_spearman: float = float("nan")
    holdout_rmse: float = float("nan")
    train_samples: int = 0
    finetune_samples: int = 0
    # The target board's tasks that the build counted exactly while labelling
    # (fine-tuning sample and hold-out), and the plain sum of their counts:
    # count_learned(..., reuse=report) skips them and adds the sum.
    target_N: int = 0
    k: int = 0
    counted_idx: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    counted_sum: int = 0


def build_cost_model(target_N: int, k: int = 6, train_N=(16, 17, 18), finetune_frac: float = 0.05,
                     seed: int = 0, pre_epochs: int = 4, ft_epochs: int = 8, batch: int = 4096, lr: float = 2e-3,
                     device: int = 0, holdout: int = 200_000):
    """Trains the cost model on the solver's logs at train_N and fine-tunes on a
    seeded finetune_frac sample of target_N's prefixes.  Returns (model, report)."""
    rep = BuildReport()
    t = time.perf_counter()
    parts = [solver_labels(Nt, k) for Nt in train_N]
    rep.label_s = time.perf_counter() - t
    tn = np.concatenate([np.full(p[0].size, Nt, np.uint8) for p, Nt in zip(parts, train_N)])
    c = np.concatenate([p[0] for p in parts])
    l = np.concatenate([p[1] for p in parts])
    r = np.concatenate([p[2] for p in parts])
    y = np.concatenate([p[3] for p in parts])
    rep.train_samples = int(c.size)
    model = CostModel(seed=seed, device=device)
    # Start the output bias at the label mean (faster, steadier first epoch).
    p = model.params()
    p[-1] = float(y.mean())
    model.set_params(p)
    t = time.perf_counter()
    rep.pretrain_losses = model.train(tn, c, l, r, y, pre_epochs, batch, lr, seed).tolist()
    rep.pretrain_s = time.perf_counter() - t

    cols, ld, rd = expand(target_N, k)
    rng = np.random.default_rng(seed)
    nsample = max(1, int(round(finetune_frac * cols.size)))
    perm = rng.permutation(cols.size)
    sample = np.sort(perm[:nsample])
    t = time.perf_counter()
    fc, fl, fr, fy, _, fcnt = solver_labels(target_N, k, index=sample)
    rep.finetune_label_s = time.perf_counter() - t
    counted = [(sample, fcnt)]
    rep.finetune_samples = int(nsample)
    t = time.perf_counter()
    rep.finetune_losses = model.train(np.full(nsample, target_N, np.uint8), fc, fl, fr, fy, ft_epochs, batch, lr,
                                      seed + 1).tolist()
    rep.finetune_s = time.perf_counter() - t
    # Hold-out quality on prefixes outside the fine-tuning sample.
    ho = np.sort(perm[nsample:nsample + min(holdout, cols.size - nsample)])
    if ho.size:
        hc, hl, hr, hy, _, hcnt = solver_labels(target_N, k, index=ho)
        counted.append((ho, hcnt))
        pred = model.predict(target_N, hc, hl, hr)
        rep.holdout_spearman = spearman(pred, hy)
        rep.holdout_rmse = float(np.sqrt(np.mean((pred.astype(np.float64) - hy) ** 2)))
    idx = np.concatenate([i for i, _ in counted]).astype(np.int64)
    cnt = np.concatenate([c for _, c in counted])
    o = np.argsort(idx, kind="stable")
    rep.target_N, rep.k = target_N, k
    rep.counted_idx = np.ascontiguousarray(idx[o])
    rep.counted_sum = int(cnt.sum(dtype=np.uint64))
    return model, rep


def count_learned(N: int, rows: int, model: CostModel, config=None, reuse: BuildReport | None = None) -> CountResult:
    """Whole-board count with the model's longest-first order (nq_count_learned).

    With ``reuse`` (the report of the build that made ``model`` for this
    board), the tasks the build already counted exactly are left out of the
    queue and their sum is added (nq_count_learned_reuse): the labelling work
    becomes part of the count."""
    tot = ctypes.c_uint64(0)
    st = Stats()
    cfg = _cfg(config)
    cfgp = ctypes.cast(cfg, ctypes.c_void_p) if cfg else None
    if reuse is None:
        rc = lib.nq_count_learned(N, rows, model._m, cfgp, ctypes.byref(tot), ctypes.byref(st))
        _check(rc, "nq_count_learned")
    else:
        if (reuse.target_N, reuse.k) != (N, rows):
            raise ValueError(f"the report labels N={reuse.target_N} k={reuse.k}, not N={N} k={rows}")
        idx = np.ascontiguousarray(reuse.counted_idx, np.int64)
        rc = lib.nq_count_learned_reuse(N, rows, model._m, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                        idx.size, reuse.counted_sum, cfgp, ctypes.byref(tot), ctypes.byref(st))
        _check(rc, "nq_count_learned_reuse")
    return CountResult(int(tot.value), None, st.as_dict())
