"""The learned subtree-cost scheduler on the GPU: the hand-written MLP kernels
against the CPU oracle (oracle/mlp_ref.py), training, the longest-first
order, exact counts with that order, and what the order gains."""
import numpy as np
import pytest

import oracle
from oracle import mlp_ref

pytestmark = pytest.mark.gpu

# Tolerances: the GPU accumulates in FP32 (different summation order), the
# oracle in float64, both with the same BF16-rounded weights.
GRAD_RTOL_MAX = 2e-3      # max |g_gpu - g_ref| <= 2e-3 * max |g_ref|
GRAD_RTOL_L2 = 2e-4       # ||g_gpu - g_ref|| <= 2e-4 * ||g_ref||
PRED_ATOL = 2e-3          # |pred_gpu - pred_ref| for outputs of size ~10
# Tensor-core forward: an FP32 layer-1 sum that lands next to a BF16 rounding
# boundary may round the other way than the oracle's float64 sum (one BF16 ulp
# of that activation), so the bound is looser than PRED_ATOL.
TC_ATOL_MAX = 2e-2
TC_ATOL_MEAN = 1e-3


def _params(seed):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-0.15, 0.15, mlp_ref.NPARAMS).astype(np.float32)
    p[mlp_ref.OFF_B1:mlp_ref.OFF_W2] += 0.05
    p[mlp_ref.OFF_B2:mlp_ref.OFF_W3] += 0.05
    p[mlp_ref.OFF_B3] = 10.0
    return p


def _mixed_tasks():
    cs, ls, rs, ns = [], [], [], []
    for N, k in ((12, 4), (13, 5), (15, 3)):
        c, l, r = oracle.expand(N, k)
        sel = np.random.default_rng(N).choice(c.size, min(400, c.size), replace=False)
        cs.append(c[sel]); ls.append(l[sel]); rs.append(r[sel]); ns.append(np.full(sel.size, N, np.uint8))
    return np.concatenate(ns), np.concatenate(cs), np.concatenate(ls), np.concatenate(rs)


def test_gradients_match_cpu_oracle(gpu):
    from n_queens_b200 import learned
    tn, c, l, r = _mixed_tasks()
    y = np.random.default_rng(3).uniform(4, 16, c.size).astype(np.float32)
    m = learned.CostModel(seed=5)
    for seed in (1, 2):
        p = _params(seed)
        m.set_params(p)
        g, loss = m.grad(tn, c, l, r, y)
        X = np.concatenate([mlp_ref.features(int(N), c[tn == N], l[tn == N], r[tn == N]) for N in np.unique(tn)])
        order = np.concatenate([np.flatnonzero(tn == N) for N in np.unique(tn)])
        ref_loss, ref_g = mlp_ref.loss_and_grad(p, X, y[order])
        assert abs(loss - ref_loss) <= 1e-5 * ref_loss
        err = np.abs(g.astype(np.float64) - ref_g)
        assert err.max() <= GRAD_RTOL_MAX * np.abs(ref_g).max()
        assert np.linalg.norm(err) <= GRAD_RTOL_L2 * np.linalg.norm(ref_g)
    m.close()


def test_predictions_match_cpu_oracle(gpu):
    from n_queens_b200 import learned
    m = learned.CostModel(seed=5)
    p = _params(4)
    m.set_params(p)
    for N, k in ((12, 4), (16, 5)):
        c, l, r = oracle.expand(N, k)
        c, l, r = c[:3000], l[:3000], r[:3000]
        got = m.predict(N, c, l, r)
        want, _ = mlp_ref.forward(p, mlp_ref.features(N, c, l, r))
        assert np.abs(got - want).max() <= PRED_ATOL
    assert np.array_equal(m.params(), p)
    m.close()


def test_training_lowers_loss_and_ranks_tasks(gpu):
    from n_queens_b200 import learned
    c, l, r, y, nodes, _ = learned.solver_labels(15, 5)
    assert np.array_equal(nodes, oracle.count_tasks(15, c, l, r, nodes=True)[1])
    tn = np.full(c.size, 15, np.uint8)
    m = learned.CostModel(seed=11)
    p = m.params(); p[-1] = float(y.mean()); m.set_params(p)
    g0, loss0 = m.grad(tn, c, l, r, y)
    losses = m.train(tn, c, l, r, y, epochs=6, batch=1024, lr=2e-3, seed=3)
    _, loss1 = m.grad(tn, c, l, r, y)
    assert loss1 < 0.5 * loss0 and losses[-1] < losses[0]
    assert learned.spearman(m.predict(15, c, l, r), y) > 0.6
    m.close()


def test_schedule_is_a_longest_first_permutation(gpu):
    import torch
    from n_queens_b200 import learned
    m = learned.CostModel(seed=2)
    m.set_params(_params(6))
    c, l, r = oracle.expand(16, 5)
    dev = torch.device("cuda:0")
    tc, tl, tr = (torch.from_numpy(a.view(np.int32)).to(dev) for a in (c, l, r))  # keep them alive
    order = torch.empty(c.size, dtype=torch.int32, device=dev)
    pred = torch.empty(c.size, dtype=torch.float32, device=dev)
    rc = learned.lib.nq_schedule_device(m._m, 16, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), c.size,
                                        order.data_ptr(), pred.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    o = order.cpu().numpy().view(np.uint32).astype(np.int64)
    pr = pred.cpu().numpy()
    assert np.array_equal(np.sort(o), np.arange(c.size))
    keys = np.clip(np.floor(pr * 8 + 0.5), 0, 65535).astype(np.int64)[o]
    assert np.all(np.diff(keys) <= 0)                      # longest first
    same = np.diff(keys) == 0
    assert np.all(np.diff(o)[same] > 0)                    # stable inside a bin
    assert np.array_equal(pr, m.predict_tensor(16, c, l, r))   # the scheduler runs the tensor-core forward
    m.close()


def test_tensor_core_forward_matches_oracle(gpu):
    # tcgen05 forward: BF16 operands (the layer-1 outputs rounded to BF16),
    # FP32 accumulation in TMEM.  Against the oracle with the same rounding,
    # and against the CUDA-core forward (which keeps layer 1 in FP32).
    from n_queens_b200 import learned
    m = learned.CostModel(seed=5)
    for seed, (N, k) in ((4, (12, 4)), (8, (16, 5)), (9, (17, 6))):
        p = _params(seed)
        m.set_params(p)
        c, l, r = oracle.expand(N, k)
        sel = np.random.default_rng(seed).choice(c.size, min(5000, c.size), replace=False)
        c, l, r = c[sel], l[sel], r[sel]
        got = m.predict_tensor(N, c, l, r)
        want, _ = mlp_ref.forward(p, mlp_ref.features(N, c, l, r), h1_bf16=True)
        err = np.abs(got - want)
        assert err.max() <= TC_ATOL_MAX and err.mean() <= TC_ATOL_MEAN, (err.max(), err.mean())
        assert np.abs(got - m.predict(N, c, l, r)).max() <= 0.05
    m.close()


def test_learned_count_is_exact_and_front_loads_work(gpu, golden):
    from n_queens_b200 import learned
    pub = golden("published.json")
    model, rep = learned.build_cost_model(18, k=6, train_N=(14, 15, 16), finetune_frac=0.05, seed=1,
                                          pre_epochs=3, ft_epochs=8, batch=2048, holdout=100_000)
    assert rep.holdout_spearman > 0.4, rep
    for N, k in ((16, 5), (17, 6), (18, 6)):
        res = learned.count_learned(N, k, model, config=dict(timing=1))
        assert res.total == pub[str(N)]["total"]
        assert res.stats["schedule_ms"] > 0
    # What the network buys: the share of all DFS work that sits in the first
    # fifth of the queue, in the order the model chose versus expander order.
    c, l, r, y, nodes, _ = learned.solver_labels(18, 6)
    pred = model.predict(18, c, l, r)
    keys = np.clip(np.floor(pred * 8 + 0.5), 0, 65535)
    order = np.lexsort((np.arange(c.size), -keys))
    head = c.size // 5
    share_plain = nodes[:head].sum() / nodes.sum()
    share_learned = nodes[order[:head]].sum() / nodes.sum()
    share_oracle = np.sort(nodes)[::-1][:head].sum() / nodes.sum()
    print(f"work in the first fifth of the queue: plain {share_plain:.3f}, learned {share_learned:.3f}, "
          f"oracle {share_oracle:.3f}")
    assert share_learned > share_plain + 0.15
    model.close()


def test_device_schedule_then_count_on_one_stream(gpu, golden):
    # Schedule and count enqueued back to back on the default stream, no
    # synchronisation in between (the bench's learned step).
    import torch
    from n_queens_b200 import learned
    N, k = 17, 6
    m = learned.CostModel(seed=9)
    c, l, r = oracle.expand(N, k)
    dev = torch.device("cuda:0")
    tc, tl, tr = (torch.from_numpy(a.view(np.int32)).to(dev) for a in (c, l, r))
    order = torch.empty(c.size, dtype=torch.int32, device=dev)
    out = torch.zeros(2, dtype=torch.int64, device=dev)
    cfg = gpu.Config()
    cfg.stack_levels = N - 1 - k
    cfg.order_kind = gpu.NQ_ORDER_GIVEN
    cfg.order = order.data_ptr()
    for _ in range(2):
        assert learned.lib.nq_schedule_device(m._m, N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), c.size,
                                              order.data_ptr(), None, None) == 0
        gpu.count_tasks_device(N, tc, tl, tr, out, config=cfg)
        assert 2 * int(out[0]) == golden("published.json")[str(N)]["total"] and int(out[1]) == 0
    m.close()


def test_learned_order_shortens_the_tail(gpu, golden):
    # What decides whether the learned order helps is the measured makespan and tail idle
    # time (per-CTA start/end stamps, nq_config.timing): over interleaved
    # repeats at N=19, k=6 the model's longest-first queue must leave less of
    # the grid idle at the end than the expander order, and the count kernel
    # must not get slower (1 % allowance for run-to-run noise).
    from n_queens_b200 import learned
    N, k = 19, 6
    want = golden("published.json")[str(N)]["total"]
    model, rep = learned.build_cost_model(N, k=k, seed=1)
    tail = {"learned": [], "plain": []}
    kern = {"learned": [], "plain": []}
    for _ in range(3):
        for kind in ("learned", "plain"):
            if kind == "learned":
                r = learned.count_learned(N, k, model, config=dict(timing=1))
            else:
                r = gpu.count(N, k, config=dict(timing=1))
            assert r.total == want
            tail[kind].append(r.stats["tail_idle_frac"])
            kern[kind].append(r.stats["kernel_ms"])
    model.close()
    mean = lambda xs: sum(xs) / len(xs)
    print(f"N={N}: tail idle learned {mean(tail['learned']):.4%} plain {mean(tail['plain']):.4%}; "
          f"kernel learned {mean(kern['learned']):.2f} ms plain {mean(kern['plain']):.2f} ms")
    assert mean(tail["learned"]) < mean(tail["plain"])
    assert mean(kern["learned"]) <= 1.01 * mean(kern["plain"])


def test_learned_count_reuses_the_labelled_tasks(gpu, golden):
    # The build counts its fine-tuning sample and hold-out exactly (to label
    # them); the reuse entry leaves those tasks out of the queue and adds
    # their sum, and the total is still the published one.
    from n_queens_b200 import learned
    N, k = 18, 6
    want = golden("published.json")[str(N)]["total"]
    model, rep = learned.build_cost_model(N, k=k, train_N=(14, 15, 16), seed=3, pre_epochs=2, ft_epochs=4,
                                          holdout=50_000)
    c, l, r = gpu.expand(N, k)
    idx = rep.counted_idx
    assert idx.size == round(0.05 * c.size) + 50_000
    assert np.all(np.diff(idx) > 0)
    assert rep.counted_sum == int(oracle.count_tasks(N, c[idx], l[idx], r[idx]).sum())
    res = learned.count_learned(N, k, model, reuse=rep)
    assert res.total == want
    # an empty reuse list is the plain learned count
    rep0 = learned.BuildReport(target_N=N, k=k)
    assert learned.count_learned(N, k, model, reuse=rep0).total == want
    # indices must be ascending and distinct, and the report must be this board's
    bad = learned.BuildReport(target_N=N, k=k, counted_idx=idx[::-1].copy(), counted_sum=rep.counted_sum)
    with pytest.raises(gpu.NQError):
        learned.count_learned(N, k, model, reuse=bad)
    with pytest.raises(ValueError):
        learned.count_learned(17, 6, model, reuse=rep)
    model.close()


def test_schedule_last_and_queue_len_skip_exactly_the_listed_tasks(gpu):
    # nq_schedule_device_last puts the listed tasks at the end of the order;
    # nq_config.queue_len = n - n_last then counts every other task once.
    import torch
    from n_queens_b200 import learned
    N, k = 15, 5
    c, l, r = oracle.expand(N, k)
    per = oracle.count_tasks(N, c, l, r)
    rng = np.random.default_rng(7)
    last = np.sort(rng.choice(c.size, c.size // 7, replace=False)).astype(np.uint32)
    dev = torch.device("cuda:0")
    tc, tl, tr = (torch.from_numpy(a.view(np.int32)).to(dev) for a in (c, l, r))
    tlast = torch.from_numpy(last.view(np.int32)).to(dev)
    order = torch.empty(c.size, dtype=torch.int32, device=dev)
    m = learned.CostModel(seed=4)
    m.set_params(_params(5))
    s = torch.cuda.current_stream().cuda_stream
    assert learned.lib.nq_schedule_device_last(m._m, N, tc.data_ptr(), tl.data_ptr(), tr.data_ptr(), c.size,
                                               tlast.data_ptr(), last.size, order.data_ptr(), None, s) == 0
    torch.cuda.synchronize()
    o = order.cpu().numpy().view(np.uint32)
    assert np.array_equal(np.sort(o), np.arange(c.size))
    assert np.array_equal(o[c.size - last.size:], last)           # listed tasks last, in index order
    out = torch.zeros(2, dtype=torch.int64, device=dev)
    cfg = gpu.Config()
    cfg.stack_levels = N - 1 - k
    cfg.order_kind = gpu.NQ_ORDER_GIVEN
    cfg.order = order.data_ptr()
    cfg.queue_len = c.size - last.size
    gpu.count_tasks_device(N, tc, tl, tr, out, config=cfg)
    keep = np.ones(c.size, bool)
    keep[last] = False
    assert int(out[0]) == int(per[keep].sum()) and int(out[1]) == 0
    cfg.queue_len = c.size + 1                                     # beyond the task list: refused
    with pytest.raises(gpu.NQError):
        gpu.count_tasks_device(N, tc, tl, tr, out, config=cfg)
    m.close()

