"""The learned selector's GPU kernels against a float64 numpy restatement (forward, every gradient,
Adam), and a short training run that must fit a known function."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net(nin=23, hidden=128, seed=0):
    from ttc_b200.cost_model import MLP
    return MLP(nin, hidden, seed)


def test_gemm_all_transposes_match_numpy():
    import torch
    from ttc_b200.cost_model import gemm
    rng = np.random.default_rng(0)
    for (M, N, K) in [(1, 1, 1), (7, 5, 3), (130, 67, 129), (1000, 128, 83), (64, 1, 128)]:
        for ta in (False, True):
            for tb in (False, True):
                A = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
                B = rng.standard_normal((N, K) if tb else (K, N)).astype(np.float32)
                bias = rng.standard_normal(N).astype(np.float32)
                want = (A.T if ta else A).astype(np.float64) @ (B.T if tb else B).astype(np.float64) + bias
                got = gemm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), ta, tb,
                           torch.from_numpy(bias).cuda()).cpu().numpy()
                assert np.allclose(got, want, rtol=1e-4, atol=1e-4 * np.sqrt(K)), (M, N, K, ta, tb)
                got = gemm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda(), ta, tb,
                           torch.from_numpy(bias).cuda(), relu=True).cpu().numpy()
                assert np.allclose(got, np.maximum(want, 0), rtol=1e-4, atol=1e-4 * np.sqrt(K))


def test_gradients_match_cpu_oracle():
    """Loss and all six gradients of the GPU network against the float64 numpy restatement
    (relative error of each gradient <= 1e-4 in norm); fp32 tolerance written here."""
    import torch
    from ttc_b200.cost_model import numpy_forward_backward
    net = _net(23, 128, 1)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((517, 23)).astype(np.float32)
    y = rng.standard_normal(517).astype(np.float32)
    out, cache = net.forward(torch.from_numpy(X).cuda())
    loss, d = net.loss_grad(out, torch.from_numpy(y).cuda().reshape(-1, 1))
    grads = net.backward(d, cache)
    ref_loss, ref_grads = numpy_forward_backward([p.cpu().numpy() for p in net.params], X, y)
    assert abs(float(loss.item()) - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    for g, r in zip(grads, ref_grads):
        g = g.cpu().numpy().reshape(r.shape).astype(np.float64)
        rel = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-12)
        assert rel <= 1e-4, rel


def test_gradients_match_torch_autograd_fp32():
    import torch
    net = _net(11, 128, 3)
    rng = np.random.default_rng(4)
    X = torch.from_numpy(rng.standard_normal((300, 11)).astype(np.float32)).cuda()
    y = torch.from_numpy(rng.standard_normal((300, 1)).astype(np.float32)).cuda()
    out, cache = net.forward(X)
    _, d = net.loss_grad(out, y)
    grads = net.backward(d, cache)
    ps = [p.clone().requires_grad_(True) for p in net.params]
    h = torch.relu(X @ ps[0] + ps[1])
    h = torch.relu(h @ ps[2] + ps[3])
    o = h @ ps[4] + ps[5]
    torch.mean((o - y) ** 2).backward()
    for g, p in zip(grads, ps):
        assert torch.allclose(g.reshape(p.grad.shape), p.grad, rtol=1e-3, atol=1e-5)


def test_adam_step_matches_formula():
    import torch
    from ttc_b200 import _native
    from ttc_b200.cost_model import _lib
    rng = np.random.default_rng(5)
    p = rng.standard_normal(1000).astype(np.float32)
    g = rng.standard_normal(1000).astype(np.float32)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    tp, tg, tm, tv = (torch.from_numpy(x.copy()).cuda() for x in (p, g, m, v))
    for t in (1, 2, 3):
        _native.check(_lib().ttcb_mlp_adam(tp.data_ptr(), tg.data_ptr(), tm.data_ptr(), tv.data_ptr(), 1000, 0.01,
                                           0.9, 0.999, 1e-8, t, torch.cuda.current_stream().cuda_stream))
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        p = p - 0.01 * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    assert np.allclose(tp.cpu().numpy(), p, rtol=1e-5, atol=1e-6)


def test_adam_step_with_weight_decay_matches_formula():
    import torch
    from ttc_b200 import _native
    from ttc_b200.cost_model import _lib
    rng = np.random.default_rng(7)
    p = rng.standard_normal(1000).astype(np.float32)
    g = rng.standard_normal(1000).astype(np.float32)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    tp, tg, tm, tv = (torch.from_numpy(x.copy()).cuda() for x in (p, g, m, v))
    wd = 0.01
    for t in (1, 2, 3):
        _native.check(_lib().ttcb_mlp_adam_l2(tp.data_ptr(), tg.data_ptr(), tm.data_ptr(), tv.data_ptr(), 1000,
                                              0.01, 0.9, 0.999, 1e-8, wd, t,
                                              torch.cuda.current_stream().cuda_stream))
        ge = g + wd * p
        m = 0.9 * m + 0.1 * ge
        v = 0.999 * v + 0.001 * ge * ge
        p = p - 0.01 * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    assert np.allclose(tp.cpu().numpy(), p, rtol=1e-5, atol=1e-6)


def test_training_fits_a_smooth_function():
    from ttc_b200.cost_model import train
    rng = np.random.default_rng(6)
    X = rng.uniform(-1, 1, (6000, 8)).astype(np.float32)
    y = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * X[:, 3] ** 2).astype(np.float32)
    m = train(X, y, epochs=60, lr=3e-3, batch=512, log=None)
    assert m.rmse < 0.15 * float(np.std(y)), (m.rmse, float(np.std(y)))


def test_trained_selector_beats_the_planner_default():
    """What the trained network gains over the method without it, on fresh timings of held-out
    problems (the first 40 of the held-out seed; no stored timing is reused): every candidate is timed
    (TTC's exhaustive method), then the search's winner, the network's top-1, the selector's choice
    (under the model's policy: the default, the top-1, or the fastest of its top k and the default,
    timed) and the
    planner default alone are re-timed alternately. The selector keeps a larger share of the winner's
    GB/s than the planner default, and tunes in a small fraction of the search's time.

    On separate B200 boxes the margin over the default measured 0.001 to 0.029 and the tuning-time
    ratio 12 to 26; the bounds below leave that spread to timing noise."""
    import ttc_b200.workloads as wl
    from ttc_b200 import cost_model
    r = cost_model.fresh_head_to_head(wl.learning_cases(cost_model.HELDOUT_SEED, 40))
    assert r["problems"] == 40
    assert r["selector_over_search"] >= r["default_over_search"], r
    assert r["selector_over_search"] >= 0.93, r
    assert r["tuning_time_ratio_selector"] >= 8, r
