"""GPU checks of the warm-start network's CUDA kernels against the FP64 oracle
(oracle/cnn64.py), through the library's C ABI.

Tolerances: forward output 1e-5 relative (FP32 accumulation, bf16 weights on
both sides); loss 1e-5 relative; parameter gradients 1e-4 relative L2 per
parameter block (FP32 accumulation over up to B*H*W*Cin*9 products)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net_and_case(seed=0, B=2, H=16):
    import torch
    from gpair_b200 import warmstart as W
    params = W.init_params(seed)
    # non-zero biases exercise the bias paths
    rng = np.random.default_rng(seed + 100)
    for name, off, n in W.param_layout():
        if name.endswith(".b"):
            params[off:off + n] = rng.normal(0, 0.05, n)
    net = W.WarmStartNet(params, 0)
    x = rng.standard_normal((B, W.N_FEATURES, H, H)).astype(np.float32)
    t = rng.uniform(0.0, 1.0, (B, H * H)).astype(np.float32)
    t /= t.sum(axis=1, keepdims=True)
    return net, params, x, t, torch


@pytest.mark.parametrize("H,mode", [(16, 1), (24, 1), (16, 0)])
def test_cnn_forward_and_gradients_match_fp64(H, mode):
    from oracle import cnn64 as N
    net, params, x, t, torch = _net_and_case(H=H)
    net.loss_mode = mode
    xt = torch.from_numpy(x).cuda()
    tt = torch.from_numpy(t).cuda()
    out = net.forward(xt, keep=True).reshape(x.shape[0], -1)
    loss, g = net.loss_and_grad(out, tt)
    net.g.zero_()
    net.backward(g)
    torch.cuda.synchronize()
    P = N.unpack(params)
    o64, a = N.forward(P, x.astype(np.float64))
    G = N.backward(P, a, t.astype(np.float64), mode)
    o = out.cpu().numpy()
    assert np.abs(o - o64).max() <= 1e-5 * np.abs(o64).max()
    l64 = N.loss(o64, t.astype(np.float64), mode)
    assert abs(float(loss.mean()) - l64) <= 1e-5 * l64
    gflat = net.g.cpu().numpy().astype(np.float64)
    g64 = N.flat_grad(G)
    from gpair_b200.warmstart import param_layout
    for name, off, n in param_layout():
        ref = g64[off:off + n]
        err = np.linalg.norm(gflat[off:off + n] - ref) / max(np.linalg.norm(ref), 1e-30)
        assert err <= 1e-4, (name, err)


def test_cnn_training_reduces_loss():
    """A few Adam steps on a fixed batch drive the loss down (optimiser + bf16 refresh)."""
    net, params, x, t, torch = _net_and_case(seed=4, B=4, H=16)
    xt = torch.from_numpy(x).cuda()
    tt = torch.from_numpy(t).cuda()
    first = float(net.train_step(xt, tt, 1e-3).mean())
    for _ in range(30):
        last = float(net.train_step(xt, tt, 1e-3).mean())
    assert last < 0.5 * first


def test_trained_network_gains_over_the_flat_start():
    """What the trained network gains over plain CG's flat start, on held-out
    problems (seeds never used in training): its start image has a lower
    objective J than the flat prior, and CG started from it needs fewer
    batched-line-search iterations to reach the objective that flat-start CG
    reaches after 300 iterations (summed over the problems)."""
    import gpair_b200 as g
    from gpair_b200.train_warmstart import SEED_HELD_OUT
    from gpair_b200.warmstart import WarmStartNet, training_case, warm_start
    net = WarmStartNet.load()
    better, it_flat, it_warm = 0, 0, 0
    n = 8
    with g.Reconstructor(0) as rec:
        rec.set_precision(g.PREC_SPLIT16)
        for k in range(n):
            p = training_case(SEED_HELD_OUT + 100 + k, 64).problem
            rec.set_problem(p)
            rec.set_image(p.start_image())
            chi2, S = rec.criterion()
            J_flat = chi2 - p.alpha * S
            img = warm_start(net, rec, p)
            rec.set_image(img)
            chi2, S = rec.criterion()
            better += (chi2 - p.alpha * S) < J_flat
            rec.set_image(p.start_image())
            ref = rec.cg(300, method=2, trace=True, line_search=g.LS_BATCH)
            target = float(ref["trace_J"][-1]) * (1 + 1e-4)
            rec.set_image(p.start_image())
            it_flat += rec.cg(300, method=2, line_search=g.LS_BATCH, target_J=target)["iterations"]
            rec.set_image(img)
            it_warm += rec.cg(300, method=2, line_search=g.LS_BATCH, target_J=target)["iterations"]
    print(f"warm start better than flat on {better}/{n}; iterations to target: flat {it_flat}, warm {it_warm}")
    # measured on a B200: better on 5 of 8, 1,304 vs 2,114 iterations (deterministic kernels)
    assert better > n // 2
    assert it_warm < 0.85 * it_flat
