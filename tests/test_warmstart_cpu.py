"""CPU checks of the warm-start network's FP64 oracle (the checker of the CUDA
kernels) and of the host-side feature and training-case code."""
import numpy as np
import pytest

from gpair_b200 import warmstart as W
from oracle import cnn64 as N


def _case(seed=0, B=2, H=16):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((B, W.N_FEATURES, H, H))
    t = rng.uniform(0.0, 1.0, (B, H * H))
    t /= t.sum(axis=1, keepdims=True)
    return x, t


@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_gradient_matches_finite_differences(mode):
    params = W.init_params(3)
    P = N.unpack(params, round_bf16=False)
    x, t = _case()
    out, a = N.forward(P, x)
    G = N.backward(P, a, t, mode)
    rng = np.random.default_rng(1)
    checked = 0
    for name in ("e1a.w", "e2b.w", "e4b.w", "d3a.w", "d1b.b", "head.w", "head.b", "e3a.b"):
        for _ in range(3):
            idx = tuple(int(rng.integers(0, s)) for s in P[name].shape)
            eps = 1e-6
            old = P[name][idx]
            P[name][idx] = old + eps
            lp = N.loss(N.forward(P, x)[0], t, mode)
            P[name][idx] = old - eps
            lm = N.loss(N.forward(P, x)[0], t, mode)
            P[name][idx] = old
            num = (lp - lm) / (2 * eps)
            ana = G[name][idx]
            assert abs(num - ana) <= 1e-5 * max(1e-3, abs(ana)) + 1e-9, (name, idx, num, ana)
            checked += 1
    assert checked == 24


def test_oracle_output_is_positive_unit_flux():
    P = N.unpack(W.init_params(0))
    x, _ = _case(B=3, H=24)
    out, _ = N.forward(P, x)
    assert out.shape == (3, 24 * 24)
    assert np.all(out > 0)
    assert np.allclose(out.sum(axis=1), 1.0)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.14159], np.float32)
    r = N.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert r[3] == -2.5
    assert abs(r[4] - 3.14159) < 2 ** -7 * 4


def test_param_layout_is_contiguous():
    off = 0
    for name, o, n in W.param_layout():
        assert o == off
        off += n
    assert off == W.n_params()


def test_training_cases_are_seeded_and_sized():
    a = W.training_case(11, 64)
    b = W.training_case(11, 64)
    c = W.training_case(12, 64)
    assert a.problem.width == 64 and abs(a.problem.pixellation - 0.1) < 1e-7
    assert np.array_equal(a.problem.data, b.problem.data)
    assert not (a.problem.npow == c.problem.npow and np.array_equal(a.problem.data, c.problem.data))
    d = W.uv_density(a.problem)
    assert d.shape == (64, 64) and d.max() == 1.0
    # conjugate symmetry of the gridded coverage about the centre cell
    assert np.array_equal(d[1:, 1:], d[1:, 1:][::-1, ::-1])


def test_many_instance_workload_shapes():
    from gpair_b200.instances import WIDTHS, instance
    for k in range(6):
        p = instance(20_000_000 + k)
        assert p.width in WIDTHS
        assert 480 <= p.npow <= 8016 and 3 * p.nbis == 2 * p.npow
        # triangle vertices match V2 points except where the reference's relative-distance
        # test misses a short baseline; the unmatched vertices become extra uv points
        assert p.npow <= p.nuv <= 1.01 * p.npow
