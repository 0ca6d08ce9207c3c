"""The CPU reference of the closure's MLP: its backward pass against
central finite differences of its own loss (smooth form, no BF16 rounding)."""
import numpy as np
import pytest

from oracle import mlp_ref as R


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.3, (n, R.IN)).astype(np.float32)
    x[:, 6] = rng.uniform(0, 1, n)
    x[:, 7] = 0
    m = rng.normal(0, 1, n)
    d = rng.uniform(0.1, 2, n)
    target = m + rng.normal(0, 0.1, n)
    w = rng.uniform(0.5, 2, n)
    return x, m, d, target, w


def _loss(p, x, m, d, target, w, gelu):
    y, _, _, _ = R.forward(p, x, rounding=False, gelu=gelu)
    return R.loss_and_dy(x, y, m, d, target, w)[0]


@pytest.mark.parametrize("gelu", [False, True])
def test_backward_matches_finite_differences(gelu):
    x, m, d, target, w = _data(24, 1)
    p = R.init_params(3).astype(np.float64)
    p += np.random.default_rng(4).normal(0, 0.05, p.shape)
    y, c, z1, z2 = R.forward(p, x, rounding=False, gelu=gelu)
    loss, dy = R.loss_and_dy(x, y, m, d, target, w)
    g = R.backward(p, x, z1, z2, dy, rounding=False, gelu=gelu)
    rng = np.random.default_rng(5)
    idx = list(rng.choice(R.P_TOTAL, 40, replace=False)) + [R.P_B3, R.P_B3 + 5, R.P_B1 + 3, R.P_W1 + 2 * R.H + 7]
    for q in idx:
        if R.P_W3 <= q < R.P_B3 and (q - R.P_W3) % R.OUT >= R.NC:
            continue                     # unused output columns
        if R.P_W1 + 7 * R.H <= q < R.P_B1:
            continue                     # padding input row
        if R.P_B3 + R.NC <= q < R.P_TOTAL:
            continue
        h = 1e-6 * max(1.0, abs(p[q]))
        pp, pm = p.copy(), p.copy()
        pp[q] += h
        pm[q] -= h
        fd = (_loss(pp, x, m, d, target, w, gelu) - _loss(pm, x, m, d, target, w, gelu)) / (2 * h)
        assert abs(fd - g[q]) <= 1e-5 * max(1.0, abs(fd)), (q, fd, g[q])


def test_coefficients_sum_to_one_and_bf16_rounding():
    x, *_ = _data(16, 2)
    p = R.init_params(0)
    y, c, _, _ = R.forward(p, x)
    assert np.allclose(c.sum(1), 1.0, atol=1e-12)
    a = np.array([1.0, 1.00390625, 1.005859375, -3.0e-5], np.float32)
    assert list(R.bf16(a)) == [1.0, 1.0, 1.0078125, np.float32(-3.0040740966796875e-05)]
