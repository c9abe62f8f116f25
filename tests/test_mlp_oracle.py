"""The CPU MLP oracle pinned on its own: the float64 analytic gradient against
central finite differences, BF16 rounding against known values, and the AdamW
step against its closed form."""
import numpy as np

from oracle import mlp_oracle as MO


def _net(dims, seed=0, scale=0.5):
    r = np.random.default_rng(seed)
    n = sum(dims[l + 1] * dims[l] + dims[l + 1] for l in range(len(dims) - 1))
    return r.standard_normal(n) * scale


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2.0**-9, 1.0 + 3 * 2.0**-9, -2.5, 3.0e-3, 65504.0], dtype=np.float64)
    got = MO.bf16_round(x)
    # 1 + 2^-9 is a tie between 1 and 1 + 2^-7: ties go to the even mantissa (1.0)
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == 1.0 + 2.0**-7
    assert got[3] == -2.5
    assert abs(got[4] - 3.0e-3) / 3.0e-3 < 2.0**-8
    assert got[5] == 65536.0


def test_analytic_gradient_matches_finite_differences():
    dims = [6, 16, 16, 8]
    p = _net(dims)
    r = np.random.default_rng(1)
    X = r.standard_normal((5, 6))
    T = r.standard_normal((5, 8))
    loss, g = MO.MLP(dims, p, bf16=False).loss_grad(X, T)
    h = 1e-6
    idx = r.choice(p.size, 40, replace=False)
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp = MO.MLP(dims, pp, bf16=False).loss_grad(X, T)[0]
        lm = MO.MLP(dims, pm, bf16=False).loss_grad(X, T)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9


def test_adamw_first_step_closed_form():
    dims = [2, 16]
    p = _net(dims)
    g = np.linspace(-1, 1, p.size)
    m0 = np.zeros_like(p)
    p1, m1, v1 = MO.adamw(p, g, m0, m0, 1, 1e-3, 0.9, 0.999, 1e-8, 0.0, dims)
    # first bias-corrected step is lr * sign(g) (up to eps)
    assert np.allclose(p - p1, 1e-3 * g / (np.abs(g) + 1e-8), rtol=1e-6, atol=1e-12)
