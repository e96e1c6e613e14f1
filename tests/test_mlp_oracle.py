"""The learned-schedule MLP oracle against central finite differences (CPU), and its BF16
rounding against hand-computed cases."""
import numpy as np

from oracle import mlp_oracle as mo


def _params(seed=3):
    rng = np.random.default_rng(seed)
    p = np.zeros(mo.N_PARAMS, np.float32)
    off = 0
    for name, shape in mo.SHAPES:
        n = int(np.prod(shape))
        fan_in = shape[1] if len(shape) == 2 else 1
        p[off:off + n] = rng.uniform(-1, 1, n) * (np.sqrt(6 / fan_in) if len(shape) == 2 else 0.1)
        off += n
    return p


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 1.0 + 2 ** -9], np.float32)
    r = mo.bf16_round(x)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties to the even mantissa (1.0)
    assert r.tolist() == [1.0, 1.0, 1.0 + 2 ** -6, -2.5, 0.0, 1.0]


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    p = _params().astype(np.float64)
    x = rng.standard_normal((16, mo.F))
    y = np.stack([rng.uniform(0, 8, 16), rng.integers(0, 2, 16)], axis=1).astype(np.float64)
    _, g = mo.loss_and_grad(p, x, y, rounding=False)
    # a sample of coordinates from every tensor
    idx = []
    off = 0
    for _, shape in mo.SHAPES:
        n = int(np.prod(shape))
        idx += list(off + rng.choice(n, size=min(n, 12), replace=False))
        off += n
    eps = 1e-5
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        lp, _ = mo.loss_and_grad(pp, x, y, rounding=False)
        lm, _ = mo.loss_and_grad(pm, x, y, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])
