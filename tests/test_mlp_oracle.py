"""The NumPy restatement of the p*-seed network: its backward pass against
central finite differences (CPU only)."""
import numpy as np

from oracle import mlp_ref


def test_mlp_ref_gradient_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.3, mlp_ref.NPARAM)
    X = rng.normal(0, 1, (40, 6))
    Y = rng.normal(0, 0.5, 40)
    _, g = mlp_ref.loss_and_grad(p, X, Y, bf=False)
    for k in list(rng.choice(mlp_ref.NPARAM, 60, replace=False)) + [mlp_ref.NPARAM - 1]:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        lp, _ = mlp_ref.loss_and_grad(pp, X, Y, bf=False)
        lm, _ = mlp_ref.loss_and_grad(pm, X, Y, bf=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 1e-3], np.float32)
    r = mlp_ref.bf16(x)
    # bf16 keeps 8 significant bits: 1 + 2^-8 is a tie -> even (1.0); 1 + 3*2^-9 -> 1 + 2^-7
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125
    assert abs(r[3] - (-3.140625)) < 1e-12
    assert abs(r[4] - 1e-3) / 1e-3 < 2 ** -8
