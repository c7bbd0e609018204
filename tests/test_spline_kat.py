"""Known-answer tests for the project B-spline (the oracle's stand-in for
einspline, which the reference calls but does not ship)."""
import numpy as np
import pytest


def _basis_eval(c, t):
    return (c[0] * (1 - t) ** 3 + c[1] * (3 * t ** 3 - 6 * t ** 2 + 4) + c[2] * (-3 * t ** 3 + 3 * t ** 2 + 3 * t + 1)
            + c[3] * t ** 3) / 6


@pytest.mark.parametrize("N", [3, 4, 7, 22])
def test_natural_interpolates_nodes_and_has_zero_curvature_at_ends(oracle, N):
    f = np.random.default_rng(N).normal(size=N)
    c = oracle.spline1d(f, 0)
    assert len(c) == N + 2
    vals = (c[:-2] + 4 * c[1:-1] + c[2:]) / 6
    np.testing.assert_allclose(vals, f, rtol=0, atol=1e-13)
    assert c[0] - 2 * c[1] + c[2] == pytest.approx(0, abs=1e-12)
    assert c[-3] - 2 * c[-2] + c[-1] == pytest.approx(0, abs=1e-12)


def test_natural_reproduces_linear(oracle):
    x = np.arange(20.0)
    c = oracle.spline1d(3 * x - 2, 0)
    for i in range(19):
        for t in (0.0, 0.3, 0.9):
            assert _basis_eval(c[i:i + 4], t) == pytest.approx(3 * (i + t) - 2, abs=1e-12)


@pytest.mark.parametrize("N", [3, 8, 33])
def test_periodic_interpolates_and_wraps(oracle, N):
    f = np.random.default_rng(N).normal(size=N)
    c = oracle.spline1d(f, 1)
    assert len(c) == N + 3
    core = c[1:N + 1]
    vals = (np.roll(core, 1) + 4 * core + np.roll(core, -1)) / 6
    np.testing.assert_allclose(vals, f, atol=1e-12)
    assert c[0] == c[N] and c[N + 1] == c[1] and c[N + 2] == c[2]


def test_periodic_fourth_order_convergence(oracle):
    errs = []
    for N in (16, 32, 64):
        h = 2 * np.pi / N
        x = (np.arange(N) + 0.5) * h
        s, _ = oracle.spline3d(np.sin(x)[:, None, None] * np.ones((N, 4, 4)), 1, (0.5 * h,) * 3, (1 / h,) * 3)
        xs = np.linspace(0.1, 6.2, 37)
        errs.append(max(abs(oracle.eval(s, a, 0.3, 0.7, 0)[0] - np.sin(a)) for a in xs))
    rate = np.log2(errs[0] / errs[1]), np.log2(errs[1] / errs[2])
    assert min(rate) > 3.7, (errs, rate)


def test_3d_gradient_and_hessian_of_trilinear_product(oracle):
    # the natural spline reproduces linear data exactly, hence products of linear functions per axis
    n = 10
    a = np.arange(n, dtype=float)
    data = (2 * a + 1)[:, None, None] * (a - 3)[None, :, None] * (0.5 * a + 2)[None, None, :]
    s, _ = oracle.spline3d(data, 0, (0.0,) * 3, (1.0,) * 3)
    for (y, x, z) in ((2.3, 4.1, 5.7), (0.0, 0.0, 0.0), (8.9, 1.2, 3.3)):
        v, g, lap, h = oracle.eval(s, y, x, z, 3)
        fy, fx, fz = 2 * y + 1, x - 3, 0.5 * z + 2
        assert v == pytest.approx(fy * fx * fz, abs=1e-10)
        np.testing.assert_allclose(g, [2 * fx * fz, fy * fz, 0.5 * fy * fx], atol=1e-10)
        np.testing.assert_allclose(h.reshape(3, 3), [[0, 2 * fz, 2 * 0.5 * fx], [2 * fz, 0, 0.5 * fy],
                                                     [2 * 0.5 * fx, 0.5 * fy, 0]], atol=1e-9)
