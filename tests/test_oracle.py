"""Pinning the CPU oracle: NUFFT vs the exact DFT, adjoint identity,
finite-difference gradients, and L-BFGS-B against scipy's L-BFGS-B (the same
v3.0 algorithm as src/lbfgsb/lbfgsb.f)."""
import numpy as np
import pytest
from scipy.optimize import minimize as sp_minimize

from conftest import make_kw


def test_nufft_type2_vs_dft(oracle):
    rng = np.random.default_rng(0)
    img = rng.standard_normal((24, 32))
    u, v = rng.uniform(-3, 3, 300), rng.uniform(-3, 3, 300)
    ex = oracle.nufft2d2(u, v, img, 0)
    k1 = np.arange(32) - 16
    k2 = np.arange(24) - 12
    direct = (img * np.exp(1j * (u[5] * k1[None, :] + v[5] * k2[:, None]))).sum()
    assert abs(direct - ex[5]) < 1e-12 * np.abs(img).sum()
    for eps in [1e-6, 1e-9, 1e-12]:
        nu = oracle.nufft2d2(u, v, img, eps)
        assert np.abs(nu - ex).max() / np.abs(ex).max() < 10 * eps


def test_nufft_type1_vs_dft(oracle):
    rng = np.random.default_rng(1)
    u, v = rng.uniform(-3, 3, 200), rng.uniform(-3, 3, 200)
    c = rng.standard_normal(200) + 1j * rng.standard_normal(200)
    ex = oracle.nufft2d1(u, v, c, 20, 16, 0)
    for eps in [1e-6, 1e-12]:
        nu = oracle.nufft2d1(u, v, c, 20, 16, eps)
        assert np.abs(nu - ex).max() / np.abs(ex).max() < 10 * eps


def test_nufft_adjoint_identity(oracle):
    rng = np.random.default_rng(2)
    img = rng.standard_normal((16, 16))
    u, v = rng.uniform(-3, 3, 100), rng.uniform(-3, 3, 100)
    c = rng.standard_normal(100) + 1j * rng.standard_normal(100)
    lhs = np.vdot(c, oracle.nufft2d2(u, v, img, 1e-12))
    rhs = np.vdot(np.conj(oracle.nufft2d1(u, v, np.conj(c), 16, 16, 1e-12)), img)
    assert abs(lhs - rhs) / abs(lhs) < 1e-12


def test_point_source_known_answer(oracle):
    # a unit point source at pixel (ix, iy) has V = exp(+i(u (ix-1-Nx/2) + v (iy-1-Ny/2)))
    img = np.zeros((16, 16))
    img[3, 11] = 1.0
    u, v = np.array([0.3, -1.2]), np.array([0.7, 2.1])
    V = oracle.nufft2d2(u, v, img, 1e-12)
    ref = np.exp(1j * (u * (11 - 8) + v * (3 - 8)))
    np.testing.assert_allclose(V, ref, atol=1e-11)


@pytest.mark.parametrize("terms", ["fcv_cp", "amp_cp_ca"])
def test_oracle_gradient_finite_difference(oracle, crescent32, closure40, terms):
    if terms == "fcv_cp":
        kw = make_kw(crescent32, l1_lambda=1.0, tsv_lambda=1.0, tv_lambda=0.5, kl_lambda=0.1,
                     gs_lambda=0.1, tfd_lambda=1.0, cen_lambda=0.1)
    else:
        kw = make_kw(closure40, l1_lambda=1.0, tv_lambda=1.0, kl_lambda=0.1)
    x = kw["iin"].copy()
    _, g = oracle.calc_cost(kw, x, eps=1e-12)
    rng = np.random.default_rng(3)
    cand = np.where(x > 1e-3 * x.max())[0]  # away from the |I| kink at zero
    for i in rng.choice(cand, 6, replace=False):
        h = 1e-6 * max(1.0, abs(x[i]))
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (oracle.calc_cost(kw, xp, 1e-12)[0]["cost"] - oracle.calc_cost(kw, xm, 1e-12)[0]["cost"]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-5 * max(abs(fd), 1e-6 * np.abs(g).max())


def _fun_factory(n, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    H = A.T @ A / n + 0.1 * np.eye(n)
    b = rng.standard_normal(n)

    def fun(x):
        f = 0.5 * x @ H @ x - b @ x + 0.05 * np.sum(x ** 4) + np.sum(np.sqrt(x * x + 1e-3))
        g = H @ x - b + 0.2 * x ** 3 + x / np.sqrt(x * x + 1e-3)
        return f, g
    return fun, np.abs(rng.standard_normal(n))


@pytest.mark.parametrize("bounded", [False, True])
def test_lbfgsb_matches_scipy_per_iteration(oracle, bounded):
    n = 200
    fun, x0 = _fun_factory(n, 1)
    nbd = np.ones(n, np.int32) if bounded else np.zeros(n, np.int32)
    _, trace, _ = oracle.minimize(fun, x0, m=5, nbd=nbd, maxiter=60)
    ref = []
    sp_minimize(fun, x0, jac=True, method="L-BFGS-B", bounds=[(0, None)] * n if bounded else None,
                options=dict(maxcor=5, ftol=10 * np.finfo(float).eps, gtol=0, maxiter=61, maxls=20),
                callback=lambda xk: ref.append(fun(xk)[0]))
    ref = np.array(ref)
    k = min(50, len(trace), len(ref))
    assert k >= 50
    np.testing.assert_allclose(trace[:k], ref[:k], rtol=1e-10)


def test_oracle_imaging_reduces_cost(oracle, crescent32):
    kw = make_kw(crescent32, niter=30)
    iout, terms, info = oracle.imaging(kw, eps=1e-6)
    tr = info["trace"]
    tr = tr[~np.isnan(tr)]
    assert info["niter"] == 31  # the driver stops once iter > niter (fftim2d.f90:324)
    assert terms["cost"] < 0.05 * oracle.calc_cost(kw, kw["iin"], 1e-6)[0]["cost"]
    assert np.all(np.diff(tr) <= 1e-12 * abs(tr[0]))
    assert iout.min() >= 0.0
