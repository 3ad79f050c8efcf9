"""The CPU oracle of dynamic imaging (fftim3d) on small movies.

The reference has no tests for this path either, so the oracle is checked
by: central finite differences of its gradient (exact DFT, no NUFFT
error); the one-frame movie against the 2D calc_cost; and the reference's
own Rt quirk (no Rt gradient on the last frame).
"""
import numpy as np
import pytest

from conftest import make_kw  # noqa: F401  (shared fixtures module)


def movie_kw(nframes=3, nx=32, extra=None, seed=1):
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs3d import prepare_imaging3d
    m = synth.dynamic_problem(seed=seed, nframes=nframes, nx=nx, nst=6, vis_per_frame=90, niter=20)
    args = dict(vistable=m.vistable, bstable=m.bstable, niter=20, **m.reg)
    args.update(extra or {})
    kw, meta = prepare_imaging3d(m.frames, **args)
    return kw, m


def _fd_check(oracle, kw, npick=12, rtol=2e-5, seed=0, last_frame=True):
    """Central differences at random pixels; ``last_frame`` False skips the
    last frame (its Rt gradient is left out by the reference)."""
    rng = np.random.default_rng(seed)
    x = np.asarray(kw["iin"], dtype=np.float64) * rng.uniform(0.5, 1.5, np.size(kw["iin"]))
    t, g = oracle.calc_cost3d(kw, x, eps=0.0)
    # pixels well above the |I| kink of smabs
    limit = x.size if last_frame else x.size - int(kw["npix"])
    cand = np.where(x[:limit] > 1e-3 * x.max())[0]
    for i in rng.choice(cand, npick, replace=False):
        h = 1e-6 * max(abs(x[i]), 1e-3)
        xp, xm = x.copy(), x.copy()
        xp[i] += h
        xm[i] -= h
        fd = (oracle.calc_cost3d(kw, xp, eps=0.0)[0]["cost"] - oracle.calc_cost3d(kw, xm, eps=0.0)[0]["cost"]) / (2 * h)
        # relative tolerance plus a floor for the difference quotient's roundoff
        assert abs(g[i] - fd) <= rtol * abs(fd) + 1e-6 * np.max(np.abs(g)), (i, g[i], fd)
    return t


def test_oracle3d_gradient_matches_finite_differences(oracle):
    kw, _ = movie_kw(extra={"ri_lambda": 0.5, "tfd_lambda": 1.0})
    t = _fd_check(oracle, kw, last_frame=False)
    assert t["rt_cost"] > 0 and t["ri_cost"] > 0 and t["tfd_cost"] > 0
    assert t["rs_cost"] == 0 and t["rf_cost"] == 0 and t["cen_cost"] == 0
    # without Rt every frame, the last included, is the exact derivative
    off = dict(kw)
    off["rt_l"] = -1.0
    _fd_check(oracle, off, seed=5)


def test_oracle3d_light_curve_gradient(oracle):
    kw, _ = movie_kw(extra={"lc_lambda": 1.0, "lc_array": [0.5, 0.6, 0.7], "lc_normalize": "both",
                            "ri_lambda": 0.3})
    t = _fd_check(oracle, kw, seed=1, last_frame=False)
    assert t["lc_cost"] > 0 and t["tfd_cost"] == 0


def test_oracle3d_single_frame_is_fftim2d(oracle):
    """One frame, no dynamic terms: the movie objective is the 2D one."""
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    from smili_b200.imaging.lbfgs3d import prepare_imaging3d
    o = synth.small_crescent(seed=2, nx=32, niter=5)
    kw2, _ = prepare_imaging(o.image, vistable=o.vistable, bstable=o.bstable, niter=5, l1_lambda=1.0,
                             tsv_lambda=1.0, tv_lambda=0.5)
    kw3, _ = prepare_imaging3d([o.image], vistable=o.vistable, bstable=o.bstable, niter=5, l1_lambda=1.0,
                               tsv_lambda=1.0, tv_lambda=0.5)
    x = np.asarray(kw2["iin"])
    t2, g2 = oracle.calc_cost(kw2, x, eps=0.0)
    t3, g3 = oracle.calc_cost3d(kw3, x, eps=0.0)
    for k in ("chisq", "chisqfcv", "chisqcp", "reg", "l1_cost", "tv_cost", "tsv_cost", "cost"):
        assert abs(t3[k] - t2[k]) <= 1e-12 * max(1.0, abs(t2[k])), k
    np.testing.assert_allclose(g3, g2, rtol=1e-12, atol=1e-12 * np.max(np.abs(g2)))


def test_oracle3d_rt_quirk_last_frame(oracle):
    """Rt adds no gradient to the last frame (image3d.f90:380-383 guards the
    gradient with iz < Nz), while its cost does depend on that frame."""
    kw, _ = movie_kw(nframes=3)
    off = dict(kw)
    off["rt_l"] = -1.0
    x = np.asarray(kw["iin"], dtype=np.float64) * np.random.default_rng(3).uniform(0.5, 1.5, np.size(kw["iin"]))
    _, g_on = oracle.calc_cost3d(kw, x, eps=0.0)
    _, g_off = oracle.calc_cost3d(off, x, eps=0.0)
    N = int(kw["npix"])
    d = g_on - g_off
    assert np.max(np.abs(d[2 * N:])) == 0.0
    assert np.max(np.abs(d[:N])) > 0 and np.max(np.abs(d[N:2 * N])) > 0


def test_oracle3d_imaging_runs(oracle):
    kw, _ = movie_kw(nframes=2)
    kw["niter"] = 5
    iout, terms, info = oracle.imaging3d(kw, eps=1e-6)
    assert info["niter"] == 6 and np.isfinite(terms["cost"])
    assert terms["cost"] < oracle.calc_cost3d(kw, kw["iin"], eps=1e-6)[0]["cost"]
    assert np.all(iout >= 0)
