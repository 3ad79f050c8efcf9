"""Dynamic imaging (fftim3d) on the GPU against the CPU oracle.

The movie objective, its 20 cost terms and its gradient in FP64 with a
tight NUFFT tolerance (1e-12) match the oracle's exact transform to 1e-9
relative (terms) and 1e-8 (gradient, max-norm); this covers Rt / Ri, the
light-curve variant, a frame without data and the one-frame movie.  Short
solves agree with the oracle's solve; FP32 stays within 1e-4 (objective).
"""
import numpy as np
import pytest

from test_oracle3d import movie_kw

pytestmark = pytest.mark.gpu

TERMS = ["chisq", "chisqfcv", "chisqcp", "reg", "l1_cost", "tsv_cost", "tfd_cost", "lc_cost", "rt_cost",
         "ri_cost", "cost"]


def _x(kw, seed=0):
    return np.asarray(kw["iin"], dtype=np.float64) * np.random.default_rng(seed).uniform(0.5, 1.5, np.size(kw["iin"]))


def _check(oracle, kw, x, rel_t=1e-9, rel_g=1e-8, precision=64, eps=1e-12):
    from smili_b200.fortlib import fftim3d
    t_g, g_g = fftim3d.calc_cost(x, precision=precision, nufft_eps=eps, **kw)
    t_o, g_o = oracle.calc_cost3d(kw, x, eps=0.0)
    for k in TERMS:
        assert abs(t_g[k] - t_o[k]) <= rel_t * max(abs(t_o["cost"]), 1e-300), (k, t_g[k], t_o[k])
    assert np.max(np.abs(g_g - g_o)) <= rel_g * np.max(np.abs(g_o)), np.max(np.abs(g_g - g_o))
    return t_g


@pytest.mark.parametrize("extra", [{"ri_lambda": 0.5, "tfd_lambda": 1.0},
                                   {"lc_lambda": 1.0, "lc_array": [0.5, 0.6, 0.7], "lc_normalize": "both",
                                    "ri_lambda": 0.3}],
                         ids=["rt_ri_tfd", "light_curve"])
def test_calc_cost3d_matches_oracle(oracle, extra):
    kw, _ = movie_kw(extra=extra)
    t = _check(oracle, kw, _x(kw))
    assert t["rt_cost"] > 0 and t["ri_cost"] > 0


def test_calc_cost3d_frame_without_data(oracle):
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs3d import prepare_imaging3d
    m = synth.dynamic_problem(seed=4, nframes=4, nx=32, nst=6, vis_per_frame=90, niter=10)
    vt = m.vistable[m.vistable.frmidx != 1].reset_index(drop=True)
    bt = m.bstable[m.bstable.frmidx != 1].reset_index(drop=True)
    kw, _ = prepare_imaging3d(m.frames, vistable=vt, bstable=bt, niter=10, l1_lambda=1.0, tsv_lambda=1.0,
                              rt_lambda=1.0, tfd_lambda=1.0)
    assert int(np.asarray(kw["nuvs"])[1]) == 0
    _check(oracle, kw, _x(kw, 2))


def test_calc_cost3d_single_frame(oracle):
    kw, _ = movie_kw(nframes=1, extra={"tfd_lambda": 1.0})
    _check(oracle, kw, _x(kw, 3))


def test_calc_cost3d_fp32_bound(oracle):
    kw, _ = movie_kw(extra={"ri_lambda": 0.5})
    _check(oracle, kw, _x(kw, 4), rel_t=1e-4, rel_g=5e-3, precision=32, eps=1e-6)


def test_imaging3d_matches_oracle(oracle):
    """A short solve: same iteration count and final cost (first iterations
    of L-BFGS-B on closure phases agree closely before chaos sets in)."""
    from smili_b200.fortlib import fftim3d
    kw, _ = movie_kw(extra={"ri_lambda": 0.5})
    kw["niter"] = 8
    info = {}
    out = fftim3d.imaging(precision=64, nufft_eps=1e-12, info=info, **kw)
    iout_o, t_o, info_o = oracle.imaging3d(kw, eps=0.0)
    assert info["niter"] == info_o["niter"] == 9
    assert abs(out[20] - t_o["cost"]) <= 1e-6 * abs(t_o["cost"])
    assert np.max(np.abs(out[0] - iout_o)) <= 1e-4 * np.max(np.abs(iout_o))
    assert np.all(out[0] >= 0)
