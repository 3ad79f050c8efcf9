"""The allocation-free calc_cost entry point against smili_calc_cost.

smili_calc_cost_noalloc keeps its device scratch in one static array per
device, so consecutive calls reuse the same memory.  Two consecutive calls
at different images (and a third back at the first image) must each agree
with the allocating entry point, whatever ran on the device before.  The
file name sorts last so the check also runs after every other GPU test.
"""
import numpy as np
import pytest

from conftest import make_kw

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    from smili_b200 import synth
    obs = synth.precision_path(seed=5, nx=48, nst=8, hours=6.0, scan_s=600.0, niter=10)
    kw = make_kw(obs)
    x1 = np.asarray(kw["iin"], dtype=np.float64).copy()
    rng = np.random.default_rng(5)
    x2 = x1 * rng.uniform(0.5, 1.5, x1.size) + 1e-3 * x1.max()
    return kw, x1, x2


def _close(a, b, rtol):
    return np.max(np.abs(a - b)) <= rtol * max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("precision,eps,rtol", [(64, 1e-12, 1e-11), (32, 1e-6, 1e-5)])
def test_noalloc_matches_calc_cost(problem, precision, eps, rtol):
    from smili_b200.fortlib import fftim2d
    kw, x1, x2 = problem
    first = None
    for x in (x1, x2, x1):
        t_ref, g_ref = fftim2d.calc_cost(x, precision=precision, nufft_eps=eps, **kw)
        t_na, g_na = fftim2d.calc_cost_noalloc(x, precision=precision, nufft_eps=eps, **kw)
        for k, v in t_ref.items():
            assert abs(t_na[k] - v) <= rtol * max(abs(v), 1e-300), k
        assert _close(g_na, g_ref, rtol)
        if first is None:
            first = (t_na, g_na)
    # the third call (back at x1) repeats the first: no state survives a call
    assert abs(t_na["cost"] - first[0]["cost"]) <= rtol * abs(first[0]["cost"])
    assert _close(g_na, first[1], rtol)


@pytest.mark.parametrize("spread_bin,transform", [(16, 0), (8, 1), (8, 2)])
def test_noalloc_honours_launch_options(problem, spread_bin, transform):
    """The spreading tile and band path of the options reach the
    allocation-free call as they reach smili_calc_cost (FP64 at the
    reference's NUFFT tolerance: the same sums, rounding only)."""
    from smili_b200.fortlib import fftim2d
    kw, x1, x2 = problem
    for x in (x1, x2):
        t_ref, g_ref = fftim2d.calc_cost(x, precision=64, nufft_eps=1e-6, spread_bin=spread_bin,
                                         transform=transform, **kw)
        t_na, g_na = fftim2d.calc_cost_noalloc(x, precision=64, nufft_eps=1e-6, spread_bin=spread_bin,
                                               transform=transform, **kw)
        assert abs(t_na["cost"] - t_ref["cost"]) <= 1e-11 * abs(t_ref["cost"])
        assert _close(g_na, g_ref, 1e-11)


def test_noalloc_rejects_oversize():
    from smili_b200 import _lib, synth
    from smili_b200.fortlib import fftim2d
    # 256x256 with ~1e5 visibilities and closure terms: about 24 MB of FP64 arena
    obs = synth.precision_path(seed=2, nx=256, nst=10, hours=12.0, scan_s=20.0, niter=1)
    kw = make_kw(obs)
    with pytest.raises(_lib.SmiliError) as e:
        fftim2d.calc_cost_noalloc(kw["iin"], precision=64, **kw)
    assert e.value.code == -1
    assert "static scratch" in str(e.value)
