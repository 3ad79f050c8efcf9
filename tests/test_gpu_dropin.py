"""The keyword arguments that the reference's own imaging driver produced
(recorded by ``tests/golden/make_dropin.py``) through the CUDA library.

Each fixture holds the exact ``fortlib.fftim2d.imaging`` call that
``smili/imaging/lbfgs.py:492-564`` made for one set of images and tables
(0-d dummies, int32 index arrays in the (3, Ncp) / (4, Nca) layout, and the
other f2py-ready types included).  The CUDA path, at the reference's default
NUFFT tolerance 1e-6 in FP64, is held to the CPU oracle on the same kwargs:
the iteration count, and the L-BFGS-B objective per iteration, which starts
equal to rounding (1e-10) and then drifts as the iteration amplifies
rounding differences (measured: below 1e-6 for 10 iterations in every case,
up to 8e-4 by iteration 20 with closure phases and amplitudes).  Bounds: the
first 10 iterations within 1e-6, every iteration and the final cost within
2e-3, the image within 1e-2 of its peak.  This project's whole driver
(``smili_b200.imaging.lbfgs.imaging``) on the same inputs returns the image
that the reference's driver returned over the oracle, to 1e-2 of its peak.
"""
import glob
import os

import numpy as np
import pytest

import reference_dropin as R

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "dropin_*.npz")))
NAMES = [os.path.basename(f)[7:-4] for f in FIXTURES]


@pytest.mark.parametrize("path", FIXTURES, ids=NAMES)
def test_recorded_call_through_cuda(oracle, path):
    from smili_b200 import _lib
    from smili_b200.fortlib import fftim2d
    _, _, kw = R.load_case(path)
    niter = int(kw["niter"])
    info = {}
    out = fftim2d.imaging(info=info, **kw)
    assert len(out) == 16 and out[0].shape == (int(kw["npix"]),)
    iout, tref, iref = oracle.imaging(kw, eps=1e-6)
    assert info["niter"] == iref["niter"]
    assert abs(out[15] - tref["cost"]) <= 2e-3 * abs(tref["cost"])
    assert np.abs(out[0] - iout).max() <= 1e-2 * np.abs(iout).max()
    b = _lib.Batch([kw], niter=niter, nonneg=bool(kw["nonneg"]), m=int(kw["m"]),
                   options=_lib.make_options(64, 1e-6))
    b.run()
    tr = b.trace(0, niter + 2)
    b.close()
    k = min(niter, len(iref["trace"]))
    np.testing.assert_allclose(tr[:10], iref["trace"][:10], rtol=1e-6)
    np.testing.assert_allclose(tr[:k], iref["trace"][:k], rtol=2e-3)


@pytest.mark.parametrize("path", FIXTURES, ids=NAMES)
def test_driver_returns_reference_image(path):
    from smili_b200.imaging.lbfgs import imaging
    init, opts, _ = R.load_case(path)
    out = imaging(init, **opts)
    want = np.load(path)["out__data"]
    assert np.abs(out.data - want).max() <= 1e-2 * np.abs(want).max()
