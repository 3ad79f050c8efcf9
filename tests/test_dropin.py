"""The drop-in contract: the reference's own imaging driver over this library.

``smili/imaging/lbfgs.py:imaging`` (the reference's driver, unchanged) turns
images and tables into one call of ``fortlib.fftim2d.imaging`` (lbfgs.py:
492-564) and rebuilds the image from its first output (565-576).  These tests
hold this project's host preparation (``prepare_imaging``) and image
reassembly (``finish_imaging``) to that driver:

- against fixtures recorded from the reference's driver
  (``tests/golden/make_dropin.py``): identical keyword names, dtype kinds and
  bit-identical values, and the same output image for the same solve;
- live, when $SMILI_REFERENCE_ROOT names a reference checkout: the reference's
  ``imaging`` runs here with ``fortlib`` redirected to this project's mirror
  (``image.init_*`` for its regularizer weights) and a recording
  ``fftim2d.imaging`` that returns the CPU oracle's solve.

The GPU side (``tests/test_gpu_dropin.py``) runs the recorded kwargs through
the CUDA library.
"""
import glob
import os

import numpy as np
import pytest

import reference_dropin as R

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "dropin_*.npz")))
NAMES = [os.path.basename(f)[7:-4] for f in FIXTURES]


def test_fixtures_cover_every_case():
    assert sorted(NAMES) == sorted(n for n, _, _ in R.cases())


@pytest.mark.parametrize("path", FIXTURES, ids=NAMES)
def test_prepare_matches_reference_driver(oracle, path):
    from smili_b200.imaging.lbfgs import finish_imaging, prepare_imaging
    init, opts, kw_ref = R.load_case(path)
    kw, meta = prepare_imaging(init, **opts)
    R.compare_kwargs(kw, kw_ref)
    # the same solve reassembled into the same image
    out = finish_imaging(init, R.oracle_solve(1e-6)(kw), meta)
    np.testing.assert_array_equal(out.data, np.load(path)["out__data"])


@pytest.mark.skipif(R.reference_root() is None, reason=f"${R.ENV} does not name a reference checkout")
@pytest.mark.parametrize("case", [c[0] for c in R.cases()])
def test_reference_driver_live(oracle, case):
    from smili_b200.imaging.lbfgs import finish_imaging, prepare_imaging
    (_, init, opts), = [c for c in R.cases() if c[0] == case]
    (_, init2, opts2), = [c for c in R.cases() if c[0] == case]
    fl = R.RecordingFortlib(R.oracle_solve(1e-6))
    with R.reference_lbfgs(R.reference_root(), fl) as ref:
        out_ref = ref.imaging(init, **opts)
    assert len(fl.calls) == 1
    kw, meta = prepare_imaging(init2, **opts2)
    R.compare_kwargs(kw, fl.calls[0])
    out = finish_imaging(init2, R.oracle_solve(1e-6)(kw), meta)
    np.testing.assert_array_equal(out.data, out_ref.data)
    # the reference normalises shared prior images in place; so does the mirror
    for k in R.IMAGES:
        if k in opts:
            np.testing.assert_array_equal(opts[k].data, opts2[k].data)


@pytest.mark.skipif(R.reference_root() is None, reason=f"${R.ENV} does not name a reference checkout")
def test_reference_driver_input_errors():
    """The reference's input checks (lbfgs.py:185-201) return -1 the same way."""
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    o = synth.precision_path(seed=7, nx=32, nst=6, hours=2.0, scan_s=900.0)
    fl = R.RecordingFortlib(R.oracle_solve(1e-6))
    bad = [dict(), dict(bstable=o.bstable), dict(bstable=o.bstable, totalflux=1.0)]
    with R.reference_lbfgs(R.reference_root(), fl) as ref:
        for opts in bad:
            assert ref.imaging(o.image.copy(), **opts) == -1
            assert prepare_imaging(o.image.copy(), **opts) == -1
    assert not fl.calls
