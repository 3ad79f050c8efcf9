"""Host preparation of the imaging kwargs (no GPU)."""
import numpy as np

from conftest import make_kw


def test_window_mask_as_array(crescent32):
    """A plain boolean (ny, nx) array selects the pixels to solve for, as an
    image region does (lbfgs.py:226-249); ndarrays also carry a ``data``
    attribute, which must not be taken for an image's pixel cube."""
    yy, xx = np.mgrid[:32, :32]
    win = (xx - 16) ** 2 + (yy - 16) ** 2 < 13 ** 2
    kw = make_kw(crescent32, imregion=win)
    assert kw["npix"] == int(win.sum()) == np.size(kw["iin"])
    assert np.all(win[np.asarray(kw["yidx"]) - 1, np.asarray(kw["xidx"]) - 1])
    full = make_kw(crescent32)
    img = np.zeros((32, 32))
    img[np.asarray(full["yidx"]) - 1, np.asarray(full["xidx"]) - 1] = full["iin"] / full["inormfactr"]
    np.testing.assert_allclose(kw["iin"] / kw["inormfactr"], img[win])
