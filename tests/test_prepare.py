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


def _gauss(n, sx, sy, th):
    yy, xx = np.mgrid[:n, :n] + 1.0
    c, s = np.cos(th), np.sin(th)
    X, Y = xx - 48.0, yy - 50.0
    a, b = c * X + s * Y, -s * X + c * Y
    img = np.exp(-0.5 * ((a / sx) ** 2 + (b / sy) ** 2))
    return img.reshape(-1), xx.reshape(-1).astype(np.int32), yy.reshape(-1).astype(np.int32)


def test_image_moments_and_sm_character():
    """fortlib.image.totalflux / xy_cen / sigma / check_sm_character as
    imdata.py:1020-1075 calls them: on an elliptical Gaussian whose major
    axis lies at theta from the x axis, the second moments give back its
    variances, and the angle is the reference's -(90 deg - theta) wrapped
    into [-90, 90] deg (both branches of image.f90:1066-1073)."""
    from smili_b200.fortlib import image
    sx, sy = 9.0, 4.0
    for th in (np.deg2rad(30.0), np.deg2rad(120.0)):
        I1d, xidx, yidx = _gauss(96, sx, sy, th)
        Isum = image.totalflux(I1d, I1d.size)
        assert Isum == image.totalflux(I1d)
        xc, yc = image.xy_cen(I1d, xidx, yidx)
        assert abs(xc - 48.0) < 1e-6 and abs(yc - 50.0) < 1e-6
        Sg = image.sigma(I1d, xidx, yidx, Isum, xc, yc)
        mj, mn, phi = image.check_sm_character(Sg)
        assert abs(mj - sx ** 2) < 1e-3 * sx ** 2 and abs(mn - sy ** 2) < 1e-3 * sy ** 2
        want = (-(np.pi / 2 - th) + np.pi / 2) % np.pi - np.pi / 2
        assert abs(phi - want) < 1e-3, (np.rad2deg(th), np.rad2deg(phi))


def test_calc_uvw_known_answers():
    """At hour angle 0 and declination 0: u = y, v = z, w = x; at the pole
    (delta = 90 deg) v = -x, w = z; the baseline length is preserved."""
    from smili_b200.fortlib import coord
    rng = np.random.default_rng(3)
    d = rng.normal(size=(3, 50)) * 1e6
    u, v, w = coord.calc_uvw(np.zeros(50), np.zeros(50), np.zeros(50), *d)
    assert np.allclose([u, v, w], [d[1], d[2], d[0]])
    u, v, w = coord.calc_uvw(np.zeros(50), np.zeros(50), np.full(50, np.pi / 2), *d)
    assert np.allclose([u, v, w], [d[1], -d[0], d[2]], atol=1e-6)
    gst, dec = rng.uniform(0, 24, 50), rng.uniform(-1, 1, 50)
    u, v, w = coord.calc_uvw(gst, np.zeros(50), dec, *d)
    assert np.allclose(u ** 2 + v ** 2 + w ** 2, (d ** 2).sum(0))
