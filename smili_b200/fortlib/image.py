"""``fortlib.image``: regularizer weight initialisers and image statistics.

Host-side set-up that the imaging driver runs once per solve
(smili/imaging/lbfgs.py:264-401).  Each function restates the Fortran routine
it replaces (src/fortlib/image.f90) with the same argument names, defaults
and return values as the f2py wrappers, in numpy.
"""
from __future__ import annotations

import math

import numpy as np

ZEROEPS = 1e-10  # image.f90:7


def _smabs(x):
    return np.sqrt(np.asarray(x, dtype=np.float64) ** 2 + ZEROEPS)


def _to2d(I1d, xidx, yidx, nx, ny):
    I2d = np.zeros((int(ny), int(nx)))
    I2d[np.asarray(yidx, dtype=np.int64) - 1, np.asarray(xidx, dtype=np.int64) - 1] = I1d
    return I2d


def _tv_e(I1d, xidx, yidx, nx, ny):
    """Per-pixel isotropic TV term (image.f90:477-508)."""
    I2d = _to2d(I1d, xidx, yidx, nx, ny)
    dx = np.zeros_like(I2d)
    dy = np.zeros_like(I2d)
    dx[:, :-1] = I2d[:, 1:] - I2d[:, :-1]
    dy[:-1, :] = I2d[1:, :] - I2d[:-1, :]
    e = np.sqrt(dx * dx + dy * dy)
    return e[np.asarray(yidx) - 1, np.asarray(xidx) - 1]


def _tsv_e(I1d, xidx, yidx, nx, ny):
    """Per-pixel TSV term (image.f90:678-711)."""
    I2d = _to2d(I1d, xidx, yidx, nx, ny)
    dx = np.zeros_like(I2d)
    dy = np.zeros_like(I2d)
    dx[:, :-1] = I2d[:, 1:] - I2d[:, :-1]
    dy[:-1, :] = I2d[1:, :] - I2d[:-1, :]
    e = dx * dx + dy * dy
    return e[np.asarray(yidx) - 1, np.asarray(xidx) - 1]


def init_l1reg(l1_prior):
    """Weighted-L1 weights normalised so sum(w*|prior|) = 1 (image.f90:207-223)."""
    p = np.asarray(l1_prior, dtype=np.float64)
    w = 1.0 / _smabs(p)
    return w / np.sum(_smabs(p) * w)


def init_tvreg(xidx, yidx, nx, ny, tv_isflat, tv_prior):
    """TV weights: flat 1/(eps+sum F)/N, else reweighted (image.f90:409-446)."""
    p = np.asarray(tv_prior, dtype=np.float64)
    N = p.size
    nx, ny = int(nx), int(ny)
    xidx = np.asarray(xidx).astype(np.int64)
    yidx = np.asarray(yidx).astype(np.int64)
    if tv_isflat:
        return np.full(N, 1.0 / (ZEROEPS + np.sum(p)) / N)
    w = 1.0 / _tv_e(p, xidx, yidx, nx, ny)
    return w / np.sum(_tv_e(p, xidx, yidx, nx, ny) * w)


def init_tsvreg(xidx, yidx, nx, ny, tsv_isflat, tsv_prior):
    """TSV weights: flat 1/(eps+(sum F)^2/N)/N, else reweighted (image.f90:620-661)."""
    p = np.asarray(tsv_prior, dtype=np.float64)
    N = p.size
    nx, ny = int(nx), int(ny)
    xidx = np.asarray(xidx).astype(np.int64)
    yidx = np.asarray(yidx).astype(np.int64)
    if tsv_isflat:
        return np.full(N, 1.0 / (ZEROEPS + np.sum(p) ** 2 / N) / N)
    w = 1.0 / (p ** 2 + ZEROEPS)
    return w / np.sum(_tsv_e(p, xidx, yidx, nx, ny) * w)


def init_klreg(kl_l_in, kl_prior):
    """KL-MEM: weights = smabs(prior); lambda normalised by KL(p, p) (image.f90:278-322)."""
    w = _smabs(kl_prior)
    a = _smabs(w)
    kl = np.sum(a * np.log(a / w) + w / math.e)
    return float(kl_l_in) / kl, w


def init_gsreg(gs_prior):
    """GS-MEM weights = smabs(prior) (image.f90:352-364)."""
    return _smabs(gs_prior)


def init_tfdreg(tfd_l_in, tfd_tgtfd, tfd_tgter):
    """Total-flux lambda normalised by (F * fractional error)^2 (image.f90:760-772)."""
    return float(tfd_l_in) / (float(tfd_tgtfd) * float(tfd_tgter)) ** 2


def totalflux(I1d, N1d=None):
    """Sum of |I| (image.f90:1125-1136).  ``N1d`` is the f2py length argument
    (optional there too; imdata.py:1029 passes it)."""
    I1d = np.asarray(I1d, dtype=np.float64)
    if N1d is not None:
        I1d = I1d[:int(N1d)]
    return float(np.sum(np.abs(I1d)))


def xy_cen(I1d, x, y, N1d=None):
    """Intensity-weighted centroid normalised by sum |I| (image.f90:1100-1123)."""
    I1d = np.asarray(I1d, dtype=np.float64)
    n = I1d.size if N1d is None else int(N1d)
    I1d, x, y = I1d[:n], np.asarray(x)[:n], np.asarray(y)[:n]
    tot = np.sum(np.abs(I1d))
    return float(np.sum(x * I1d) / tot), float(np.sum(y * I1d) / tot)


def sigma(I1d, xidx, yidx, Isum, xcen, ycen, N1d=None):
    """Second moments of the image about (xcen, ycen), divided by Isum:
    [sum I (x - xc)^2, sum I (y - yc)^2, sum I (x - xc)(y - yc)] / Isum
    (``Sigma``, image.f90:1039-1053; imdata.py:1031 calls it as sigma)."""
    I1d = np.asarray(I1d, dtype=np.float64)
    n = I1d.size if N1d is None else int(N1d)
    I1d = I1d[:n]
    dx = np.asarray(xidx, dtype=np.float64)[:n] - xcen
    dy = np.asarray(yidx, dtype=np.float64)[:n] - ycen
    return np.array([np.sum(I1d * dx ** 2 / Isum), np.sum(I1d * dy ** 2 / Isum), np.sum(I1d * dx * dy / Isum)])


# check_sm_character's pi is the single-precision literal 3.1415926535
# widened to double (image.f90:1062), kept for parity
_PI_SM = float(np.float32(3.1415926535))


def check_sm_character(Sg):
    """Major / minor second moments and the position angle of the ellipse
    with second-moment matrix [[Sg1, Sg3], [Sg3, Sg2]] (image.f90:1055-1078):
    returns (maj, min, phi), phi measured from the RA axis."""
    s1, s2, s3 = (float(v) for v in np.asarray(Sg, dtype=np.float64)[:3])
    root = np.sqrt(4.0 * s3 ** 2 + (s1 - s2) ** 2) / 2.0
    mj = (s1 + s2) / 2.0 + root
    mn = (s1 + s2) / 2.0 - root
    with np.errstate(invalid="ignore", divide="ignore"):
        phi = float(np.arcsin(2.0 * s3 / (mj - mn)) / 2.0)
    if s1 / s2 > 1.0:
        if s3 > 0.0:
            phi = 0.5 * _PI_SM - phi
        if s3 < 0.0:
            phi = -0.5 * _PI_SM - phi
    return mj, mn, -phi
