"""``fortlib.fftlib``: the NUFFT entry points used outside the solver.

``nufft_fwd_real`` (src/fortlib/fftlib.f90:86-100) evaluates model
visibilities of an image (used by the UVFITS simulator,
smili/uvdata/uvfits/uvfits.py:2616); ``nufft_adj_real1d``
(fftlib.f90:118-133) forms the real part of the adjoint transform (dirty
maps, smili/uvdata/uvtable/vistable.py:2691).  Same arguments and sign
conventions; ``u, v`` are already multiplied by 2*pi*dx, 2*pi*dy.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib


def nufft_fwd_real(u, v, i2d, precision=64, nufft_eps=0.0, device=0):
    """Type-2 NUFFT of the (nx, ny) Fortran-order image ``i2d``; returns (Vreal, Vimag)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    img = np.asarray(i2d, dtype=np.float64)
    nx, ny = img.shape
    flat = np.ascontiguousarray(img.reshape(-1, order="F"))
    vr, vi = np.zeros(u.size), np.zeros(u.size)
    opt = _lib.make_options(precision, nufft_eps, 0, device)
    _lib.check(_lib.lib().smili_nufft_fwd_real(u.size, _lib.dptr(u), _lib.dptr(v), nx, ny,
                                               _lib.dptr(flat), C.byref(opt), _lib.dptr(vr),
                                               _lib.dptr(vi)))
    return vr, vi


def nufft_adj_real1d(u, v, vreal, vimag, nx, ny, precision=64, nufft_eps=0.0, device=0):
    """Real part of the type-1 NUFFT of Vreal + i Vimag, as an Nx*Ny vector."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    vr = np.ascontiguousarray(vreal, dtype=np.float64)
    vi = np.ascontiguousarray(vimag, dtype=np.float64)
    out = np.zeros(int(nx) * int(ny))
    opt = _lib.make_options(precision, nufft_eps, 0, device)
    _lib.check(_lib.lib().smili_nufft_adj_real1d(u.size, _lib.dptr(u), _lib.dptr(v), _lib.dptr(vr),
                                                 _lib.dptr(vi), int(nx), int(ny), C.byref(opt),
                                                 _lib.dptr(out)))
    return out
