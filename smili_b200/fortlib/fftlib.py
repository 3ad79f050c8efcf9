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


def nufft_fwd_real(u, v, i2d, precision=64, nufft_eps=0.0, device=0, transform=0):
    """Type-2 NUFFT of the (nx, ny) Fortran-order image ``i2d``; returns (Vreal, Vimag).
    ``transform``: 0 automatic, 1 FFT passes, 2 dense twiddle products (narrow bands)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    img = np.asarray(i2d, dtype=np.float64)
    nx, ny = img.shape
    flat = np.ascontiguousarray(img.reshape(-1, order="F"))
    vr, vi = np.zeros(u.size), np.zeros(u.size)
    opt = _lib.make_options(precision, nufft_eps, 0, device, transform=transform)
    _lib.check(_lib.lib().smili_nufft_fwd_real(u.size, _lib.dptr(u), _lib.dptr(v), nx, ny,
                                               _lib.dptr(flat), C.byref(opt), _lib.dptr(vr),
                                               _lib.dptr(vi)))
    return vr, vi


def nufft_adj_real1d(u, v, vreal, vimag, nx, ny, precision=64, nufft_eps=0.0, device=0, transform=0):
    """Real part of the type-1 NUFFT of Vreal + i Vimag, as an Nx*Ny vector."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    vr = np.ascontiguousarray(vreal, dtype=np.float64)
    vi = np.ascontiguousarray(vimag, dtype=np.float64)
    out = np.zeros(int(nx) * int(ny))
    opt = _lib.make_options(precision, nufft_eps, 0, device, transform=transform)
    _lib.check(_lib.lib().smili_nufft_adj_real1d(u.size, _lib.dptr(u), _lib.dptr(v), _lib.dptr(vr),
                                                 _lib.dptr(vi), int(nx), int(ny), C.byref(opt),
                                                 _lib.dptr(out)))
    return out


def _model(iin, xidx, yidx, nxref, nyref, nx, ny, u, v, term, precision=64, nufft_eps=0.0, device=0):
    """One data term's raw chi-square, gradient, models and residuals
    (smili_model_terms); ``term`` holds that term's kwargs."""
    kw = dict(iin=iin, xidx=xidx, yidx=yidx, nxref=nxref, nyref=nyref, nx=nx, ny=ny, u=u, v=v,
              npix=np.size(iin), l1_l=-1.0, tv_l=-1.0, tsv_l=-1.0, kl_l=-1.0, gs_l=-1.0, tfd_l=-1.0,
              tfd_tgtfd=1.0, cen_l=-1.0, cen_alpha=1.0, sm_l=-1.0, sm_maj=0.0, sm_min=0.0, sm_phi=0.0,
              l1_wgt=_ONE, tv_wgt=_ONE, tsv_wgt=_ONE, kl_wgt=_ONE, gs_wgt=_ONE, l1_nwgt=1, tv_nwgt=1,
              tsv_nwgt=1, kl_nwgt=1, gs_nwgt=1, isfcv=False, uvidxfcv=_IZ, vfcvr=_ONE, vfcvi=_ONE,
              varfcv=_ONE, wfcv=1.0, isamp=False, uvidxamp=_IZ, vamp=_ONE, varamp=_ONE, wamp=1.0,
              iscp=False, uvidxcp=np.zeros((3, 1), np.int32), cp=_ONE, varcp=_ONE, wcp=1.0, isca=False,
              uvidxca=np.zeros((4, 1), np.int32), ca=_ONE, varca=_ONE, wca=1.0, inormfactr=1.0)
    kw.update(term)
    prob = _lib.Problem(kw)
    opt = _lib.make_options(precision, nufft_eps, 0, device)
    n = {"isfcv": prob.c.nfcv, "isamp": prob.c.namp, "iscp": prob.c.ncp, "isca": prob.c.nca}
    nd = next(n[k] for k in n if term.get(k))
    x = np.ascontiguousarray(iin, dtype=np.float64)
    chisq = C.c_double(0.0)
    grad = np.zeros(prob.npix)
    mr, mi, rr, ri = (np.zeros(nd) for _ in range(4))
    _lib.check(_lib.lib().smili_model_terms(C.addressof(prob.c), _lib.dptr(x), C.byref(opt), C.byref(chisq),
                                            _lib.dptr(grad), _lib.dptr(mr), _lib.dptr(mi), _lib.dptr(rr),
                                            _lib.dptr(ri)))
    return chisq.value, grad, mr, mi, rr, ri


_ONE = np.ones(1)
_IZ = np.zeros(1, np.int32)


def model_fcv(iin, xidx, yidx, nxref, nyref, nx, ny, u, v, uvidxfcv, vfcvr, vfcvi, varfcv, **opt):
    """model_fcv (fftlib.f90:744-895): (chisq, gradchisq, modelr, modeli,
    residr, residi) with model and residual shifted back to the reference
    pixel (phashift_c2r)."""
    return _model(iin, xidx, yidx, nxref, nyref, nx, ny, u, v,
                  dict(isfcv=True, uvidxfcv=uvidxfcv, vfcvr=vfcvr, vfcvi=vfcvi, varfcv=varfcv), **opt)


def model_amp(iin, xidx, yidx, nxref, nyref, nx, ny, u, v, uvidxamp, vamp, varamp, **opt):
    """model_amp (fftlib.f90:898-996): (chisq, gradchisq, model, resid)."""
    c, g, m, _, r, _ = _model(iin, xidx, yidx, nxref, nyref, nx, ny, u, v,
                              dict(isamp=True, uvidxamp=uvidxamp, vamp=vamp, varamp=varamp), **opt)
    return c, g, m, r


def model_cp(iin, xidx, yidx, nxref, nyref, nx, ny, u, v, uvidxcp, cp, varcp, **opt):
    """model_cp (fftlib.f90:1126-1254): (chisq, gradchisq, model, resid),
    model and residual wrapped into (-pi, pi]."""
    c, g, m, _, r, _ = _model(iin, xidx, yidx, nxref, nyref, nx, ny, u, v,
                              dict(iscp=True, uvidxcp=uvidxcp, cp=cp, varcp=varcp), **opt)
    return c, g, m, r


def model_ca(iin, xidx, yidx, nxref, nyref, nx, ny, u, v, uvidxca, ca, varca, **opt):
    """model_ca (fftlib.f90:999-1123): (chisq, gradchisq, model, resid)."""
    c, g, m, _, r, _ = _model(iin, xidx, yidx, nxref, nyref, nx, ny, u, v,
                              dict(isca=True, uvidxca=uvidxca, ca=ca, varca=varca), **opt)
    return c, g, m, r
