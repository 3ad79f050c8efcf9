"""``fortlib.fftim2d``: the static-imaging driver on the GPU.

``imaging`` has the keyword signature of the f2py wrapper of
src/fortlib/fftim2d.f90:11-382 as called at smili/imaging/lbfgs.py:492-564
and returns the same 16-tuple ``(Iout, chisq, chisqfcv, chisqamp, chisqcp,
chisqca, reg, l1_cost, tv_cost, tsv_cost, kl_cost, gs_cost, tfd_cost,
cen_cost, sm_cost, cost)``.  Work runs in libsmili_b200.so; extra keywords
``precision`` (64 | 32) and ``nufft_eps`` (default 1e-6, the reference's
ffteps) select the arithmetic.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib


def imaging(precision=64, nufft_eps=0.0, ctas_per_problem=0, device=0, info=None, **kw):
    prob = _lib.Problem(kw)
    opt = _lib.make_options(precision, nufft_eps, ctas_per_problem, device)
    iout = np.zeros(prob.npix)
    terms = np.zeros(15)
    si = _lib.SolveInfo()
    _lib.check(_lib.lib().smili_fftim2d_imaging(
        C.addressof(prob.c), int(kw["niter"]), int(bool(kw["nonneg"])), int(kw.get("nprint", 0)),
        int(kw.get("m", 5)), float(kw.get("factr", 1e1)), float(kw.get("pgtol", 0.0)),
        C.byref(opt), _lib.dptr(iout), _lib.dptr(terms), C.byref(si)))
    if info is not None:
        info.update({"task": si.task, "niter": si.niter, "nfg": si.nfg, "error": si.error})
    return (iout,) + tuple(float(t) for t in terms)


def calc_cost(x, precision=64, nufft_eps=0.0, device=0, spread_bin=0, transform=0, **kw):
    """calc_cost (fftim2d.f90:387-607) at image vector x: (terms dict, grad).
    ``spread_bin`` (8 | 16) and ``transform`` (0 automatic, 1 radix passes,
    2 dense band products) select the launch's spreading tile and band path."""
    prob = _lib.Problem(kw)
    opt = _lib.make_options(precision, nufft_eps, 0, device, spread_bin=spread_bin, transform=transform)
    x = np.ascontiguousarray(x, dtype=np.float64)
    terms = np.zeros(15)
    grad = np.zeros(prob.npix)
    _lib.check(_lib.lib().smili_calc_cost(C.addressof(prob.c), _lib.dptr(x), C.byref(opt),
                                          _lib.dptr(terms), _lib.dptr(grad)))
    return dict(zip(_lib.TERM_NAMES, terms)), grad


def calc_cost_noalloc(x, precision=64, nufft_eps=0.0, device=0, spread_bin=0, transform=0, **kw):
    """calc_cost through the allocation-free entry point: the same result as
    ``calc_cost`` (same options) for problems whose device arena fits the
    library's static scratch (others raise SmiliError with code -1).  Calls
    on one device must not overlap, and none may be made while a stream is
    capturing (the call is synchronous)."""
    prob = _lib.Problem(kw)
    opt = _lib.make_options(precision, nufft_eps, 0, device, spread_bin=spread_bin, transform=transform)
    x = np.ascontiguousarray(x, dtype=np.float64)
    terms = np.zeros(15)
    grad = np.zeros(prob.npix)
    _lib.check(_lib.lib().smili_calc_cost_noalloc(C.addressof(prob.c), _lib.dptr(x), C.byref(opt),
                                                  _lib.dptr(terms), _lib.dptr(grad)))
    return dict(zip(_lib.TERM_NAMES, terms)), grad
