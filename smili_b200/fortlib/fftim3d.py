"""``fortlib.fftim3d``: the dynamic-imaging (movie) driver on the GPU.

``imaging`` has the keyword signature of the f2py wrapper of
src/fortlib/fftim3d.f90:11-467 as called at smili/imaging/lbfgs3d.py:732-784
and returns the same 21-tuple ``(Iout, chisq, chisqfcv, chisqamp, chisqcp,
chisqca, reg, l1_cost, sm_cost, tv_cost, tsv_cost, kl_cost, gs_cost,
tfd_cost, lc_cost, cen_cost, rt_cost, ri_cost, rs_cost, rf_cost, cost)``.
Work runs in libsmili_b200.so; ``precision`` (64 | 32) and ``nufft_eps``
(default 1e-6) select the arithmetic.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .. import _lib


def imaging(precision=64, nufft_eps=0.0, ctas_per_problem=0, device=0, info=None, **kw):
    mv = _lib.Movie(kw)
    opt = _lib.make_options(precision, nufft_eps, ctas_per_problem, device)
    iout = np.zeros(mv.n)
    terms = np.zeros(20)
    si = _lib.SolveInfo()
    _lib.check(_lib.lib().smili_fftim3d_imaging(
        C.addressof(mv.c), int(kw["niter"]), int(bool(kw["nonneg"])), int(kw.get("nprint", 0)),
        int(kw.get("m", 5)), float(kw.get("factr", 1e1)), float(kw.get("pgtol", 0.0)),
        C.byref(opt), _lib.dptr(iout), _lib.dptr(terms), C.byref(si)))
    if info is not None:
        info.update({"task": si.task, "niter": si.niter, "nfg": si.nfg, "error": si.error})
    return (iout,) + tuple(float(t) for t in terms)


def calc_cost(x, precision=64, nufft_eps=0.0, ctas_per_problem=0, device=0, **kw):
    """calc_cost of fftim3d (fftim3d.f90:473-614) at movie vector x:
    (terms dict, grad)."""
    mv = _lib.Movie(kw)
    opt = _lib.make_options(precision, nufft_eps, ctas_per_problem, device)
    x = np.ascontiguousarray(x, dtype=np.float64)
    terms = np.zeros(20)
    grad = np.zeros(mv.n)
    _lib.check(_lib.lib().smili_calc_cost3d(C.addressof(mv.c), _lib.dptr(x), C.byref(opt), _lib.dptr(terms),
                                            _lib.dptr(grad)))
    return dict(zip(_lib.TERM_NAMES_3D, terms)), grad
