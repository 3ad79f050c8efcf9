"""Python driver of the CPU oracle (``liboracle.so``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` as the checker / CPU baseline.
The product (``smili_b200``) never imports it.

Arguments use the keyword names of ``fortlib.fftim2d.imaging`` as called at
smili/imaging/lbfgs.py:492-564, so a kwargs dict built for the product's
drop-in can be handed to the oracle unchanged.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "-s"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        _lib.orc_nufft2d2.argtypes = [C.c_int, dp, dp, C.c_int, C.c_int, dp, C.c_double, dp, dp]
        _lib.orc_nufft2d1.argtypes = [C.c_int, dp, dp, dp, dp, C.c_int, C.c_int, C.c_double, dp, dp]
        _lib.orc_calc_cost.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_double, C.c_double,
                                       C.c_double, dp, C.c_double, dp, dp]
        _lib.orc_imaging.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                     C.c_double, C.c_double, dp, dp, dp, ip, ip, ip]
        _lib.orc_calc_cost3d.argtypes = [C.c_void_p, dp, dp, C.c_double, C.c_double, C.c_double,
                                         C.c_double, dp, C.c_double, dp, dp]
        _lib.orc_imaging3d.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                       C.c_double, C.c_double, dp, dp, dp, ip, ip, ip]
        _lib.orc_lbfgsb_new.restype = C.c_void_p
        _lib.orc_lbfgsb_new.argtypes = [C.c_int, C.c_int, dp, dp, ip, C.c_double, C.c_double]
        _lib.orc_lbfgsb_step.argtypes = [C.c_void_p, dp, C.c_double, dp]
        _lib.orc_lbfgsb_info.argtypes = [C.c_void_p, ip, ip, ip, dp, dp]
        _lib.orc_lbfgsb_free.argtypes = [C.c_void_p]
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class _Args(C.Structure):
    _fields_ = [
        ("npix", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
        ("iin", C.c_void_p), ("xidx", C.c_void_p), ("yidx", C.c_void_p),
        ("nxref", C.c_double), ("nyref", C.c_double),
        ("nuv", C.c_int), ("u", C.c_void_p), ("v", C.c_void_p),
        ("l1_l", C.c_double), ("l1_wgt", C.c_void_p), ("l1_nwgt", C.c_int),
        ("tv_l", C.c_double), ("tv_wgt", C.c_void_p), ("tv_nwgt", C.c_int),
        ("tsv_l", C.c_double), ("tsv_wgt", C.c_void_p), ("tsv_nwgt", C.c_int),
        ("kl_l", C.c_double), ("kl_wgt", C.c_void_p), ("kl_nwgt", C.c_int),
        ("gs_l", C.c_double), ("gs_wgt", C.c_void_p), ("gs_nwgt", C.c_int),
        ("tfd_l", C.c_double), ("tfd_tgtfd", C.c_double),
        ("cen_l", C.c_double), ("cen_alpha", C.c_double),
        ("sm_l", C.c_double), ("sm_maj", C.c_double), ("sm_min", C.c_double), ("sm_phi", C.c_double),
        ("isfcv", C.c_int), ("nfcv", C.c_int), ("uvidxfcv", C.c_void_p), ("vfcvr", C.c_void_p),
        ("vfcvi", C.c_void_p), ("varfcv", C.c_void_p), ("wfcv", C.c_double),
        ("isamp", C.c_int), ("namp", C.c_int), ("uvidxamp", C.c_void_p), ("vamp", C.c_void_p),
        ("varamp", C.c_void_p), ("wamp", C.c_double),
        ("iscp", C.c_int), ("ncp", C.c_int), ("uvidxcp", C.c_void_p), ("cp", C.c_void_p),
        ("varcp", C.c_void_p), ("wcp", C.c_double),
        ("isca", C.c_int), ("nca", C.c_int), ("uvidxca", C.c_void_p), ("ca", C.c_void_p),
        ("varca", C.c_void_p), ("wca", C.c_double),
        ("inormfactr", C.c_double),
    ]


class Args:
    """Owns contiguous copies of the kwargs arrays and the C struct over them."""

    def __init__(self, kw: dict):
        f64 = lambda k: np.ascontiguousarray(np.asarray(kw[k], dtype=np.float64).reshape(-1))
        i32 = lambda k: np.ascontiguousarray(np.asarray(kw[k], dtype=np.int32).reshape(-1))
        self.keep = {}
        a = _Args()
        for k in ["iin", "u", "v", "l1_wgt", "tv_wgt", "tsv_wgt", "kl_wgt", "gs_wgt",
                  "vfcvr", "vfcvi", "varfcv", "vamp", "varamp", "cp", "varcp", "ca", "varca"]:
            self.keep[k] = f64(k)
        for k in ["xidx", "yidx", "uvidxfcv", "uvidxamp"]:
            self.keep[k] = i32(k)
        # (3,Ncp) / (4,Nca) Fortran order == the per-datum indices contiguous
        self.keep["uvidxcp"] = np.ascontiguousarray(np.asarray(kw["uvidxcp"], dtype=np.int32).T).reshape(-1)
        self.keep["uvidxca"] = np.ascontiguousarray(np.asarray(kw["uvidxca"], dtype=np.int32).T).reshape(-1)
        for k, arr in self.keep.items():
            setattr(a, k, arr.ctypes.data)
        a.npix = int(kw["npix"])
        a.nx, a.ny = int(kw["nx"]), int(kw["ny"])
        a.nxref, a.nyref = float(kw["nxref"]), float(kw["nyref"])
        a.nuv = self.keep["u"].size
        for k in ["l1_l", "tv_l", "tsv_l", "kl_l", "gs_l", "tfd_l", "tfd_tgtfd", "cen_l",
                  "cen_alpha", "sm_l", "sm_maj", "sm_min", "sm_phi", "wfcv", "wamp", "wcp", "wca",
                  "inormfactr"]:
            setattr(a, k, float(kw[k]))
        for k in ["l1", "tv", "tsv", "kl", "gs"]:
            setattr(a, k + "_nwgt", int(kw[k + "_nwgt"]))
        a.isfcv, a.isamp, a.iscp, a.isca = (int(bool(kw[k])) for k in ["isfcv", "isamp", "iscp", "isca"])
        a.nfcv = self.keep["uvidxfcv"].size
        a.namp = self.keep["uvidxamp"].size
        a.ncp = self.keep["uvidxcp"].size // 3
        a.nca = self.keep["uvidxca"].size // 4
        self.c = a
        self.kw = kw

    def ptr(self):
        return C.byref(self.c)

    def weights(self):
        """Normalised data weights (fftim2d.f90:178-213)."""
        a = self.c
        wt = 0.0
        if a.isfcv:
            wt += 2 * a.nfcv * a.wfcv
        if a.isamp:
            wt += a.namp * a.wamp
        if a.iscp:
            wt += a.ncp * a.wcp
        if a.isca:
            wt += a.nca * a.wca
        return (a.wfcv / wt if a.isfcv else 0.0, a.wamp / wt if a.isamp else 0.0,
                a.wcp / wt if a.iscp else 0.0, a.wca / wt if a.isca else 0.0)

    def shifted_fcv(self):
        """Data visibilities moved from the reference pixel to the image centre
        (phashift_r2c, fftlib.f90:223-244; fftim2d.f90:224-241)."""
        k = self.keep
        vr, vi = k["vfcvr"].copy(), k["vfcvi"].copy()
        if self.c.isfcv:
            idx = np.abs(k["uvidxfcv"]) - 1
            sg = np.sign(k["uvidxfcv"])
            ut, vt = k["u"][idx] * sg, k["v"][idx] * sg
            dix = self.c.nxref - self.c.nx / 2.0 - 1
            diy = self.c.nyref - self.c.ny / 2.0 - 1
            z = (vr + 1j * vi) * np.exp(1j * (ut * dix + vt * diy))
            vr, vi = np.ascontiguousarray(z.real), np.ascontiguousarray(z.imag)
        return vr, vi


TERM_NAMES = ["chisq", "chisqfcv", "chisqamp", "chisqcp", "chisqca", "reg", "l1_cost", "tv_cost",
              "tsv_cost", "kl_cost", "gs_cost", "tfd_cost", "cen_cost", "sm_cost", "cost"]


def nufft2d2(u, v, img, eps=1e-6):
    """Type-2 NUFFT of an (ny, nx) image (eps <= 0: exact DFT)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    img = np.ascontiguousarray(img, dtype=np.float64)
    ny, nx = img.shape
    vr, vi = np.empty(u.size), np.empty(u.size)
    lib().orc_nufft2d2(u.size, _d(u), _d(v), nx, ny, _d(img), float(eps), _d(vr), _d(vi))
    return vr + 1j * vi


def nufft2d1(u, v, c, nx, ny, eps=1e-6):
    """Type-1 NUFFT onto an (ny, nx) grid (eps <= 0: exact DFT)."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    cr = np.ascontiguousarray(np.real(c), dtype=np.float64)
    ci = np.ascontiguousarray(np.imag(c), dtype=np.float64)
    ore, oim = np.empty(nx * ny), np.empty(nx * ny)
    lib().orc_nufft2d1(u.size, _d(u), _d(v), _d(cr), _d(ci), nx, ny, float(eps), _d(ore), _d(oim))
    return (ore + 1j * oim).reshape(ny, nx)


def calc_cost(kw: dict, x, eps=1e-6):
    """One evaluation of calc_cost at image vector x: returns (terms dict, grad)."""
    a = kw if isinstance(kw, Args) else Args(kw)
    vr, vi = a.shifted_fcv()
    w = a.weights()
    x = np.ascontiguousarray(x, dtype=np.float64)
    terms = np.zeros(15)
    grad = np.zeros(a.c.npix)
    lib().orc_calc_cost(a.ptr(), _d(vr), _d(vi), *w, _d(x), float(eps), _d(terms), _d(grad))
    return dict(zip(TERM_NAMES, terms)), grad


def imaging(kw: dict, eps=1e-6, trace_len=None):
    """fftim2d.imaging on the CPU.  Returns (Iout, terms dict, info dict)."""
    a = Args(kw)
    niter = int(kw["niter"])
    iout = np.zeros(a.c.npix)
    terms = np.zeros(15)
    tl = (trace_len or niter + 2)
    trace = np.full(tl, np.nan)
    nfg, nit, task = C.c_int(0), C.c_int(0), C.c_int(0)
    lib().orc_imaging(a.ptr(), niter, int(bool(kw["nonneg"])), int(kw["nprint"]), int(kw["m"]),
                      float(kw["factr"]), float(kw["pgtol"]), float(eps), _d(iout), _d(terms),
                      _d(trace), C.byref(nfg), C.byref(nit), C.byref(task))
    return iout, dict(zip(TERM_NAMES, terms)), {"nfg": nfg.value, "niter": nit.value,
                                                  "task": task.value, "trace": trace}


class _Args3d(C.Structure):
    _fields_ = [
        ("npix", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("iin", C.c_void_p), ("xidx", C.c_void_p), ("yidx", C.c_void_p),
        ("nxref", C.c_double), ("nyref", C.c_double),
        ("nuv", C.c_int), ("u", C.c_void_p), ("v", C.c_void_p), ("nuvs", C.c_void_p),
        ("l1_l", C.c_double), ("l1_wgt", C.c_void_p), ("tv_l", C.c_double), ("tv_wgt", C.c_void_p),
        ("tsv_l", C.c_double), ("tsv_wgt", C.c_void_p), ("kl_l", C.c_double), ("kl_wgt", C.c_void_p),
        ("gs_l", C.c_double), ("gs_wgt", C.c_void_p),
        ("tfd_l", C.c_double), ("tfd_tgtfd", C.c_double),
        ("lc_l", C.c_void_p), ("lc_tgtfd", C.c_void_p), ("lc_nidx", C.c_int),
        ("cen_l", C.c_double), ("cen_alpha", C.c_double),
        ("sm_l", C.c_double), ("sm_maj", C.c_double), ("sm_min", C.c_double), ("sm_phi", C.c_double),
        ("rt_l", C.c_double), ("rt_wgt", C.c_void_p), ("ri_l", C.c_double), ("ri_wgt", C.c_void_p),
        ("rs_l", C.c_double), ("rf_l", C.c_double),
        ("isfcv", C.c_int), ("nfcv", C.c_int), ("uvidxfcv", C.c_void_p), ("vfcvr", C.c_void_p),
        ("vfcvi", C.c_void_p), ("varfcv", C.c_void_p), ("wfcv", C.c_double),
        ("isamp", C.c_int), ("namp", C.c_int), ("uvidxamp", C.c_void_p), ("vamp", C.c_void_p),
        ("varamp", C.c_void_p), ("wamp", C.c_double),
        ("iscp", C.c_int), ("ncp", C.c_int), ("uvidxcp", C.c_void_p), ("cp", C.c_void_p),
        ("varcp", C.c_void_p), ("wcp", C.c_double),
        ("isca", C.c_int), ("nca", C.c_int), ("uvidxca", C.c_void_p), ("ca", C.c_void_p),
        ("varca", C.c_void_p), ("wca", C.c_double),
        ("inormfactr", C.c_double),
    ]


TERM_NAMES_3D = ["chisq", "chisqfcv", "chisqamp", "chisqcp", "chisqca", "reg", "l1_cost", "sm_cost",
                 "tv_cost", "tsv_cost", "kl_cost", "gs_cost", "tfd_cost", "lc_cost", "cen_cost",
                 "rt_cost", "ri_cost", "rs_cost", "rf_cost", "cost"]


class Args3d(Args):
    """fortlib.fftim3d.imaging kwargs (fftim3d.f90:11-44) as a C struct."""

    def __init__(self, kw: dict):
        f64 = lambda k: np.ascontiguousarray(np.asarray(kw[k], dtype=np.float64).reshape(-1))
        i32 = lambda k: np.ascontiguousarray(np.asarray(kw[k], dtype=np.int32).reshape(-1))
        self.keep = {}
        a = _Args3d()
        for k in ["iin", "u", "v", "l1_wgt", "tv_wgt", "tsv_wgt", "kl_wgt", "gs_wgt", "lc_l", "lc_tgtfd",
                  "rt_wgt", "ri_wgt", "vfcvr", "vfcvi", "varfcv", "vamp", "varamp", "cp", "varcp", "ca",
                  "varca"]:
            self.keep[k] = f64(k)
        for k in ["xidx", "yidx", "uvidxfcv", "uvidxamp", "nuvs"]:
            self.keep[k] = i32(k)
        self.keep["uvidxcp"] = np.ascontiguousarray(np.asarray(kw["uvidxcp"], dtype=np.int32).T).reshape(-1)
        self.keep["uvidxca"] = np.ascontiguousarray(np.asarray(kw["uvidxca"], dtype=np.int32).T).reshape(-1)
        for k, arr in self.keep.items():
            setattr(a, k, arr.ctypes.data)
        a.npix = int(kw["npix"])
        a.nx, a.ny, a.nz = int(kw["nx"]), int(kw["ny"]), int(kw["nz"])
        a.nxref, a.nyref = float(kw["nxref"]), float(kw["nyref"])
        a.nuv = self.keep["u"].size
        for k in ["l1_l", "tv_l", "tsv_l", "kl_l", "gs_l", "tfd_l", "tfd_tgtfd", "cen_l", "cen_alpha",
                  "sm_l", "sm_maj", "sm_min", "sm_phi", "rt_l", "ri_l", "rs_l", "rf_l", "wfcv", "wamp", "wcp",
                  "wca", "inormfactr"]:
            setattr(a, k, float(kw[k]))
        a.lc_nidx = int(kw["lc_nidx"])
        a.isfcv, a.isamp, a.iscp, a.isca = (int(bool(kw[k])) for k in ["isfcv", "isamp", "iscp", "isca"])
        a.nfcv = self.keep["uvidxfcv"].size
        a.namp = self.keep["uvidxamp"].size
        a.ncp = self.keep["uvidxcp"].size // 3
        a.nca = self.keep["uvidxca"].size // 4
        self.c = a
        self.kw = kw


def calc_cost3d(kw: dict, x, eps=1e-6):
    """calc_cost of fftim3d at movie vector x (npix * nz): (terms dict, grad)."""
    a = kw if isinstance(kw, Args3d) else Args3d(kw)
    vr, vi = a.shifted_fcv()
    w = a.weights()
    x = np.ascontiguousarray(x, dtype=np.float64)
    terms = np.zeros(20)
    grad = np.zeros(a.c.npix * a.c.nz)
    lib().orc_calc_cost3d(C.byref(a.c), _d(vr), _d(vi), *w, _d(x), float(eps), _d(terms), _d(grad))
    return dict(zip(TERM_NAMES_3D, terms)), grad


def imaging3d(kw: dict, eps=1e-6, trace_len=None):
    """fftim3d.imaging on the CPU.  Returns (Iout, terms dict, info dict)."""
    a = Args3d(kw)
    niter = int(kw["niter"])
    iout = np.zeros(a.c.npix * a.c.nz)
    terms = np.zeros(20)
    trace = np.full(trace_len or niter + 2, np.nan)
    nfg, nit, task = C.c_int(0), C.c_int(0), C.c_int(0)
    lib().orc_imaging3d(C.byref(a.c), niter, int(bool(kw["nonneg"])), int(kw["nprint"]), int(kw["m"]),
                        float(kw["factr"]), float(kw["pgtol"]), float(eps), _d(iout), _d(terms), _d(trace),
                        C.byref(nfg), C.byref(nit), C.byref(task))
    return iout, dict(zip(TERM_NAMES_3D, terms)), {"nfg": nfg.value, "niter": nit.value,
                                                     "task": task.value, "trace": trace}


TASK_FG, TASK_NEW_X, TASK_CONV, TASK_ABNORMAL, TASK_ERROR, TASK_STOP = 1, 2, 3, 4, 5, 6


class Lbfgsb:
    """Reverse-communication L-BFGS-B (restatement of src/lbfgsb/lbfgsb.f)."""

    def __init__(self, n, m=5, lower=None, upper=None, nbd=None, factr=1e1, pgtol=0.0):
        self.n = n
        self.l = np.zeros(n) if lower is None else np.ascontiguousarray(lower, dtype=np.float64)
        self.u = np.zeros(n) if upper is None else np.ascontiguousarray(upper, dtype=np.float64)
        self.nbd = np.zeros(n, np.int32) if nbd is None else np.ascontiguousarray(nbd, dtype=np.int32)
        self.h = lib().orc_lbfgsb_new(n, m, _d(self.l), _d(self.u), _i(self.nbd), factr, pgtol)

    def step(self, x, f, g):
        g = np.ascontiguousarray(g, dtype=np.float64)
        return lib().orc_lbfgsb_step(self.h, _d(x), float(f), _d(g))

    def info(self):
        it, nf, col = C.c_int(), C.c_int(), C.c_int()
        th, sb = C.c_double(), C.c_double()
        lib().orc_lbfgsb_info(self.h, C.byref(it), C.byref(nf), C.byref(col), C.byref(th), C.byref(sb))
        return {"iter": it.value, "nfgv": nf.value, "col": col.value, "theta": th.value,
                "sbgnrm": sb.value}

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_lbfgsb_free(self.h)
            self.h = None


def minimize(fun, x0, m=5, lower=None, nbd=None, factr=1e1, pgtol=0.0, maxiter=100):
    """Drive the restated L-BFGS-B like fftim2d does; returns (x, f trace at NEW_X)."""
    x = np.array(x0, dtype=np.float64)
    opt = Lbfgsb(x.size, m, lower, None, nbd, factr, pgtol)
    f, g = fun(x)
    task = opt.step(x, f, g)
    trace = []
    while task in (TASK_FG, TASK_NEW_X):
        if task == TASK_FG:
            f, g = fun(x)
        else:
            trace.append(f)
            if opt.info()["iter"] > maxiter:
                break
        task = opt.step(x, f, g)
    return x, np.array(trace), task


def model_terms(kw: dict, term: str, x, eps=0.0):
    """model_fcv / amp / cp / ca (fftlib.f90:744-1254) restated in numpy over
    the oracle's transforms: (chisq, grad, model, resid) of one data term
    with unit weight; model / resid complex for fcv, real otherwise."""
    a = Args(kw)
    k = a.keep
    nx, ny = a.c.nx, a.c.ny
    img = np.zeros((ny, nx))
    img[k["yidx"] - 1, k["xidx"] - 1] = x
    V = nufft2d2(k["u"], k["v"], img, eps)
    rre, rim = np.zeros(V.size), np.zeros(V.size)
    if term == "fcv":
        idx, sg = np.abs(k["uvidxfcv"]) - 1, np.sign(k["uvidxfcv"])
        dix, diy = a.c.nxref - nx / 2.0 - 1, a.c.nyref - ny / 2.0 - 1
        ph = np.exp(1j * (k["u"][idx] * sg * dix + k["v"][idx] * sg * diy))
        data = (k["vfcvr"] + 1j * k["vfcvi"]) * ph
        model = np.where(sg > 0, V[idx], np.conj(V[idx]))
        resid = data - model
        var = k["varfcv"]
        chisq = float(np.sum(np.abs(resid) ** 2 / var))
        np.add.at(rre, idx, -2 / var * resid.real)
        np.add.at(rim, idx, -2 / var * resid.imag * sg)
        model, resid = model / ph, resid / ph
    elif term == "amp":
        idx = np.abs(k["uvidxamp"]) - 1
        model = np.abs(V[idx])
        resid = k["vamp"] - model
        var = k["varamp"]
        chisq = float(np.sum(resid ** 2 / var))
        f = -2 * resid / var / model
        np.add.at(rre, idx, f * V[idx].real)
        np.add.at(rim, idx, f * V[idx].imag)
    elif term == "cp":
        ii = k["uvidxcp"].reshape(-1, 3)
        idx, sg = np.abs(ii) - 1, np.sign(ii)
        Vq = V[idx]
        model = np.sum(np.angle(Vq) * sg, axis=1)
        resid = k["cp"] - model
        var = k["varcp"]
        chisq = float(np.sum(2 * (1 - np.cos(resid)) / var))
        f = -2 * np.sin(resid) / var
        a2 = np.abs(Vq) ** 2
        for q in range(3):
            np.add.at(rre, idx[:, q], -f / a2[:, q] * Vq[:, q].imag * sg[:, q])
            np.add.at(rim, idx[:, q], f / a2[:, q] * Vq[:, q].real * sg[:, q])
        resid = np.arctan2(np.sin(resid), np.cos(resid))
        model = np.arctan2(np.sin(model), np.cos(model))
    else:
        ii = k["uvidxca"].reshape(-1, 4)
        idx = np.abs(ii) - 1
        Vq = V[idx]
        amp = np.abs(Vq)
        model = np.log(amp[:, 0]) + np.log(amp[:, 1]) - np.log(amp[:, 2]) - np.log(amp[:, 3])
        resid = k["ca"] - model
        var = k["varca"]
        chisq = float(np.sum(resid ** 2 / var))
        f = -2 * resid / var
        for q, s in enumerate((1, 1, -1, -1)):
            np.add.at(rre, idx[:, q], s * f / amp[:, q] ** 2 * Vq[:, q].real)
            np.add.at(rim, idx[:, q], s * f / amp[:, q] ** 2 * Vq[:, q].imag)
    g2 = nufft2d1(k["u"], k["v"], rre - 1j * rim, nx, ny, eps).real
    return chisq, g2[k["yidx"] - 1, k["xidx"] - 1], model, resid
