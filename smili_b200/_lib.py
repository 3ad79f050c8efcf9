"""ctypes binding of ``libsmili_b200.so`` (declared in include/smili_b200.h).

The library is built in-tree by ``smili_b200.build`` (nvcc, sm_100a).  There
is no CPU fallback: loading fails loudly when the library is missing, and
every call raises ``SmiliError`` on a nonzero status.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsmili_b200.so")

_lib = None


class SmiliError(RuntimeError):
    """A nonzero status returned by the CUDA library."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"smili_b200 error {code}: {msg}")
        self.code = code


class ImagingArgs(C.Structure):
    """``smili_imaging_args``: the arguments of fortlib.fftim2d.imaging."""
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


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("nufft_eps", C.c_double), ("ctas_per_problem", C.c_int),
                ("device", C.c_int), ("stream", C.c_void_p), ("spread_bin", C.c_int),
                ("transform", C.c_int)]


class ImagingArgs3D(C.Structure):
    """``smili_imaging3d_args``: the arguments of fortlib.fftim3d.imaging."""
    _fields_ = [
        ("npix", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("iin", C.c_void_p), ("xidx", C.c_void_p), ("yidx", C.c_void_p),
        ("nxref", C.c_double), ("nyref", C.c_double),
        ("nuv", C.c_int), ("u", C.c_void_p), ("v", C.c_void_p), ("nuvs", C.c_void_p),
        ("l1_l", C.c_double), ("l1_wgt", C.c_void_p), ("l1_nwgt", C.c_int),
        ("sm_l", C.c_double), ("sm_maj", C.c_double), ("sm_min", C.c_double), ("sm_phi", C.c_double),
        ("tv_l", C.c_double), ("tv_wgt", C.c_void_p), ("tv_nwgt", C.c_int),
        ("tsv_l", C.c_double), ("tsv_wgt", C.c_void_p), ("tsv_nwgt", C.c_int),
        ("kl_l", C.c_double), ("kl_wgt", C.c_void_p), ("kl_nwgt", C.c_int),
        ("gs_l", C.c_double), ("gs_wgt", C.c_void_p), ("gs_nwgt", C.c_int),
        ("tfd_l", C.c_double), ("tfd_tgtfd", C.c_double),
        ("lc_l", C.c_void_p), ("lc_tgtfd", C.c_void_p), ("lc_nidx", C.c_int),
        ("cen_l", C.c_double), ("cen_alpha", C.c_double),
        ("rt_l", C.c_double), ("rt_wgt", C.c_void_p), ("rt_nwgt", C.c_int),
        ("ri_l", C.c_double), ("ri_wgt", C.c_void_p), ("ri_nwgt", C.c_int),
        ("rs_l", C.c_double), ("rs_wgt", C.c_void_p), ("rs_nwgt", C.c_int),
        ("rf_l", C.c_double), ("rf_wgt", C.c_void_p), ("rf_nwgt", C.c_int),
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


class SolveInfo(C.Structure):
    _fields_ = [("task", C.c_int), ("niter", C.c_int), ("nfg", C.c_int), ("error", C.c_int)]


TERM_NAMES = ["chisq", "chisqfcv", "chisqamp", "chisqcp", "chisqca", "reg", "l1_cost", "tv_cost",
              "tsv_cost", "kl_cost", "gs_cost", "tfd_cost", "cen_cost", "sm_cost", "cost"]
TERM_NAMES_3D = ["chisq", "chisqfcv", "chisqamp", "chisqcp", "chisqca", "reg", "l1_cost", "sm_cost",
                 "tv_cost", "tsv_cost", "kl_cost", "gs_cost", "tfd_cost", "lc_cost", "cen_cost",
                 "rt_cost", "ri_cost", "rs_cost", "rf_cost", "cost"]
TASK_CONV, TASK_ABNORMAL, TASK_STOP, TASK_ERROR, TASK_TARGET = 3, 4, 5, 6, 8

EXPORTS = ["smili_fftim2d_imaging", "smili_calc_cost", "smili_batch_create", "smili_batch_run",
           "smili_batch_fetch", "smili_batch_trace", "smili_batch_destroy", "smili_nufft_fwd_real",
           "smili_nufft_adj_real1d", "smili_last_error", "smili_version", "smili_batch_profile",
           "smili_batch_set_targets", "smili_calc_cost_noalloc", "smili_fftim3d_imaging",
           "smili_calc_cost3d", "smili_model_terms", "smili_get_uvlist", "smili_batch_set_start", "smili_batch_set_niter",
           "smili_batch_images", "smili_batch_set_starts_from_images", "smili_batch_reset_starts"]
STAGES = ["t2_rows", "t2_cols", "interp", "chisq", "spread", "t1_rows", "t1_cols", "reg_grad",
          "lb_post", "cauchy", "formk", "subsm", "lnsrch", "init", "other", "n_fg", "c_select",
          "c_gather", "c_sort", "c_scan", "c_rounds"]


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with smili_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.smili_last_error.restype = C.c_char_p
        L.smili_fftim2d_imaging.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                            C.c_double, vp, dp, dp, vp]
        L.smili_calc_cost.argtypes = [vp, dp, vp, dp, dp]
        L.smili_calc_cost_noalloc.argtypes = [vp, dp, vp, dp, dp]
        L.smili_fftim3d_imaging.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                            C.c_double, vp, dp, dp, vp]
        L.smili_calc_cost3d.argtypes = [vp, dp, vp, dp, dp]
        L.smili_model_terms.argtypes = [vp, dp, vp, C.POINTER(C.c_double), dp, dp, dp, dp, dp]
        L.smili_get_uvlist.argtypes = [C.c_int, dp, dp, vp, C.POINTER(C.c_int), dp, dp, C.POINTER(C.c_int)]
        L.smili_batch_create.argtypes = [C.c_int, C.POINTER(vp), ip, C.c_int, C.c_int, C.c_double,
                                         C.c_double, vp, C.POINTER(vp)]
        L.smili_batch_run.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        L.smili_batch_fetch.argtypes = [vp, C.c_int, dp, dp, dp, vp]
        L.smili_batch_trace.argtypes = [vp, C.c_int, dp, C.c_int]
        L.smili_batch_destroy.argtypes = [vp]
        L.smili_batch_destroy.restype = None
        L.smili_batch_profile.argtypes = [vp, C.c_int, dp, C.c_int]
        L.smili_batch_set_targets.argtypes = [vp, dp]
        L.smili_batch_set_start.argtypes = [vp, C.c_int, dp]
        L.smili_batch_set_niter.argtypes = [vp, ip]
        L.smili_batch_images.argtypes = [vp, vp, C.c_int, C.c_int]
        L.smili_batch_set_starts_from_images.argtypes = [vp, vp, C.c_int, C.c_int, vp]
        L.smili_batch_reset_starts.argtypes = [vp]
        L.smili_nufft_fwd_real.argtypes = [C.c_int, dp, dp, C.c_int, C.c_int, dp, vp, dp, dp]
        L.smili_nufft_adj_real1d.argtypes = [C.c_int, dp, dp, dp, dp, C.c_int, C.c_int, vp, dp]
        _lib = L
    return _lib


def check(rc: int):
    if rc != 0:
        raise SmiliError(rc, lib().smili_last_error().decode())


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_options(precision=64, nufft_eps=0.0, ctas_per_problem=0, device=0, stream=None, spread_bin=0,
                 transform=0):
    o = Options()
    o.spread_bin = int(spread_bin)
    o.transform = int(transform)
    o.precision = int(precision)
    o.nufft_eps = float(nufft_eps)
    o.ctas_per_problem = int(ctas_per_problem)
    o.device = int(device)
    o.stream = stream
    return o


class Problem:
    """Holds contiguous copies of the fftim2d.imaging keyword arrays and the
    ``smili_imaging_args`` struct that points into them."""

    F64 = ["iin", "u", "v", "l1_wgt", "tv_wgt", "tsv_wgt", "kl_wgt", "gs_wgt", "vfcvr", "vfcvi",
           "varfcv", "vamp", "varamp", "cp", "varcp", "ca", "varca"]
    I32 = ["xidx", "yidx", "uvidxfcv", "uvidxamp"]
    SCAL = ["l1_l", "tv_l", "tsv_l", "kl_l", "gs_l", "tfd_l", "tfd_tgtfd", "cen_l", "cen_alpha",
            "sm_l", "sm_maj", "sm_min", "sm_phi", "wfcv", "wamp", "wcp", "wca", "inormfactr"]

    def __init__(self, kw: dict):
        self.kw = kw
        self.keep = {}
        a = ImagingArgs()
        for k in self.F64:
            self.keep[k] = np.ascontiguousarray(np.asarray(kw[k], dtype=np.float64).reshape(-1))
        for k in self.I32:
            self.keep[k] = np.ascontiguousarray(np.asarray(kw[k], dtype=np.int32).reshape(-1))
        # (3,Ncp) / (4,Nca) in Fortran order: the indices of one datum contiguous
        self.keep["uvidxcp"] = np.ascontiguousarray(np.asarray(kw["uvidxcp"], dtype=np.int32).T).reshape(-1)
        self.keep["uvidxca"] = np.ascontiguousarray(np.asarray(kw["uvidxca"], dtype=np.int32).T).reshape(-1)
        for k, arr in self.keep.items():
            setattr(a, k, arr.ctypes.data)
        a.npix = int(kw["npix"])
        a.nx, a.ny = int(kw["nx"]), int(kw["ny"])
        a.nxref, a.nyref = float(kw["nxref"]), float(kw["nyref"])
        a.nuv = self.keep["u"].size
        for k in self.SCAL:
            setattr(a, k, float(kw[k]))
        for k in ["l1", "tv", "tsv", "kl", "gs"]:
            setattr(a, k + "_nwgt", int(kw[k + "_nwgt"]))
        a.isfcv, a.isamp, a.iscp, a.isca = (int(bool(kw[k])) for k in ["isfcv", "isamp", "iscp", "isca"])
        a.nfcv = self.keep["uvidxfcv"].size
        a.namp = self.keep["uvidxamp"].size
        a.ncp = self.keep["uvidxcp"].size // 3
        a.nca = self.keep["uvidxca"].size // 4
        self.c = a

    @property
    def npix(self):
        return self.c.npix


class Movie:
    """Contiguous copies of the fftim3d.imaging keyword arrays and the
    ``smili_imaging3d_args`` struct that points into them."""

    F64 = ["iin", "u", "v", "l1_wgt", "tv_wgt", "tsv_wgt", "kl_wgt", "gs_wgt", "lc_l", "lc_tgtfd", "rt_wgt",
           "ri_wgt", "rs_wgt", "rf_wgt", "vfcvr", "vfcvi", "varfcv", "vamp", "varamp", "cp", "varcp", "ca",
           "varca"]
    I32 = ["xidx", "yidx", "uvidxfcv", "uvidxamp", "nuvs"]
    SCAL = ["l1_l", "sm_l", "sm_maj", "sm_min", "sm_phi", "tv_l", "tsv_l", "kl_l", "gs_l", "tfd_l", "tfd_tgtfd",
            "cen_l", "cen_alpha", "rt_l", "ri_l", "rs_l", "rf_l", "wfcv", "wamp", "wcp", "wca", "inormfactr"]

    def __init__(self, kw: dict):
        self.kw = kw
        self.keep = {}
        a = ImagingArgs3D()
        for k in self.F64:
            self.keep[k] = np.ascontiguousarray(np.asarray(kw[k], dtype=np.float64).reshape(-1))
        for k in self.I32:
            self.keep[k] = np.ascontiguousarray(np.asarray(kw[k], dtype=np.int32).reshape(-1))
        self.keep["uvidxcp"] = np.ascontiguousarray(np.asarray(kw["uvidxcp"], dtype=np.int32).T).reshape(-1)
        self.keep["uvidxca"] = np.ascontiguousarray(np.asarray(kw["uvidxca"], dtype=np.int32).T).reshape(-1)
        for k, arr in self.keep.items():
            setattr(a, k, arr.ctypes.data)
        a.npix = int(kw["npix"])
        a.nx, a.ny, a.nz = int(kw["nx"]), int(kw["ny"]), int(kw["nz"])
        a.nxref, a.nyref = float(kw["nxref"]), float(kw["nyref"])
        a.nuv = self.keep["u"].size
        for k in self.SCAL:
            setattr(a, k, float(kw[k]))
        for k in ["l1", "tv", "tsv", "kl", "gs", "rt", "ri", "rs", "rf"]:
            setattr(a, k + "_nwgt", int(kw[k + "_nwgt"]))
        a.lc_nidx = int(kw["lc_nidx"])
        a.isfcv, a.isamp, a.iscp, a.isca = (int(bool(kw[k])) for k in ["isfcv", "isamp", "iscp", "isca"])
        a.nfcv = self.keep["uvidxfcv"].size
        a.namp = self.keep["uvidxamp"].size
        a.ncp = self.keep["uvidxcp"].size // 3
        a.nca = self.keep["uvidxca"].size // 4
        self.c = a

    @property
    def n(self):
        return self.c.npix * self.c.nz


class Batch:
    """Device-resident batch of imaging problems (smili_batch_*)."""

    def __init__(self, problems, niter, nonneg=True, m=5, factr=1e1, pgtol=0.0, options=None):
        self.problems = [p if isinstance(p, Problem) else Problem(p) for p in problems]
        n = len(self.problems)
        ptrs = (C.c_void_p * n)(*[C.addressof(p.c) for p in self.problems])
        nit = np.ascontiguousarray(np.broadcast_to(np.asarray(niter, dtype=np.int32), (n,)))
        self.options = options or make_options()
        h = C.c_void_p()
        check(lib().smili_batch_create(n, ptrs, nit.ctypes.data_as(C.POINTER(C.c_int)), int(bool(nonneg)),
                                       int(m), float(factr), float(pgtol), C.byref(self.options),
                                       C.byref(h)))
        self.h = h
        self.n = n

    def run(self, fg_only=False):
        """Run on the device; returns the launch's device time in ms.
        fg_only: False solve, True one evaluation, 2 time 1000 group barriers,
        3 check the bounded waits (a barrier one CTA skips: SMILI_ERR_TIMEOUT)."""
        ms = C.c_float(0.0)
        mode = fg_only if fg_only in (2, 3) else int(bool(fg_only))
        check(lib().smili_batch_run(self.h, mode, C.byref(ms)))
        return float(ms.value)

    def fetch(self, p):
        npix = self.problems[p].npix
        x, g = np.zeros(npix), np.zeros(npix)
        terms = np.zeros(15)
        info = SolveInfo()
        check(lib().smili_batch_fetch(self.h, p, dptr(x), dptr(terms), dptr(g), C.byref(info)))
        return x, dict(zip(TERM_NAMES, terms)), g, {"task": info.task, "niter": info.niter,
                                                     "nfg": info.nfg, "error": info.error}

    def set_targets(self, ftarget):
        """Stop problem p once its cost <= ftarget[p] (None clears)."""
        if ftarget is None:
            check(lib().smili_batch_set_targets(self.h, None))
        else:
            t = np.ascontiguousarray(np.broadcast_to(np.asarray(ftarget, dtype=np.float64), (self.n,)))
            check(lib().smili_batch_set_targets(self.h, dptr(t)))

    def set_niter(self, niter):
        """Iteration caps of the next runs (each at most the cap at creation); None restores them."""
        if niter is None:
            check(lib().smili_batch_set_niter(self.h, None))
        else:
            n = np.ascontiguousarray(np.broadcast_to(np.asarray(niter, dtype=np.int32), (self.n,)))
            check(lib().smili_batch_set_niter(self.h, n.ctypes.data_as(C.POINTER(C.c_int))))

    def info(self, p):
        """Task, iteration and evaluation counts of problem p after the last run."""
        info = SolveInfo()
        check(lib().smili_batch_fetch(self.h, p, None, None, None, C.byref(info)))
        return {"task": info.task, "niter": info.niter, "nfg": info.nfg, "error": info.error}

    def images(self, dst):
        """Every problem's current image, scaled to max 1, into the device
        tensor dst of shape (n, ny, nx), float32 (all problems nx x ny)."""
        n, ny, nx = dst.shape
        if n != self.n or not dst.is_cuda or not dst.is_contiguous() or str(dst.dtype) != "torch.float32":
            raise ValueError("dst must be a contiguous float32 CUDA tensor of shape (n, ny, nx)")
        check(lib().smili_batch_images(self.h, C.c_void_p(dst.data_ptr()), int(nx), int(ny)))

    def set_starts_from_images(self, img, keep=None):
        """Start images from the device tensor img (n, ny, nx), float32: relu(img)
        at each problem's pixels scaled to its current image's total; the
        current image where keep[p] (or where that is not possible)."""
        n, ny, nx = img.shape
        if n != self.n or not img.is_cuda or not img.is_contiguous() or str(img.dtype) != "torch.float32":
            raise ValueError("img must be a contiguous float32 CUDA tensor of shape (n, ny, nx)")
        k = None
        if keep is not None:
            k = np.ascontiguousarray(np.asarray(keep, dtype=bool).astype(np.uint8))
            if k.size != self.n:
                raise ValueError("keep needs one flag per problem")
        check(lib().smili_batch_set_starts_from_images(
            self.h, C.c_void_p(img.data_ptr()), int(nx), int(ny), None if k is None else k.ctypes.data_as(C.c_void_p)))

    def reset_starts(self):
        """Put back the start images the problems were created with."""
        check(lib().smili_batch_reset_starts(self.h))

    def set_start(self, p, x):
        """Problem p starts its next run from the pixel vector x (scaled units)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != self.problems[p].npix:
            raise ValueError("start image has the wrong number of pixels")
        check(lib().smili_batch_set_start(self.h, int(p), dptr(x)))

    def profile(self, enable=True):
        check(lib().smili_batch_profile(self.h, int(bool(enable)), None, 0))

    def stage_times(self):
        """Accumulated stage times (ms) of the last profiled run, and the FG count."""
        t = np.zeros(len(STAGES))
        check(lib().smili_batch_profile(self.h, 1, dptr(t), len(STAGES)))
        out = {k: t[i] / 1e6 for i, k in enumerate(STAGES)}
        out["n_fg"] = int(t[STAGES.index("n_fg")])
        out["c_rounds"] = int(t[STAGES.index("c_rounds")])
        return out

    def trace(self, p, length):
        t = np.zeros(length)
        check(lib().smili_batch_trace(self.h, p, dptr(t), int(length)))
        return t

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().smili_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
