"""Run the reference's own imaging driver over a replacement ``fortlib``.

``smili/imaging/lbfgs.py`` is pure Python around one f2py call.  Its package
``__init__`` and its module imports pull in matplotlib, astropy and the rest
of SMILI, none of which exist here, so the file is loaded by path as
``smili.imaging.lbfgs`` inside a throw-away ``smili`` package whose
submodules are:

- ``fortlib``: whatever the caller passes (this project's ``fortlib`` mirror,
  or a recorder around it);
- ``uvdata.uvtable.tools``: the reference's own ``tools.py``, also loaded by
  path (``get_uvlist``, smili/uvdata/uvtable/tools.py:12-132);
- ``imdata``: ``IMFITS`` is the duck-typed image of ``smili_b200.synth``;
- ``util``: ``angconv`` only.

matplotlib and mpl_toolkits get empty stand-ins: ``imaging`` never calls
them.  Everything is removed from ``sys.modules`` again on exit.

Test infrastructure: used by ``tests/`` and the fixture script in
``tests/golden/`` only.
"""
from __future__ import annotations

import contextlib
import importlib.util
import os
import sys
import types

import numpy as np

ENV = "SMILI_REFERENCE_ROOT"


def reference_root():
    """The reference checkout named by $SMILI_REFERENCE_ROOT, or None."""
    root = os.environ.get(ENV)
    if root and os.path.isfile(os.path.join(root, "smili", "imaging", "lbfgs.py")):
        return root
    return None


def _module(name, **attrs):
    m = types.ModuleType(name)
    m.__dict__.update(attrs)
    return m


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class _IMRegion:  # isinstance target only; the tests pass images as windows
    pass


@contextlib.contextmanager
def reference_lbfgs(ref_root, fortlib):
    """Yield the reference's ``smili.imaging.lbfgs`` module bound to ``fortlib``."""
    from smili_b200 import synth
    names = ["smili", "smili.imaging", "smili.imaging.lbfgs", "smili.util", "smili.imdata",
             "smili.fortlib", "smili.uvdata", "smili.uvdata.uvtable", "smili.uvdata.uvtable.tools",
             "matplotlib", "matplotlib.pyplot", "matplotlib.backends", "matplotlib.backends.backend_pdf",
             "matplotlib.ticker", "mpl_toolkits", "mpl_toolkits.axes_grid1"]
    saved = {n: sys.modules[n] for n in names if n in sys.modules}
    try:
        mpl = _module("matplotlib", use=lambda *a, **k: None)
        sys.modules.update({
            "matplotlib": mpl,
            "matplotlib.pyplot": _module("matplotlib.pyplot"),
            "matplotlib.backends": _module("matplotlib.backends"),
            "matplotlib.backends.backend_pdf": _module("matplotlib.backends.backend_pdf", PdfPages=object),
            "matplotlib.ticker": _module("matplotlib.ticker", NullFormatter=object),
            "mpl_toolkits": _module("mpl_toolkits"),
            "mpl_toolkits.axes_grid1": _module("mpl_toolkits.axes_grid1", make_axes_locatable=None),
        })
        smili = _module("smili", __path__=[])
        imaging_pkg = _module("smili.imaging", __path__=[])
        util = _module("smili.util", angconv=lambda a, b: synth.Image(1, 1, 1.0).angconv(a, b))
        imdata = _module("smili.imdata", IMFITS=synth.Image, IMRegion=_IMRegion)
        uvtable = _module("smili.uvdata.uvtable", __path__=[])
        uvdata = _module("smili.uvdata", __path__=[], uvtable=uvtable)
        sys.modules.update({"smili": smili, "smili.imaging": imaging_pkg, "smili.util": util,
                            "smili.imdata": imdata, "smili.fortlib": fortlib, "smili.uvdata": uvdata,
                            "smili.uvdata.uvtable": uvtable})
        uvtable.tools = _load("smili.uvdata.uvtable.tools",
                              os.path.join(ref_root, "smili", "uvdata", "uvtable", "tools.py"))
        smili.util, smili.imdata, smili.fortlib, smili.uvdata = util, imdata, fortlib, uvdata
        smili.imaging = imaging_pkg
        mod = _load("smili.imaging.lbfgs", os.path.join(ref_root, "smili", "imaging", "lbfgs.py"))
        yield mod
    finally:
        for n in names:
            sys.modules.pop(n, None)
        sys.modules.update(saved)


class RecordingFortlib(types.ModuleType):
    """A ``fortlib`` whose ``image`` is this project's mirror and whose
    ``fftim2d.imaging`` records its keyword arguments and returns what
    ``solve(kwargs)`` returns (the 16-tuple of fftim2d.f90:29-32)."""

    def __init__(self, solve):
        super().__init__("smili.fortlib")
        from smili_b200.fortlib import fftlib, image
        self.image = image
        self.fftlib = fftlib
        self.calls = []

        def imaging(**kw):
            self.calls.append(kw)
            return solve(kw)

        self.fftim2d = _module("smili.fortlib.fftim2d", imaging=imaging)


def oracle_solve(eps=1e-6):
    """``solve`` for ``RecordingFortlib``: the CPU oracle's solve as the 16-tuple."""
    from oracle import oracle as O

    def solve(kw):
        iout, t, _ = O.imaging(kw, eps=eps)
        keys = ["chisq", "chisqfcv", "chisqamp", "chisqcp", "chisqca", "reg", "l1_cost", "tv_cost",
                "tsv_cost", "kl_cost", "gs_cost", "tfd_cost", "cen_cost", "sm_cost", "cost"]
        return (np.asarray(iout),) + tuple(t[k] for k in keys)
    return solve


def compare_kwargs(got: dict, want: dict):
    """Assert that two fftim2d.imaging keyword sets are identical: the same
    names, numpy dtypes and bit-identical values."""
    assert sorted(got) == sorted(want), set(got) ^ set(want)
    for k in want:
        a, b = np.asarray(got[k]), np.asarray(want[k])
        assert a.shape == b.shape, (k, a.shape, b.shape)
        if a.dtype.kind in "fiub" or b.dtype.kind in "fiub":
            assert a.dtype.kind == b.dtype.kind, (k, a.dtype, b.dtype)
            assert np.array_equal(a, b, equal_nan=a.dtype.kind == 'f'), (k, np.abs(a.astype(float) - b.astype(float)).max())
        else:
            assert a.tolist() == b.tolist(), k


# ---------------------------------------------------------------------------
# fixtures: the driver's inputs and the keyword arguments it produced
# ---------------------------------------------------------------------------
TABLES = ("vistable", "amptable", "bstable", "catable")
IMAGES = ("l1_prior", "tv_prior", "tsv_prior", "kl_prior", "gs_prior", "imregion")


def _image_to(prefix, img, out):
    out[prefix + "__data"] = np.asarray(img.data)
    for k, v in img.header.items():
        out[prefix + "__h__" + k] = np.asarray(v)


def _image_from(prefix, z):
    from smili_b200 import synth
    h = {k[len(prefix) + 5:]: z[k][()] for k in z.files if k.startswith(prefix + "__h__")}
    img = synth.Image(int(h["nx"]), int(h["ny"]), 1.0)
    img.header = {k: (int(v) if k in ("nx", "ny") else float(v)) for k, v in h.items()}
    img.data = np.array(z[prefix + "__data"])
    return img


def save_case(path, initimage, options, kwargs):
    """Write one case: the driver's inputs (image, tables, scalar options,
    prior and window images) and the fftim2d.imaging kwargs it produced."""
    out = {}
    _image_to("init", initimage, out)
    for name, val in options.items():
        if name in TABLES:
            for col in val.columns:
                out[f"tab__{name}__{col}"] = np.asarray(val[col])
        elif name in IMAGES:
            _image_to(f"img__{name}", val, out)
        else:
            out[f"opt__{name}"] = np.asarray(val)
    for k, v in kwargs.items():
        out[f"kw__{k}"] = np.asarray(v)
    np.savez_compressed(path, **out)


def load_case(path):
    """Inverse of ``save_case``: (initimage, options, kwargs)."""
    import pandas as pd
    z = np.load(path)
    init = _image_from("init", z)
    options = {}
    for t in TABLES:
        cols = [k for k in z.files if k.startswith(f"tab__{t}__")]
        if cols:
            options[t] = pd.DataFrame({k[len(f"tab__{t}__"):]: z[k] for k in cols})
    for n in IMAGES:
        if f"img__{n}__data" in z.files:
            options[n] = _image_from(f"img__{n}", z)
    for k in z.files:
        if k.startswith("opt__"):
            options[k[5:]] = z[k][()]
    kwargs = {k[4:]: (z[k][()] if z[k].ndim == 0 else np.array(z[k])) for k in z.files if k.startswith("kw__")}
    return init, options, kwargs


def cases():
    """Inputs of the driver cases: (name, initimage, options)."""
    from smili_b200 import synth
    out = []
    # 1) the crescent workload's data terms and regularizers at 32x32
    o = synth.small_crescent(seed=0, nx=32, niter=30)
    out.append(("fcv_cp_l1_tsv", o.image, dict(vistable=o.vistable, bstable=o.bstable, niter=30,
                                               l1_lambda=1.0, tsv_lambda=1.0)))
    # 2) the precision path's data terms, every regularizer, priors shared
    #    between regularizers, data weights.  (A reweighted TV prior is left
    #    out: image.f90:439 divides by tv_e, which is 0 at the last row and
    #    column, so the reference's TV weights are NaN there.)
    p = synth.precision_path(seed=7, nx=40, nst=7, hours=4.0, scan_s=900.0, niter=20)
    prior = p.image.copy()
    prior.data[0, 0] = synth.gaussian_image(p.image, 30.0, 1.0, 3.0, -2.0)
    out.append(("amp_cp_ca_allreg", p.image, dict(
        amptable=p.amptable, bstable=p.bstable, catable=p.catable, niter=20, w_amp=0.5, w_bs=2.0,
        w_ca=1.5, l1_lambda=1.0, l1_prior=prior, l1_noise=1e-2, tv_lambda=0.5,
        tsv_lambda=0.7, tsv_prior=prior, kl_lambda=0.1, kl_prior=prior, gs_lambda=0.1, tfd_lambda=1.0,
        tfd_tgterror=0.02, cen_lambda=0.1, cen_alpha=2.0, sm_lambda=0.1, sm_maj=30.0, sm_min=20.0,
        sm_phi=30.0, totalflux=float(p.totalflux), inorm=2.0)))
    # 3) closure quantities only (total flux fixed by tfd), an image window,
    #    no non-negativity, no intensity scaling
    win = p.image.copy()
    yy, xx = np.mgrid[:40, :40]
    win.data[0, 0] = ((xx - 20) ** 2 + (yy - 20) ** 2 < 15 ** 2).astype(float)
    out.append(("closure_window_tfd", p.image, dict(
        bstable=p.bstable, catable=p.catable, imregion=win, niter=15, totalflux=float(p.totalflux),
        tfd_lambda=1.0, l1_lambda=0.5, tsv_lambda=0.5, nonneg=False, inorm=-1.0)))
    return out
