"""Golden values of the reference's own analytic source models.

``smili/geomodel/geomodel.py`` is pure numpy: ``GeoModel`` carries a source's
image I(x, y) and its visibility function V(u, v), and derives from V the
amplitudes (``Vamp``, geomodel.py:120-129), bispectrum phases (``Bphase``,
geomodel.py:206-217) and log closure amplitudes (``logCamp``,
geomodel.py:237-253).  This script builds a source of three elliptical
Gaussians with the reference's ``Gaussian`` (geomodel.py:326-357), samples its
image on a 64 x 64 grid of 2 uas pixels, forms seeded VLBI tables (8
stations, 230 GHz, 12 h; every data type) and evaluates the reference's model
functions at the tables' uv coordinates.  The tests compare them with the
models that this project's forward model gives for the pixel image
(model_fcv / amp / cp / ca, fftlib.f90:744-1254): the same transform sign,
axes, phase centre and closure conventions.

The offsets are applied as ``GeoModel.shift`` intends (geomodel.py:84-91:
V exp(+i dphase) with dphase from the reference's ``phaseshift``,
geomodel.py:309-323, and I(x - dx, y - dy)).  ``shift`` itself cannot be
called: it uses u and v outside the lambda that defines them, which raises
NameError.

The module is loaded by path inside a throw-away ``smili`` package (its
``__init__`` needs astropy and matplotlib, which are absent).

Usage: ``python tests/golden/make_geomodel.py /path/to/reference`` (or with
$SMILI_REFERENCE_ROOT set) writes ``tests/golden/geomodel_pin.npz``.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from smili_b200 import synth  # noqa: E402

SEED = 4242
NX, DX_UAS = 64, 2.0
# (x0, y0, flux, major FWHM, minor FWHM, position angle), uas and degrees
COMPONENTS = [(6.0, -4.0, 0.35, 18.0, 10.0, 35.0),
              (-8.0, 5.0, 0.25, 12.0, 12.0, 0.0),
              (2.0, 9.0, 0.15, 8.0, 6.0, -20.0)]


def load_geomodel(ref_root: str):
    names = ["smili", "smili.util", "smili.geomodel", "smili.geomodel.geomodel"]
    saved = {n: sys.modules[n] for n in names if n in sys.modules}
    try:
        smili = types.ModuleType("smili")
        smili.__path__ = []
        util = types.ModuleType("smili.util")
        geo = types.ModuleType("smili.geomodel")
        geo.__path__ = []
        smili.util, smili.geomodel = util, geo
        sys.modules.update({"smili": smili, "smili.util": util, "smili.geomodel": geo})
        path = os.path.join(ref_root, "smili", "geomodel", "geomodel.py")
        spec = importlib.util.spec_from_file_location("smili.geomodel.geomodel", path)
        mod = importlib.util.module_from_spec(spec)
        sys.modules["smili.geomodel.geomodel"] = mod
        spec.loader.exec_module(mod)
        return mod
    finally:
        for n in names:
            sys.modules.pop(n, None)
        sys.modules.update(saved)


def source(gm):
    total = None
    for x0, y0, flux, maj, mnr, pa in COMPONENTS:
        g = gm.Gaussian(totalflux=flux, majsize=maj, minsize=mnr, pa=pa, angunit="uas")
        dx, dy = x0 * gm.angconv("uas", "rad"), y0 * gm.angconv("uas", "rad")
        g = gm.GeoModel(V=(lambda g_, a, b: lambda u, v: g_.V(u, v) * np.exp(
            1j * gm.phaseshift(u, v, a, b, angunit="uas")))(g, x0, y0),
            I=(lambda g_, a, b: lambda x, y: g_.I(x - a, y - b))(g, dx, dy))
        total = g if total is None else total + g
    return total


def tables():
    """The seeded tables (uv coordinates; the data values are not used)."""
    img = synth.Image(NX, NX, DX_UAS)
    rng = np.random.default_rng(SEED)
    t = synth.observe(np.zeros((NX, NX)), img, rng, nst=8, dec_deg=12.0, freq_hz=230e9, hours=12.0,
                      scan_min=10.0, fcv=True, amp=True, cp=True, ca=True,
                      model=lambda truth, im, u, v: np.ones(u.size, dtype=complex))
    return img, t


def main(ref_root: str):
    gm = load_geomodel(ref_root)
    src = source(gm)
    img, t = tables()
    x, y = img.get_xygrid(twodim=True, angunit="rad")
    pix = abs(img.header["dx"] * img.header["dy"]) * (np.pi / 180.0) ** 2
    image = src.I(x, y) * pix  # flux per pixel
    vt, bt, ct = t["vistable"], t["bstable"], t["catable"]
    out = dict(
        image=image, seed=SEED,
        vis_u=vt["u"].values, vis_v=vt["v"].values,
        V=src.V(vt["u"].values, vt["v"].values),
        Vamp=src.Vamp(vt["u"].values, vt["v"].values),
        bs_uv=bt[["u12", "v12", "u23", "v23", "u31", "v31"]].values,
        Bphase=src.Bphase(*[bt[c].values for c in ("u12", "v12", "u23", "v23", "u31", "v31")]),
        ca_uv=ct[["u1", "v1", "u2", "v2", "u3", "v3", "u4", "v4"]].values,
        logCamp=src.logCamp(*[ct[c].values for c in ("u1", "v1", "u2", "v2", "u3", "v3", "u4", "v4")]))
    np.savez_compressed(os.path.join(HERE, "geomodel_pin.npz"), **out)
    print("wrote geomodel_pin.npz:", {k: np.shape(v) for k, v in out.items()})


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SMILI_REFERENCE_ROOT")
    if not root:
        raise SystemExit("usage: make_geomodel.py /path/to/reference (or set SMILI_REFERENCE_ROOT)")
    main(root)
