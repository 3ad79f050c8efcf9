"""The forward model and the model terms against the reference's own
analytic source models (``smili/geomodel/geomodel.py``, run here by
``tests/golden/make_geomodel.py``; fixture ``tests/golden/geomodel_pin.npz``).

A source of three offset elliptical Gaussians is sampled on a 64 x 64 grid of
2 uas pixels.  The models of the pixel image (model_fcv / amp / cp / ca,
fftlib.f90:744-1254, with the reference's phase centre shift and closure
conventions) must equal the reference's analytic values at the same uv
coordinates:

- V(u, v) (geomodel.py:114-118, with the offsets of geomodel.py:84-91);
- |V| (``Vamp``, geomodel.py:120-129);
- the bispectrum phase (``Bphase``, geomodel.py:206-217);
- the log closure amplitude (``logCamp``, geomodel.py:237-253).

The Gaussians are resolved by many pixels and lie well inside the field, so
the pixel sum equals the continuous transform to rounding.  The CPU oracle
(exact DFT) agrees to 1e-13; the bounds are 1e-11 (visibilities and
amplitudes relative to the largest, phases and log amplitudes absolute).  On
the GPU (FP64, NUFFT tolerance 1e-12) the bounds are 1e-10.  This pins the
transform's sign, axes, units and phase centre (A2, A3) and the four models
(A5) against reference code.
"""
import importlib.util
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "geomodel_pin.npz")


def _maker():
    spec = importlib.util.spec_from_file_location("make_geomodel", os.path.join(HERE, "golden", "make_geomodel.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def pin():
    z = np.load(FIX)
    img, t = _maker().tables()
    # the tables the fixture was made on
    assert np.array_equal(t["vistable"]["u"].values, z["vis_u"])
    assert np.array_equal(t["vistable"]["v"].values, z["vis_v"])
    assert np.array_equal(t["bstable"][["u12", "v12", "u23", "v23", "u31", "v31"]].values, z["bs_uv"])
    assert np.array_equal(t["catable"][["u1", "v1", "u2", "v2", "u3", "v3", "u4", "v4"]].values, z["ca_uv"])
    img.data[0, 0] = z["image"]
    return z, img, t


TERMS = [("fcv", "vistable", "V"), ("amp", "amptable", "Vamp"), ("cp", "bstable", "Bphase"),
         ("ca", "catable", "logCamp")]


def _kw(img, table_name, table, z):
    from smili_b200.imaging.lbfgs import prepare_imaging
    extra = {} if table_name in ("vistable", "amptable") else {
        "totalflux": float(z["image"].sum()), "tfd_lambda": 1.0}  # closure data need a flux constraint
    kw, _ = prepare_imaging(img, niter=1, **{table_name: table}, **extra)
    return kw


def _err(term, model, ref):
    if term in ("fcv", "amp"):
        return np.abs(model - ref).max() / np.abs(ref).max()
    if term == "cp":
        return np.abs(np.angle(np.exp(1j * (model - ref)))).max()
    return np.abs(model - ref).max()


@pytest.mark.parametrize("term,table,key", TERMS)
def test_oracle_models_equal_reference_geomodel(oracle, pin, term, table, key):
    z, img, t = pin
    kw = _kw(img, table, t[table], z)
    x = np.asarray(kw["iin"]) / float(kw["inormfactr"])  # flux per pixel
    _, _, model, _ = oracle.model_terms(kw, term, x, eps=0.0)
    assert _err(term, np.asarray(model), z[key]) <= 1e-11
    if term == "cp":
        assert np.abs(z[key]).max() > 1.0  # the source is not symmetric: closure phases are not trivial


@pytest.mark.gpu
@pytest.mark.parametrize("term,table,key", TERMS)
def test_gpu_models_equal_reference_geomodel(pin, term, table, key):
    from smili_b200.fortlib import fftlib
    z, img, t = pin
    kw = _kw(img, table, t[table], z)
    x = np.asarray(kw["iin"]) / float(kw["inormfactr"])
    args = [x] + [kw[k] for k in ("xidx", "yidx", "nxref", "nyref", "nx", "ny", "u", "v")]
    if term == "fcv":
        out = fftlib.model_fcv(*args, kw["uvidxfcv"], kw["vfcvr"], kw["vfcvi"], kw["varfcv"], nufft_eps=1e-12)
        model = out[2] + 1j * out[3]
    elif term == "amp":
        model = fftlib.model_amp(*args, kw["uvidxamp"], kw["vamp"], kw["varamp"], nufft_eps=1e-12)[2]
    elif term == "cp":
        model = fftlib.model_cp(*args, kw["uvidxcp"], kw["cp"], kw["varcp"], nufft_eps=1e-12)[2]
    else:
        model = fftlib.model_ca(*args, kw["uvidxca"], kw["ca"], kw["varca"], nufft_eps=1e-12)[2]
    assert _err(term, np.asarray(model), z[key]) <= 1e-10
