"""model_fcv / model_amp / model_cp / model_ca on the GPU against the oracle.

Each call evaluates one data term with unit weight: the raw chi-square,
its gradient, and every datum's model and residual, in FP64 with a tight
NUFFT tolerance (1e-12) against the oracle's exact transform: 1e-9
relative on the chi-square, models and residuals, 1e-8 on the gradient.
"""
import numpy as np
import pytest

from conftest import make_kw

pytestmark = pytest.mark.gpu


def _args(kw):
    return [kw[k] for k in ("iin", "xidx", "yidx", "nxref", "nyref", "nx", "ny", "u", "v")]


def _close(got, want, rel):
    want = np.asarray(want)
    return np.max(np.abs(np.asarray(got) - want)) <= rel * max(np.max(np.abs(want)), 1e-300)


@pytest.mark.parametrize("term", ["fcv", "cp"])
def test_model_terms_fcv_cp(oracle, crescent32, term):
    from smili_b200.fortlib import fftlib
    kw = make_kw(crescent32)
    x = np.asarray(kw["iin"]) * np.random.default_rng(0).uniform(0.5, 1.5, np.size(kw["iin"]))
    kwx = dict(kw, iin=x)
    if term == "fcv":
        c, g, mr, mi, rr, ri = fftlib.model_fcv(*_args(kwx), kw["uvidxfcv"], kw["vfcvr"], kw["vfcvi"], kw["varfcv"],
                                                nufft_eps=1e-12)
        model, resid = mr + 1j * mi, rr + 1j * ri
    else:
        c, g, model, resid = fftlib.model_cp(*_args(kwx), kw["uvidxcp"], kw["cp"], kw["varcp"], nufft_eps=1e-12)
    co, go, mo, ro = oracle.model_terms(kw, term, x, eps=0.0)
    assert abs(c - co) <= 1e-9 * co
    assert _close(g, go, 1e-8)
    assert _close(model, mo, 1e-9) and _close(resid, ro, 1e-9)
    if term == "cp":
        assert np.all(np.abs(model) <= np.pi) and np.all(np.abs(resid) <= np.pi)


@pytest.mark.parametrize("term", ["amp", "ca"])
def test_model_terms_amp_ca(oracle, closure40, term):
    from smili_b200.fortlib import fftlib
    kw = make_kw(closure40)
    x = np.asarray(kw["iin"]) * np.random.default_rng(1).uniform(0.5, 1.5, np.size(kw["iin"]))
    kwx = dict(kw, iin=x)
    fn = fftlib.model_amp if term == "amp" else fftlib.model_ca
    keys = ("uvidxamp", "vamp", "varamp") if term == "amp" else ("uvidxca", "ca", "varca")
    c, g, model, resid = fn(*_args(kwx), *[kw[k] for k in keys], nufft_eps=1e-12)
    co, go, mo, ro = oracle.model_terms(kw, term, x, eps=0.0)
    assert abs(c - co) <= 1e-9 * co
    assert _close(g, go, 1e-8)
    assert _close(model, mo, 1e-9) and _close(resid, ro, 1e-9)


def test_model_terms_reject_two_terms(crescent32):
    from smili_b200 import _lib as lib
    kw = make_kw(crescent32)
    prob = lib.Problem(kw)  # fcv and cp both present
    import ctypes as C
    x = np.ascontiguousarray(kw["iin"], dtype=np.float64)
    rc = lib.lib().smili_model_terms(C.addressof(prob.c), lib.dptr(x), None, None, None, None, None, None, None)
    assert rc == -1


def test_statistics_uses_model_terms(oracle, crescent32):
    """statistics(): chi-squares of the tables from the model terms and the
    image costs; against the oracle's model terms and numpy sums."""
    from smili_b200.imaging.lbfgs import statistics
    o = crescent32
    st = statistics(o.image, vistable=o.vistable, bstable=o.bstable, lambl1=1.0, lambtsv=1.0, nufft_eps=1e-12)
    kw = make_kw(o)
    x = np.asarray(kw["iin"]) / float(kw["inormfactr"])
    # the oracle on the raw (unnormalised) data of the same tables
    raw = dict(kw, vfcvr=kw["vfcvr"] / kw["inormfactr"], vfcvi=kw["vfcvi"] / kw["inormfactr"],
               varfcv=kw["varfcv"] / kw["inormfactr"] ** 2)
    cf = oracle.model_terms(raw, "fcv", x, eps=0.0)[0]
    cc = oracle.model_terms(raw, "cp", x, eps=0.0)[0]
    assert abs(st["chisqfcv"] - cf) <= 1e-9 * cf and abs(st["chisqcp"] - cc) <= 1e-9 * cc
    assert abs(st["rchisq"] - (cf + cc) / (2 * len(o.vistable) + len(o.bstable))) <= 1e-9 * st["rchisq"]
    I = o.image.data[0, 0]
    assert abs(st["l1"] - np.sum(np.sqrt(I * I + 1e-10))) <= 1e-12 * st["l1"]
    assert st["isfcv"] and st["iscp"] and not st["isamp"] and not st["isca"]
