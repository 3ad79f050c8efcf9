"""The C ABI without a GPU: every function that include/*.h declares is
exported by its library, and invalid inputs are rejected with the
documented error codes before any device is touched."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import make_kw

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = {"smili_b200.h": "smili_b200/libsmili_b200.so", "smili_unet.h": "smili_b200/libsmili_unet.so"}


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(smili_[a-z0-9_]+)\s*\(", text)))


@pytest.mark.parametrize("header", sorted(HEADERS))
def test_library_exports_every_declared_function(header):
    from smili_b200 import build
    build.build()
    lib = C.CDLL(os.path.join(ROOT, HEADERS[header]))
    names = declared(header)
    assert len(names) >= 8
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_lists_every_solver_export():
    from smili_b200 import _lib
    assert set(declared("smili_b200.h")) == set(_lib.EXPORTS)


def test_invalid_inputs_rejected_without_device(crescent32):
    from smili_b200 import _lib
    from smili_b200.fortlib import fftim2d
    kw = make_kw(crescent32, niter=5)
    bad = dict(kw)
    bad["varfcv"] = kw["varfcv"].copy()
    bad["varfcv"][0] = 0.0
    with pytest.raises(_lib.SmiliError) as e:
        fftim2d.calc_cost(kw["iin"], **bad)
    assert e.value.code == -2
    bad = dict(kw)
    bad["xidx"] = np.asarray(kw["xidx"]).copy()
    bad["xidx"][0] = 10 ** 6
    with pytest.raises(_lib.SmiliError) as e:
        fftim2d.calc_cost(kw["iin"], **bad)
    assert e.value.code == -1
    assert _lib.lib().smili_calc_cost(None, None, None, None, None) == -1
    assert _lib.lib().smili_version() > 0


def test_movie_closure_across_frames_rejected():
    """A closure phase whose baselines lie in two frames has no per-frame
    evaluation: the library refuses it (SMILI_ERR_UNSUPPORTED)."""
    from smili_b200 import _lib
    from smili_b200.fortlib import fftim3d
    from test_oracle3d import movie_kw
    kw, _ = movie_kw(nframes=2)
    cp = np.array(kw["uvidxcp"], copy=True)
    n0 = int(np.asarray(kw["nuvs"])[0])
    cp[0, 0] = n0 + 1  # first uv point of frame 1 in a closure of frame 0
    bad = dict(kw)
    bad["uvidxcp"] = cp
    with pytest.raises(_lib.SmiliError) as e:
        fftim3d.calc_cost(kw["iin"], **bad)
    assert e.value.code == -6


def test_batch_packing_reports_the_failing_problem_without_device(crescent32, closure40):
    """Problems of a batch are packed in parallel on the host; a bad problem
    in the middle of the batch fails the whole creation with its own error
    code and message, before any device is touched."""
    from smili_b200 import _lib
    good = make_kw(crescent32)
    bad = dict(make_kw(closure40))
    bad["varamp"] = np.asarray(bad["varamp"]).copy()
    bad["varamp"][3] = -1.0  # a non-positive variance
    probs = [_lib.Problem(good), _lib.Problem(good), _lib.Problem(bad), _lib.Problem(good)]
    with pytest.raises(_lib.SmiliError) as e:
        _lib.Batch(probs, niter=5, options=_lib.make_options(64, 1e-6))
    assert e.value.code == -2
    assert "varia" in str(e.value).lower()
