import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


def make_kw(obs, **over):
    """fftim2d.imaging kwargs for a synthetic observation."""
    from smili_b200.imaging.lbfgs import prepare_imaging
    args = dict(vistable=obs.vistable, amptable=obs.amptable, bstable=obs.bstable,
                catable=obs.catable, niter=obs.niter)
    args.update(obs.reg)
    args.update(over)
    kw, _ = prepare_imaging(obs.image, **args)
    return kw


@pytest.fixture(scope="session")
def crescent32():
    from smili_b200 import synth
    return synth.small_crescent(seed=0, nx=32, niter=50)


@pytest.fixture(scope="session")
def closure40():
    """amplitudes + closure phases + log closure amplitudes on a 40x40 grid"""
    from smili_b200 import synth
    return synth.precision_path(seed=7, nx=40, nst=7, hours=4.0, scan_s=900.0, niter=50)
