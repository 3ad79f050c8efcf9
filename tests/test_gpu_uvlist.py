"""The uv list on the GPU (smili_get_uvlist) against numpy's: the same
distinct points bit for bit, in the same order, and the same signed indices."""
import numpy as np
import pandas as pd
import pytest

from conftest import make_kw

pytestmark = pytest.mark.gpu


def _same(host, dev):
    for a, b in zip(host, dev):
        assert a.shape == b.shape
        assert np.array_equal(a, b)
        if a.dtype.kind == "f":
            assert np.array_equal(np.signbit(a), np.signbit(b))  # same representative of +-0


def _tables(rng, n, span, dup=0.0):
    """A vis table and a closure-phase table whose points repeat, include v < 0,
    v = -0, u = +-0 and exact conjugates."""
    grid = rng.integers(-span, span + 1, (n, 2)).astype(np.float64) * 0.5
    grid[rng.random(n) < 0.05] *= 0.0  # zeros, some of them -0 after sign flips below
    grid[rng.random(n) < 0.05, 1] = -0.0
    if dup:
        k = rng.random(n) < dup
        grid[k] = -grid[k][::-1]  # conjugates of other points
    vis = pd.DataFrame({"u": grid[:, 0], "v": grid[:, 1]})
    m = max(1, n // 3)
    bs = pd.DataFrame({c: rng.choice(grid[:, i % 2], m) * (-1) ** rng.integers(0, 2, m)
                       for i, c in enumerate(["u12", "v12", "u23", "v23", "u31", "v31"])})
    return vis, bs


@pytest.mark.parametrize("n", [1, 2, 7, 682, 683, 2048, 5000])
def test_device_uvlist_equals_host_edge_sizes(n):
    from smili_b200.uvdata import tools
    rng = np.random.default_rng(n)
    vis, bs = _tables(rng, n, span=6, dup=0.2)
    host = tools.get_uvlist(fcvtable=vis, bstable=bs)
    dev = tools.get_uvlist(fcvtable=vis, bstable=bs, device=0)
    _same(host, dev)


def test_device_uvlist_equals_host_at_workload_size():
    """The 256x256 / 1e5-visibility workload's tables (amplitudes, closure
    phases, log closure amplitudes): ~6.5e5 stacked points, so the sort runs
    its global merge steps."""
    from smili_b200 import synth
    from smili_b200.uvdata import tools
    obs = synth.precision_path(seed=1000, niter=10, model=lambda truth, img, u, v: np.ones(len(u), complex))
    args = dict(amptable=obs.amptable, bstable=obs.bstable, catable=obs.catable)
    host = tools.get_uvlist(**args)
    dev = tools.get_uvlist(device=0, **args)
    assert len(obs.amptable) + 3 * len(obs.bstable) + 4 * len(obs.catable) > 4 * 2048 * 16
    _same(host, dev)


def test_prepare_imaging_with_device_uvlist(closure40):
    from smili_b200.imaging.lbfgs import prepare_imaging
    o = closure40
    kw0 = make_kw(o)
    kw1, _ = prepare_imaging(o.image, amptable=o.amptable, bstable=o.bstable, catable=o.catable, niter=50,
                             uvlist_device=0, **o.reg)
    for k, v in kw0.items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, kw1[k]), k
