"""Failure detection on the device without a GPU fault: every group-barrier
wait of the persistent kernel is bounded.  A launch in which one CTA of each
group never arrives must end with SMILI_ERR_TIMEOUT after the short test
limit (not hang), and the batch and the context stay usable."""
import numpy as np
import pytest

from conftest import make_kw

pytestmark = pytest.mark.gpu


def test_wait_that_nothing_releases_times_out_and_batch_recovers(crescent32):
    from smili_b200 import _lib
    kw = make_kw(crescent32, niter=5)
    ref = _lib.Batch([kw, kw], niter=5, options=_lib.make_options(64, 1e-9, 2))
    ref.run()
    cost_ref = ref.fetch(1)[1]["cost"]
    ref.close()
    b = _lib.Batch([kw, kw], niter=5, options=_lib.make_options(64, 1e-9, 2))  # 2 CTAs per problem
    for _ in range(2):
        with pytest.raises(_lib.SmiliError) as e:
            b.run(3)
        assert e.value.code == -5  # SMILI_ERR_TIMEOUT
    b.run()  # the same batch solves normally afterwards
    _, t, _, info = b.fetch(1)
    b.close()
    assert info["task"] != 6 and np.isfinite(t["cost"])
    assert abs(t["cost"] - cost_ref) <= 1e-6 * abs(cost_ref)  # atomic spreading: roundoff-level differences


def test_one_cta_per_problem_has_no_barrier_to_miss(crescent32):
    from smili_b200 import _lib
    kw = make_kw(crescent32, niter=5)
    b = _lib.Batch([kw], niter=5, options=_lib.make_options(64, 1e-9, 1))
    b.run(3)  # G == 1: block barriers only, nothing to time out
    b.close()


def test_non_finite_problem_is_contained(oracle, closure40):
    """A problem whose objective is not finite (closure amplitudes of an
    all-zero start image: log |V| = -inf) ends as the oracle's does, and the
    problems beside it in the batch are unaffected."""
    from smili_b200 import _lib
    kw = make_kw(closure40, niter=20)
    bad = dict(kw, iin=np.zeros_like(kw["iin"]))
    _, tref, iref = oracle.imaging(bad, eps=1e-12)
    assert not np.isfinite(tref["cost"])
    single = _lib.Batch([kw], niter=20, options=_lib.make_options(64, 1e-12))
    single.run()
    good_cost = single.fetch(0)[1]["cost"]
    single.close()
    b = _lib.Batch([kw, bad, kw], niter=20, options=_lib.make_options(64, 1e-12))
    b.run()
    _, tb, _, ib = b.fetch(1)
    assert not np.isfinite(tb["cost"])
    assert ib["task"] == iref["task"] and ib["niter"] == iref["niter"]
    for p in (0, 2):
        _, t, _, _ = b.fetch(p)
        assert abs(t["cost"] - good_cost) <= 1e-6 * abs(good_cost)
    b.close()
