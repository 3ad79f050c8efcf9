"""CUDA path against the CPU oracle, through the C ABI.

FP64 mode with a tight NUFFT tolerance (1e-12) must match the oracle's exact
or tight-tolerance result to 1e-9 relative (objective) and 1e-8 relative
(gradient, max-norm).  At the reference's own tolerance (1e-6) both sides
use the same kernel width, shape parameter, fine grid and deconvolution, so
they agree to rounding: 1e-10 (objective) and 1e-9 (gradient).
FP32 mode is bounded against the FP64 oracle (see test_calc_cost_fp32_bound).
L-BFGS-B trajectories agree per iteration: the first 10 iterations to 1e-9
relative (1e-7 with closure terms), the first 50 to 2e-5 (parallel reductions and atomic spreading change
the rounding, which the iteration then amplifies slowly).
"""
import numpy as np
import pytest

from conftest import make_kw

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from smili_b200 import _lib
    return _lib


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("nx,ny", [(32, 32), (24, 40), (96, 96)])
def test_nufft_fwd_matches_dft(oracle, nx, ny):
    from smili_b200.fortlib import fftlib
    rng = np.random.default_rng(nx)
    img = rng.standard_normal((ny, nx))
    u, v = rng.uniform(-2.5, 2.5, 700), rng.uniform(-2.5, 2.5, 700)
    ex = oracle.nufft2d2(u, v, img, 0)
    vr, vi = fftlib.nufft_fwd_real(u, v, img.T, nufft_eps=1e-12)  # (nx, ny) Fortran-order image
    assert _rel(vr + 1j * vi, ex) < 1e-10
    vr, vi = fftlib.nufft_fwd_real(u, v, img.T, precision=32, nufft_eps=1e-6)
    assert _rel(vr + 1j * vi, ex) < 2e-5


@pytest.mark.parametrize("nx,ny", [(32, 32), (40, 24)])
def test_nufft_adj_matches_dft(oracle, nx, ny):
    from smili_b200.fortlib import fftlib
    rng = np.random.default_rng(nx + 1)
    u, v = rng.uniform(-2.5, 2.5, 500), rng.uniform(-2.5, 2.5, 500)
    c = rng.standard_normal(500) + 1j * rng.standard_normal(500)
    ex = oracle.nufft2d1(u, v, c, nx, ny, 0).real.reshape(-1)
    got = fftlib.nufft_adj_real1d(u, v, c.real, c.imag, nx, ny, nufft_eps=1e-12)
    assert _rel(got, ex) < 1e-10


def _band(u, nf, eps):
    """Band width in fine-grid cells that the library computes for these
    coordinates (kernel width w = ceil(log10(10 / eps)))."""
    w = int(np.ceil(np.log10(10.0 / eps)))
    l = np.ceil(np.asarray(u) * nf / (2 * np.pi) - 0.5 * w)
    return int(l.max() - l.min() + w)


@pytest.mark.parametrize("transform", [1, 2])
@pytest.mark.parametrize("nx,ny", [(32, 32), (40, 24), (96, 96)])
def test_nufft_transform_paths_match_dft(oracle, nx, ny, transform):
    """Both fine-grid paths (radix passes, dense twiddle products) against
    the exact transform, in both directions and precisions.  The points lie
    in |u|, |v| < 0.4 rad/pixel, so the band is narrow enough for the dense
    path (at most 64 x 64 cells, 2048 in all)."""
    from smili_b200.fortlib import fftlib
    rng = np.random.default_rng(nx + 7 * ny)
    img = rng.standard_normal((ny, nx))
    u, v = rng.uniform(-0.4, 0.4, 900), rng.uniform(-0.4, 0.4, 900)
    nf1, nf2 = 2 * nx, 2 * ny  # next235even(2n) for these sizes
    b1, b2 = _band(u, nf1, 1e-12), _band(v, nf2, 1e-12)
    assert b1 <= 64 and b2 <= 64 and b1 * b2 <= 2048
    ex = oracle.nufft2d2(u, v, img, 0)
    vr, vi = fftlib.nufft_fwd_real(u, v, img.T, nufft_eps=1e-12, transform=transform)
    assert _rel(vr + 1j * vi, ex) < 1e-10
    vr, vi = fftlib.nufft_fwd_real(u, v, img.T, precision=32, nufft_eps=1e-6, transform=transform)
    assert _rel(vr + 1j * vi, ex) < 2e-5
    c = rng.standard_normal(u.size) + 1j * rng.standard_normal(u.size)
    ex1 = oracle.nufft2d1(u, v, c, nx, ny, 0).real.reshape(-1)
    got = fftlib.nufft_adj_real1d(u, v, c.real, c.imag, nx, ny, nufft_eps=1e-12, transform=transform)
    assert _rel(got, ex1) < 1e-10
    got = fftlib.nufft_adj_real1d(u, v, c.real, c.imag, nx, ny, precision=32, nufft_eps=1e-6,
                                  transform=transform)
    assert _rel(got, ex1) < 2e-5


@pytest.mark.parametrize("prec,tol", [(64, 1e-12), (32, 1e-5)])
def test_calc_cost_transform_paths_agree(oracle, closure40, lib, prec, tol):
    """One evaluation of the closure-term problem through the radix passes
    and through the dense twiddle products: the same objective and gradient
    (FP64: roundoff; FP32: both within FP32 accuracy), and the oracle's."""
    kw = make_kw(closure40)
    nf = 2 * int(kw["nx"])
    b1, b2 = _band(kw["u"], nf, 1e-6), _band(kw["v"], nf, 1e-6)
    assert b1 <= 64 and b2 <= 64 and b1 * b2 <= 2048, (b1, b2)
    x = np.asarray(kw["iin"]) * np.random.default_rng(4).uniform(0.5, 1.5, np.size(kw["iin"]))
    prob = lib.Problem(dict(kw, iin=x))
    out = []
    for tr in (1, 2):
        bt = lib.Batch([prob], niter=1, options=lib.make_options(prec, 1e-6, transform=tr))
        bt.run(fg_only=1)
        _, t, g, _ = bt.fetch(0)
        bt.close()
        out.append((t["cost"], g))
    assert abs(out[1][0] - out[0][0]) <= tol * abs(out[0][0])
    assert np.max(np.abs(out[1][1] - out[0][1])) <= 10 * tol * np.max(np.abs(out[0][1]))
    t_o, g_o = oracle.calc_cost(kw, x, eps=0.0)
    assert abs(out[1][0] - t_o["cost"]) <= 1e-5 * abs(t_o["cost"])


def test_nufft_band_localised_points(oracle):
    """VLBI-like coverage: all points within a narrow band of the fine grid."""
    from smili_b200.fortlib import fftlib
    rng = np.random.default_rng(5)
    img = rng.random((64, 64))
    u, v = rng.uniform(-0.3, 0.3, 2000), rng.uniform(-0.25, 0.25, 2000)
    ex = oracle.nufft2d2(u, v, img, 0)
    vr, vi = fftlib.nufft_fwd_real(u, v, img.T, nufft_eps=1e-12)
    assert _rel(vr + 1j * vi, ex) < 1e-10


REG_ALL = dict(l1_lambda=1.0, tsv_lambda=1.0, tv_lambda=0.5, kl_lambda=0.1, gs_lambda=0.1,
               tfd_lambda=1.0, cen_lambda=0.1, sm_lambda=0.1, sm_maj=30.0, sm_min=20.0, sm_phi=30.0)


@pytest.mark.parametrize("case", ["fcv_cp_allreg", "amp_cp_ca"])
def test_calc_cost_fp64_matches_oracle(oracle, crescent32, closure40, case):
    from smili_b200.fortlib import fftim2d
    kw = make_kw(crescent32, **REG_ALL) if case == "fcv_cp_allreg" else make_kw(closure40)
    rng = np.random.default_rng(11)
    x = kw["iin"] * (1 + 0.3 * rng.random(kw["iin"].size))
    t_ref, g_ref = oracle.calc_cost(kw, x, eps=1e-12)
    t_gpu, g_gpu = fftim2d.calc_cost(x, nufft_eps=1e-12, **kw)
    for k in ["cost", "chisq", "reg", "chisqfcv", "chisqamp", "chisqcp", "chisqca", "l1_cost",
              "tv_cost", "tsv_cost", "kl_cost", "gs_cost", "tfd_cost", "cen_cost", "sm_cost"]:
        assert abs(t_gpu[k] - t_ref[k]) <= 1e-9 * max(abs(t_ref[k]), 1e-12), k
    assert _rel(g_gpu, g_ref) < 1e-8
    # at the reference's own tolerance (wrapfinufft.f90:8)
    t6, g6 = fftim2d.calc_cost(x, nufft_eps=1e-6, **kw)
    t6r, g6r = oracle.calc_cost(kw, x, eps=1e-6)
    assert abs(t6["cost"] - t6r["cost"]) <= 1e-10 * abs(t6r["cost"])
    assert _rel(g6, g6r) < 1e-9


@pytest.mark.parametrize("case", ["fcv_cp_allreg", "amp_cp_ca"])
def test_calc_cost_fp32_bound(oracle, crescent32, closure40, case):
    """FP32 mode (NUFFT tolerance 1e-6) against the exact FP64 objective: the
    objective within 1e-4 relative, and the gradient error no larger than
    twice the error that the reference's own FP64 NUFFT at ffteps = 1e-6
    makes (closure terms divide by |V|^2, so near-null visibilities amplify
    any transform error in both)."""
    from smili_b200.fortlib import fftim2d
    kw = make_kw(crescent32, **REG_ALL) if case == "fcv_cp_allreg" else make_kw(closure40)
    x = kw["iin"]
    t_ref, g_ref = oracle.calc_cost(kw, x, eps=1e-12)
    _, g_ref6 = oracle.calc_cost(kw, x, eps=1e-6)
    t32, g32 = fftim2d.calc_cost(x, precision=32, nufft_eps=1e-6, **kw)
    assert abs(t32["cost"] - t_ref["cost"]) <= 1e-4 * abs(t_ref["cost"])
    assert _rel(g32, g_ref) <= 2.0 * _rel(g_ref6, g_ref) + 1e-4


def test_solve_per_iteration_matches_oracle(oracle, crescent32, lib):
    """First 50 L-BFGS-B iterations: objective per iteration (FP64)."""
    kw = make_kw(crescent32, niter=50)
    b = lib.Batch([kw], niter=50, options=lib.make_options(64, 1e-12))
    b.run()
    x, terms, _, info = b.fetch(0)
    tr = b.trace(0, 52)
    b.close()
    iout, tref, iref = oracle.imaging(kw, eps=1e-12)
    trr = iref["trace"]
    assert info["niter"] == iref["niter"] == 51
    np.testing.assert_allclose(tr[:10], trr[:10], rtol=1e-9)
    np.testing.assert_allclose(tr[:50], trr[:50], rtol=2e-5)
    assert abs(terms["cost"] - tref["cost"]) <= 1e-4 * abs(tref["cost"])


def _window(n, r):
    yy, xx = np.mgrid[:n, :n]
    return (xx - n // 2) ** 2 + (yy - n // 2) ** 2 < r * r


@pytest.mark.parametrize("variant", ["m1", "m3", "m6", "unbounded", "window"])
def test_solve_variants_match_oracle(oracle, crescent32, lib, variant):
    """The optimiser's other settings against the oracle, per iteration (FP64):
    L-BFGS-B memories 1, 3 and 6 (the largest the device accepts), no
    non-negativity bound (the unconstrained path: no Cauchy search), and a
    windowed pixel set (a disc of 13 pixels radius in the 32 x 32 grid)."""
    over = {"niter": 20}
    if variant == "window":
        over["imregion"] = _window(32, 13)
    kw = make_kw(crescent32, **over)
    if variant.startswith("m"):
        kw["m"] = int(variant[1:])
    if variant == "unbounded":
        kw["nonneg"] = False
    if variant == "window":
        assert kw["npix"] == int(_window(32, 13).sum()) < 32 * 32
    b = lib.Batch([kw], niter=20, nonneg=kw["nonneg"], m=kw["m"], options=lib.make_options(64, 1e-12))
    b.run()
    _, terms, _, info = b.fetch(0)
    tr = b.trace(0, 22)
    b.close()
    _, tref, iref = oracle.imaging(kw, eps=1e-12)
    assert info["niter"] == iref["niter"]
    np.testing.assert_allclose(tr[:10], iref["trace"][:10], rtol=1e-9)
    np.testing.assert_allclose(tr[:20], iref["trace"][:20], rtol=2e-5)


def test_solve_closure_terms_matches_oracle(oracle, closure40, lib):
    kw = make_kw(closure40, niter=40)
    b = lib.Batch([kw], niter=40, options=lib.make_options(64, 1e-12))
    b.run()
    _, terms, _, info = b.fetch(0)
    tr = b.trace(0, 42)
    b.close()
    _, tref, iref = oracle.imaging(kw, eps=1e-12)
    # closure phases/amplitudes (atan2, log of |V|) amplify rounding more
    np.testing.assert_allclose(tr[:10], iref["trace"][:10], rtol=1e-7)
    np.testing.assert_allclose(tr[:30], iref["trace"][:30], rtol=2e-5)
    # after 41 unconverged iterations the two trajectories have drifted apart
    assert abs(terms["cost"] - tref["cost"]) <= 2e-2 * abs(tref["cost"])


def test_fftim2d_imaging_dropin(oracle, crescent32):
    from smili_b200.fortlib import fftim2d
    kw = make_kw(crescent32, niter=30)
    out = fftim2d.imaging(nufft_eps=1e-12, **kw)
    assert len(out) == 16 and out[0].shape == (kw["npix"],)
    iout, tref, _ = oracle.imaging(kw, eps=1e-12)
    assert abs(out[15] - tref["cost"]) <= 1e-4 * abs(tref["cost"])
    assert np.abs(out[0] - iout).max() <= 1e-2 * np.abs(iout).max()


def test_batched_equals_single(crescent32, closure40, lib):
    kws = [make_kw(crescent32, niter=20), make_kw(closure40, niter=20), make_kw(crescent32, niter=10)]
    singles = []
    for kw in kws:
        b = lib.Batch([kw], niter=kw["niter"], options=lib.make_options(64, 1e-9))
        b.run()
        singles.append(b.fetch(0))
        b.close()
    b = lib.Batch(kws, niter=[k["niter"] for k in kws], options=lib.make_options(64, 1e-9))
    b.run()
    for p, s in enumerate(singles):
        x, t, _, info = b.fetch(p)
        assert info["niter"] == s[3]["niter"]
        assert abs(t["cost"] - s[1]["cost"]) <= 1e-9 * abs(s[1]["cost"])
    b.close()


def test_set_start_equals_packing(crescent32, lib):
    """A device-resident batch restarted from a new image (smili_batch_set_start)
    solves exactly as a batch packed with that image."""
    kw = make_kw(crescent32, niter=10)
    x1 = np.asarray(kw["iin"]) * np.random.default_rng(3).uniform(0.5, 1.5, np.size(kw["iin"]))
    b = lib.Batch([kw], niter=10, options=lib.make_options(64, 1e-9))
    b.run()
    b.set_start(0, x1)
    b.run()
    _, t, _, i = b.fetch(0)
    b.close()
    c = lib.Batch([dict(kw, iin=x1)], niter=10, options=lib.make_options(64, 1e-9))
    c.run()
    _, t2, _, i2 = c.fetch(0)
    c.close()
    assert i["niter"] == i2["niter"]
    assert abs(t["cost"] - t2["cost"]) <= 1e-9 * abs(t2["cost"])
    with pytest.raises(lib.SmiliError):
        b2 = lib.Batch([kw], niter=1, options=lib.make_options(64, 1e-9))
        try:
            b2.set_start(0, np.full(np.size(kw["iin"]), np.nan))
        finally:
            b2.close()


def test_set_niter_equals_packing(crescent32, lib):
    """Lowered iteration caps (smili_batch_set_niter) solve as a batch packed
    with them; caps above the packed ones are refused; None restores them."""
    kw = make_kw(crescent32, niter=12)
    b = lib.Batch([kw], niter=12, options=lib.make_options(64, 1e-9))
    b.set_niter(5)
    b.run()
    _, t, _, i = b.fetch(0)
    c = lib.Batch([dict(kw, niter=5)], niter=5, options=lib.make_options(64, 1e-9))
    c.run()
    _, t2, _, i2 = c.fetch(0)
    c.close()
    assert i["niter"] == i2["niter"] == 6
    assert abs(t["cost"] - t2["cost"]) <= 1e-9 * abs(t2["cost"])
    with pytest.raises(lib.SmiliError):
        b.set_niter(13)
    b.set_niter(None)
    b.run()
    assert b.fetch(0)[3]["niter"] == 13
    b.close()


def test_device_warm_start_matches_host(crescent32, lib):
    """smili_batch_images, smili_batch_set_starts_from_images and
    smili_batch_reset_starts do on the device what the host warm start does
    with fetch, to_grid, normalise, warm_init and set_start."""
    import torch
    from smili_b200.warmstart import closure, data
    kw = make_kw(crescent32, niter=8)
    rng = np.random.default_rng(5)
    kws = [dict(kw, iin=np.asarray(kw["iin"]) * rng.uniform(0.5, 1.5, np.size(kw["iin"]))) for _ in range(3)]
    opts = lib.make_options(64, 1e-9)
    b = lib.Batch(kws, niter=8, options=opts)
    b.run()
    xs = [b.fetch(p)[0] for p in range(3)]
    nx, ny = int(kw["nx"]), int(kw["ny"])
    img = torch.zeros((3, ny, nx), dtype=torch.float32, device="cuda")
    b.images(img)
    want = closure.normalise([data.to_grid(k, x) for k, x in zip(kws, xs)])
    np.testing.assert_allclose(img.cpu().numpy(), want, rtol=1e-6, atol=1e-7)
    pred = rng.standard_normal((3, ny, nx)).astype(np.float32)
    pred[2] = -np.abs(pred[2])  # no positive cell: the current image is kept
    keep = np.array([False, True, False])
    b.set_starts_from_images(torch.as_tensor(pred, device="cuda"), keep=keep)
    starts = [xs[p] if keep[p] else closure.warm_init(kws[p], pred[p], xs[p]) for p in range(3)]
    b.run()
    c = lib.Batch([dict(k, iin=s) for k, s in zip(kws, starts)], niter=8, options=opts)
    c.run()
    for p in range(3):
        _, t, _, i = b.fetch(p)
        _, t2, _, i2 = c.fetch(p)
        assert i["niter"] == i2["niter"]
        assert abs(t["cost"] - t2["cost"]) <= 1e-8 * abs(t2["cost"])
    c.close()
    b.reset_starts()
    b.run()
    d = lib.Batch(kws, niter=8, options=opts)
    d.run()
    for p in range(3):
        _, t, _, i = b.fetch(p)
        _, t2, _, i2 = d.fetch(p)
        assert i["niter"] == i2["niter"]
        assert abs(t["cost"] - t2["cost"]) <= 1e-8 * abs(t2["cost"])
    d.close()
    with pytest.raises(ValueError):
        b.images(torch.zeros((2, ny, nx), dtype=torch.float32, device="cuda"))
    b.close()


def test_invalid_inputs_raise(crescent32, lib):
    kw = make_kw(crescent32, niter=5)
    bad = dict(kw)
    bad["varfcv"] = kw["varfcv"].copy()
    bad["varfcv"][3] = 0.0
    with pytest.raises(lib.SmiliError) as e:
        lib.Batch([bad], niter=5)
    assert e.value.code == -2


def test_target_stop(crescent32, lib):
    """A solve with an objective target stops at the first completed
    iteration whose cost is at or below it; without a target it runs on."""
    kw = make_kw(crescent32, niter=40)
    opts = lib.make_options(64, 1e-9)
    b = lib.Batch([kw, kw], niter=40, options=opts)
    b.run()
    tr = b.trace(0, 42)
    assert b.fetch(0)[3]["task"] == lib.TASK_STOP
    k = 15
    assert tr[k] < tr[k - 1]
    target = 0.5 * (tr[k - 1] + tr[k])  # robust to run-to-run rounding
    first = int(np.argmax(tr <= target))
    assert first == k
    b.set_targets([target, -np.inf])
    b.run()
    _, t0, _, i0 = b.fetch(0)
    _, t1, _, i1 = b.fetch(1)
    assert i0["task"] == lib.TASK_TARGET
    assert i0["niter"] == first + 1
    assert t0["cost"] <= target
    assert i1["task"] == lib.TASK_STOP and i1["niter"] == 41
    b.set_targets(None)
    b.run()
    assert b.fetch(0)[3]["task"] == lib.TASK_STOP
    b.close()


def test_survey_batch_mixed_sizes(lib):
    """The survey configuration: problems of different image sizes (64..256),
    visibility counts and regularizer weights in one launch give the same
    solves as one launch per problem (FP64, 10 iterations)."""
    from smili_b200 import synth
    kws = [make_kw(synth.survey_problem(i, seed=3, niter=10, model=synth.nufft_model)) for i in range(8)]
    assert len({int(k["nx"]) for k in kws}) >= 3
    b = lib.Batch(kws, niter=10, options=lib.make_options(64, 1e-9))
    b.run()
    for p, kw in enumerate(kws):
        s = lib.Batch([kw], niter=10, options=lib.make_options(64, 1e-9))
        s.run()
        _, ts, _, is_ = s.fetch(0)
        s.close()
        _, tb, _, ib = b.fetch(p)
        assert ib["niter"] == is_["niter"]
        assert abs(tb["cost"] - ts["cost"]) <= 1e-6 * abs(ts["cost"]), (p, tb["cost"], ts["cost"])
    b.close()


def test_spread_bin16_equals_bin8(oracle, closure40, lib):
    """16-cell spreading tiles give the same evaluation as 8-cell tiles (and
    as the oracle); the autotuner returns one of its candidates.  FP64 at
    nufft_eps 1e-6 (kernel width 7): eight warp subgrids of 22 x 22 complex
    values and their weight tables (about 69 KB) fit the 96 KB of staging,
    so the 16-cell tiles are really used."""
    from smili_b200 import autotune
    kw = make_kw(closure40)
    x = np.asarray(kw["iin"]) * np.random.default_rng(2).uniform(0.5, 1.5, np.size(kw["iin"]))
    prob = lib.Problem(dict(kw, iin=x))
    out = []
    for b in (8, 16):
        bt = lib.Batch([prob], niter=1, options=lib.make_options(64, 1e-6, spread_bin=b))
        bt.run(fg_only=1)
        _, t, g, _ = bt.fetch(0)
        bt.close()
        out.append((t["cost"], g))
    # the same sums in another order: FP64 roundoff only
    assert abs(out[1][0] - out[0][0]) <= 1e-12 * abs(out[0][0])
    assert np.max(np.abs(out[1][1] - out[0][1])) <= 1e-10 * np.max(np.abs(out[0][1]))
    # against the exact transform: the NUFFT tolerance
    t_o, g_o = oracle.calc_cost(kw, x, eps=0.0)
    assert abs(out[1][0] - t_o["cost"]) <= 1e-5 * abs(t_o["cost"])
    assert np.max(np.abs(out[1][1] - g_o)) <= 1e-4 * np.max(np.abs(g_o))
    r = autotune.tune([kw] * 4, 32, niter=3, repeats=1, cands=[(1, 8), (2, 16)])
    assert (r["ctas_per_problem"], r["spread_bin"]) in [(1, 8), (2, 16)] and len(r["table"]) == 2
