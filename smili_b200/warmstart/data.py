"""Training and evaluation data of the learned warm start.

A pair is (dirty image, converged reconstruction) for one synthetic
observation (``synth.warmstart_problem``):

- the dirty image is the negative gradient of the complex-visibility
  chi-square at the zero image (the natural-weighted back-projection of the
  data, in the solver's own conventions), computed for a whole set in one
  batched evaluation on the GPU;
- the reconstruction is the plain method's result: L-BFGS-B from the
  Gaussian prior, run by the batched solver in FP64.

Images are (ny, nx) arrays in Jy/pixel; the network sees the dirty image
scaled to max |.| = 1 and predicts the reconstruction scaled to max 1.

A warm-started solve uses exactly the plain solve's kwargs (same
normalisation, data and regularizer weights); only the initial pixel
vector changes, so both solves minimise the same objective.
"""
from __future__ import annotations

import numpy as np

from .. import _lib, synth
from ..imaging.lbfgs import prepare_imaging


def make_set(seeds, niter=1000, nx=128):
    """[(kw, truth, tf)] for the given seeds (fftim2d kwargs, truth image,
    prior flux).  Model visibilities come from the library's NUFFT."""
    out = []
    for s in seeds:
        obs = synth.warmstart_problem(int(s), nx=nx, niter=niter, model=synth.nufft_model)
        kw, _ = prepare_imaging(obs.image, vistable=obs.vistable, bstable=obs.bstable, niter=niter,
                                **obs.reg)
        out.append((kw, obs.truth, obs.totalflux))
    return out


def to_grid(kw, x):
    """Pixel vector (scaled units) -> (ny, nx) image in Jy/pixel."""
    img = np.zeros((int(kw["ny"]), int(kw["nx"])))
    img[np.asarray(kw["yidx"]) - 1, np.asarray(kw["xidx"]) - 1] = np.asarray(x) / float(kw["inormfactr"])
    return img


def from_grid(kw, img):
    """(ny, nx) image in Jy/pixel -> pixel vector in the kwargs' scaled units."""
    return np.ascontiguousarray(np.asarray(img)[np.asarray(kw["yidx"]) - 1, np.asarray(kw["xidx"]) - 1]
                                * float(kw["inormfactr"]), dtype=np.float64)


def dirty_images(kws, device=0, chunk=1024, kernel_ms=None):
    """Normalised dirty images (N, ny, nx): -grad chi2_fcv at x = 0, max |.| 1.
    ``kernel_ms`` (a list) receives the device time of each evaluation launch."""
    out = []
    for c0 in range(0, len(kws), chunk):
        part = kws[c0:c0 + chunk]
        probs = []
        for kw in part:
            k = dict(kw)
            k["iin"] = np.zeros_like(np.asarray(kw["iin"], dtype=np.float64))
            k["iscp"] = False
            for name in ("l1_l", "tv_l", "tsv_l", "kl_l", "gs_l", "tfd_l", "cen_l", "sm_l"):
                k[name] = -1.0
            probs.append(k)
        b = _lib.Batch(probs, niter=0, options=_lib.make_options(64, 1e-6, device=device))
        ms = b.run(fg_only=1)
        if kernel_ms is not None:
            kernel_ms.append(ms)
        for p, kw in enumerate(part):
            g = b.fetch(p)[2]
            d = -to_grid(kw, g)
            out.append(d / max(np.max(np.abs(d)), 1e-300))
        b.close()
    return np.asarray(out, np.float32)


def solve(kws, niter, precision=64, targets=None, device=0, x0=None, chunk=1024, ctas_per_problem=0):
    """Batched L-BFGS-B solves (``chunk`` problems per launch); x0 (list of
    pixel vectors in scaled units) replaces the kwargs' initial images;
    ``ctas_per_problem`` fixes the CTA group size (0: automatic).
    Returns (x list, info list, cost array, traces, total kernel ms)."""
    xs, infos, costs, traces, ms = [], [], [], [], 0.0
    for c0 in range(0, len(kws), chunk):
        probs = []
        for i in range(c0, min(len(kws), c0 + chunk)):
            k = dict(kws[i])
            if x0 is not None:
                k["iin"] = x0[i]
            probs.append(k)
        b = _lib.Batch(probs, niter=niter, options=_lib.make_options(precision, 1e-6, ctas_per_problem,
                                                                     device=device))
        if targets is not None:
            b.set_targets(np.asarray(targets)[c0:c0 + len(probs)])
        ms += b.run()
        for p in range(len(probs)):
            x, t, _, info = b.fetch(p)
            xs.append(x.copy())
            infos.append(info)
            costs.append(t["cost"])
            traces.append(b.trace(p, niter + 2))
        b.close()
    return xs, infos, np.asarray(costs), traces, ms


def warm_init(kw, pred, tf):
    """Starting pixel vector from a network output (max-1 scale): ReLU,
    rescaled to the prior's total flux; the Gaussian prior when the output
    has no positive pixel."""
    img = np.maximum(np.asarray(pred, np.float64), 0.0)
    s = img.sum()
    if not np.isfinite(s) or s <= 0:
        return np.asarray(kw["iin"], dtype=np.float64).copy()
    return from_grid(kw, img * (tf / s))


def nrmse(img, truth):
    return float(np.linalg.norm(img - truth) / np.linalg.norm(truth))
