"""The learned warm start for data without absolute phases.

Amplitudes, closure phases and log closure amplitudes (the 256x256
precision-path workload, ``synth.precision_path``) carry no absolute
visibility phase, so there is no dirty image to start from.  The proposal's
input is instead the image after ``K`` FP32 L-BFGS-B iterations from the
Gaussian prior: it already holds the source's position and rough shape, and
the network maps it to the plain method's converged image.

- Training pairs: (image after K FP32 iterations, the plain FP64 solve's
  final image), both scaled to max 1, for seeded precision-path problems
  disjoint from the benchmark's seeds (the benchmark uses 1000..1015).
- A warm-started solve: K FP32 iterations from the prior, the network's
  proposal (ReLU, rescaled to the K-iteration image's total flux), then the
  same L-BFGS-B with the remaining iteration budget.  The plain FP64 solve's
  final cost stays the judge: a solve counts when it reaches it.

    python -m smili_b200.warmstart.closure --ntrain 2048 --workers 8 --out unet_closure256.npz
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from .. import _lib, synth
from ..imaging.lbfgs import prepare_imaging
from . import data
from .train import augment
from .unet import UNet

K_DEFAULT = 50


def make_set(seeds, niter=1000):
    """[(kw, truth, tf)] for precision-path seeds (model visibilities from
    the library's NUFFT)."""
    out = []
    for s in seeds:
        obs = synth.precision_path(seed=int(s), niter=niter, model=synth.nufft_model)
        kw, _ = prepare_imaging(obs.image, amptable=obs.amptable, bstable=obs.bstable, catable=obs.catable,
                                niter=niter, **obs.reg)
        out.append((kw, obs.truth, obs.totalflux))
    return out


def _make_chunk(args):
    seeds, niter = args
    return make_set(seeds, niter)


def make_set_parallel(seeds, niter=1000, workers=1):
    """``make_set`` over host worker processes (started with spawn; each
    computes its model visibilities on the GPU)."""
    seeds = list(seeds)
    if workers <= 1 or len(seeds) < 2 * workers:
        return make_set(seeds, niter)
    import multiprocessing as mp
    parts = [seeds[i::workers] for i in range(workers)]
    with mp.get_context("spawn").Pool(workers) as pool:
        done = pool.map(_make_chunk, [(part, niter) for part in parts])
    by_seed = {}
    for part, res in zip(parts, done):
        by_seed.update(zip(part, res))
    return [by_seed[s] for s in seeds]


def normalise(imgs):
    imgs = np.asarray(imgs, np.float32)
    return imgs / np.maximum(imgs.reshape(len(imgs), -1).max(axis=1), 1e-30)[:, None, None]


def early_images(kws, K=K_DEFAULT, device=0, ctas_per_problem=0, targets=None):
    """K FP32 iterations from each problem's prior in one batched launch:
    (pixel vectors, images scaled to max 1, infos, device ms)."""
    xs, infos, _, _, ms = data.solve(kws, K, 32, targets=targets, device=device,
                                     ctas_per_problem=ctas_per_problem)
    imgs = normalise([data.to_grid(kw, x) for kw, x in zip(kws, xs)])
    return xs, imgs, infos, ms


def warm_init(kw, pred, x_early):
    """Starting pixel vector: the network output (max-1 scale), ReLU'd and
    rescaled to the total flux of the K-iteration image; that image itself
    when the output has no positive pixel."""
    img = np.maximum(np.asarray(pred, np.float64), 0.0)
    s, f = img.sum(), float(np.sum(x_early))
    if not np.isfinite(s) or s <= 0 or f <= 0:
        return np.asarray(x_early, dtype=np.float64).copy()
    return data.from_grid(kw, img * (f / s / float(kw["inormfactr"])))


def train(net, X, Y, epochs, batch, lr, seed=0, log=None):
    import torch
    rng = np.random.default_rng(seed)
    n = len(X)
    steps = epochs * max(1, n // batch)
    losses, step = [], 0
    for ep in range(epochs):
        perm = rng.permutation(n)
        acc = []
        for i in range(0, n - batch + 1, batch):
            xb, yb = augment(X[perm[i:i + batch]], Y[perm[i:i + batch]], rng)
            net.forward(torch.as_tensor(xb, device=net.device))
            acc.append(net.loss(yb))
            net.backward()
            net.adam_step(float(0.5 * lr * (1 + np.cos(np.pi * step / max(1, steps)))))
            step += 1
        torch.cuda.synchronize()
        losses.append(float(torch.stack(acc).mean()))
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {losses[-1]:.5f}")
    return losses


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ntrain", type=int, default=768)
    ap.add_argument("--neval", type=int, default=64)
    ap.add_argument("--niter", type=int, default=1000)
    ap.add_argument("--K", type=int, default=K_DEFAULT)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--rtol", type=float, default=1e-4)
    ap.add_argument("--out", default="unet_closure256.npz")
    ap.add_argument("--report", default=None)
    ap.add_argument("--workers", type=int, default=1, help="host processes that make the training problems")
    ap.add_argument("--chunk", type=int, default=512, help="training problems made and solved at a time")
    args = ap.parse_args(argv)

    def log(msg):
        print(f"[{time.strftime('%H:%M:%S')}] {msg}", flush=True)

    rep = {"args": vars(args)}
    X, Y = [], []
    t_gen = ms_k = ms_p = 0.0
    for c0 in range(0, args.ntrain, args.chunk):  # pairs made a chunk at a time: only images are kept
        t0 = time.time()
        tr = make_set_parallel(range(20000 + c0, 20000 + min(args.ntrain, c0 + args.chunk)), args.niter,
                               args.workers)
        kws = [e[0] for e in tr]
        t_gen += time.time() - t0
        _, xk, _, ms = early_images(kws, args.K)
        ms_k += ms
        xs, _, _, _, ms = data.solve(kws, args.niter, 64, chunk=256)
        ms_p += ms
        X.append(xk)
        Y.append(normalise([data.to_grid(kw, x) for kw, x in zip(kws, xs)]))
        del tr, kws, xs
        log(f"training pairs {min(args.ntrain, c0 + args.chunk)}/{args.ntrain}")
    X, Y = np.concatenate(X), np.concatenate(Y)
    rep["t_generate_s"], rep["plain_fp64_batched_s"] = t_gen, ms_p / 1000.0
    log(f"generation {t_gen:.0f} s; early images {ms_k / 1000:.1f} s, plain FP64 solves {ms_p / 1000:.1f} s "
        "on the device")
    net = UNet(seed=0)
    t0 = time.time()
    rep["losses"] = train(net, X, Y, args.epochs, args.batch, args.lr, log=log)
    rep["t_train_s"] = time.time() - t0
    net.save(args.out)
    log(f"saved {args.out}")
    # held-out check: cold vs warm FP32 solves against FP64 plain targets
    ev = make_set(range(30000, 30000 + args.neval), args.niter)
    ekws = [e[0] for e in ev]
    _, _, cost_p, _, _ = data.solve(ekws, args.niter, 64)
    tg = cost_p * (1 + args.rtol)
    _, icold, _, _, ms_cold = data.solve(ekws, args.niter, 32, targets=tg)
    xk, imk, ik, ms_k = early_images(ekws, args.K, targets=tg)
    pred = net.predict(imk)
    x0 = [warm_init(kw, p, x) for kw, p, x in zip(ekws, pred, xk)]
    _, iw, _, _, ms_w = data.solve(ekws, args.niter - args.K, 32, targets=tg, x0=x0)
    hit_k = np.array([i["task"] == 8 for i in ik])
    hit_w = np.array([i["task"] == 8 for i in iw]) | hit_k
    rep["eval"] = {"n": args.neval, "cold_hits": int(sum(i["task"] == 8 for i in icold)), "cold_ms": ms_cold,
                   "warm_hits": int(hit_w.sum()), "warm_ms": ms_k + ms_w,
                   "cold_iterations_mean": float(np.mean([i["niter"] for i in icold])),
                   "warm_iterations_mean": float(np.mean([args.K + (0 if h else i["niter"])
                                                          for h, i in zip(hit_k, iw)]))}
    log(json.dumps(rep["eval"]))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)


if __name__ == "__main__":
    main()
