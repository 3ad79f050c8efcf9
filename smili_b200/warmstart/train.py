"""Train the warm-start U-Net on pairs the plain method generates, then
evaluate it on held-out seeds.

    python -m smili_b200.warmstart.train --ntrain 2000 --neval 200 \\
        --out weights.npz --report report.json

Steps (all on one GPU):

1. synthetic problems (``synth.warmstart_problem``), training seeds
   0..ntrain-1 and held-out seeds 10**6 + i, generated 1024 at a time;
2. dirty images in one batched evaluation per chunk;
3. plain solves (FP64 L-BFGS-B from the Gaussian prior, niter iterations)
   in batched launches: the training targets, and for the held-out set
   the reference final costs;
4. training with Adam on the MSE between the network output and the
   reconstruction scaled to max 1 (random flips and transposes);
5. held-out evaluation: warm-started FP64 solves with the plain final cost
   x (1 + rtol) as objective target and the same iteration cap, giving the
   iterations to equal chi-square and the image NRMSE against the truth,
   beside the plain solves; plus the FP32 batched plain and warm-started
   launch times.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import data
from .unet import UNet


def augment(x, y, rng):
    """Random flips / transposes applied identically to inputs and targets."""
    k = int(rng.integers(0, 8))
    if k & 1:
        x, y = x[:, :, ::-1], y[:, :, ::-1]
    if k & 2:
        x, y = x[:, ::-1, :], y[:, ::-1, :]
    if k & 4:
        x, y = np.transpose(x, (0, 2, 1)), np.transpose(y, (0, 2, 1))
    return np.ascontiguousarray(x), np.ascontiguousarray(y)


def train(net, X, Y, epochs, batch, lr, seed=0, log=None):
    """Adam with cosine decay; returns the per-epoch mean losses and the
    median wall time of one training step in ms (device-synchronised every
    50 steps, so launch and host overheads are included)."""
    import torch
    rng = np.random.default_rng(seed)
    n = len(X)
    steps = epochs * (n // batch)
    losses, step, t_steps = [], 0, []
    for ep in range(epochs):
        perm = rng.permutation(n)
        acc = []
        for i in range(0, n - batch + 1, batch):
            idx = perm[i:i + batch]
            xb, yb = augment(X[idx], Y[idx], rng)
            lr_t = 0.5 * lr * (1 + np.cos(np.pi * step / max(1, steps)))
            t0 = time.perf_counter()
            net.forward(torch.as_tensor(xb, device=net.device))
            loss = net.loss(yb)
            net.backward()
            net.adam_step(float(lr_t))
            acc.append(loss)
            step += 1
            if step % 50 == 0:
                torch.cuda.synchronize()
            t_steps.append(time.perf_counter() - t0)
        torch.cuda.synchronize()
        losses.append(float(torch.stack(acc).mean()))
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {losses[-1]:.5f}")
    return losses, 1000.0 * float(np.median(t_steps[len(t_steps) // 2:]))


def unet_flops(net, H, W):
    """Multiply-add FLOPs of one forward pass on an H x W image."""
    f = 0
    for L in net.layers:
        h, w = net.hw[L.name]
        f += 2 * h * w * 9 * L.cin * L.cout
    return f


def evaluate(net, ev, niter, rtol, log=None):
    """Plain vs warm-started solves on the held-out set."""
    kws = [e[0] for e in ev]
    truths = [e[1] for e in ev]
    xs_p, inf_p, cost_p, tr_p, ms_p = data.solve(kws, niter, 64)
    targets = cost_p * (1 + rtol)
    dirty = data.dirty_images(kws)
    pred = net.predict(dirty)
    x0 = [data.warm_init(kw, pr, e[2]) for kw, pr, e in zip(kws, pred, ev)]
    xs_w, inf_w, cost_w, tr_w, ms_w = data.solve(kws, niter, 64, targets=targets, x0=x0)
    # the plain solve's own first iteration at or below the target
    it_plain = np.array([int(np.argmax(np.asarray(t) <= g)) + 1 if np.any(np.asarray(t) <= g) else niter + 1
                         for t, g in zip(tr_p, targets)])
    reached = np.array([i["task"] == 8 for i in inf_w])
    it_warm = np.array([i["niter"] for i in inf_w])
    nr_p = np.array([data.nrmse(data.to_grid(kw, x), t) for kw, x, t in zip(kws, xs_p, truths)])
    nr_w = np.array([data.nrmse(data.to_grid(kw, x), t) for kw, x, t in zip(kws, xs_w, truths)])
    nr_0 = np.array([data.nrmse(data.to_grid(kw, x), t) for kw, x, t in zip(kws, x0, truths)])
    nr_g = np.array([data.nrmse(data.to_grid(kw, kw["iin"]), t) for kw, t in zip(kws, truths)])
    # FP32 batched: plain (Gaussian prior, niter) vs warm (target stop)
    _, inf32p, _, _, ms32p = data.solve(kws, niter, 32)
    _, inf32w, _, _, ms32w = data.solve(kws, niter, 32, targets=targets, x0=x0)
    rep = {
        "n_eval": len(ev), "niter": niter, "target_rtol": rtol,
        "warm_reached_target": int(reached.sum()),
        "iterations_to_target_warm_median": float(np.median(it_warm[reached])) if reached.any() else None,
        "iterations_to_target_warm_mean": float(np.mean(np.where(reached, it_warm, niter + 1))),
        "iterations_plain_mean": float(np.mean(it_plain)),
        "final_cost_warm_over_plain_median": float(np.median(cost_w / cost_p)),
        "nrmse_truth_plain_median": float(np.median(nr_p)),
        "nrmse_truth_warm_median": float(np.median(nr_w)),
        "nrmse_truth_warm_init_median": float(np.median(nr_0)),
        "nrmse_truth_gaussian_prior_median": float(np.median(nr_g)),
        "fp64_batch_ms_plain": ms_p, "fp64_batch_ms_warm": ms_w,
        "fp32_batch_ms_plain": ms32p, "fp32_batch_ms_warm": ms32w,
        "fp32_warm_reached_target": int(sum(i["task"] == 8 for i in inf32w)),
        "fp32_warm_iterations_mean": float(np.mean([i["niter"] for i in inf32w])),
    }
    if log:
        log(json.dumps(rep))
    return rep


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--ntrain", type=int, default=2000)
    ap.add_argument("--neval", type=int, default=200)
    ap.add_argument("--niter", type=int, default=1000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--rtol", type=float, default=1e-4)
    ap.add_argument("--out", default="unet_warmstart.npz")
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)

    def log(msg):
        print(f"[{time.strftime('%H:%M:%S')}] {msg}", flush=True)

    rep = {"args": vars(args)}
    # training pairs, generated and solved 1024 seeds at a time
    X, Y = [], []
    t_gen = t_sol = ms_sum = 0.0
    for c0 in range(0, args.ntrain, 1024):
        t0 = time.time()
        tr = data.make_set(range(c0, min(args.ntrain, c0 + 1024)), args.niter)
        t_gen += time.time() - t0
        t0 = time.time()
        kws = [e[0] for e in tr]
        X.append(data.dirty_images(kws))
        xs, _, _, _, ms = data.solve(kws, args.niter, 64)
        y = np.asarray([data.to_grid(kw, x) for kw, x in zip(kws, xs)], np.float32)
        Y.append(y / np.maximum(y.reshape(len(y), -1).max(axis=1), 1e-30)[:, None, None])
        t_sol += time.time() - t0
        ms_sum += ms
        log(f"training pairs {c0 + len(tr)}/{args.ntrain}")
    X, Y = np.concatenate(X), np.concatenate(Y)
    rep["t_generate_s"], rep["t_plain_solves_s"], rep["plain_batch_ms"] = t_gen, t_sol, ms_sum
    log(f"training set: generation {t_gen:.1f} s, dirty images + plain solves {t_sol:.1f} s "
        f"({ms_sum / 1000:.1f} s on the device)")
    ev = data.make_set(range(10 ** 6, 10 ** 6 + args.neval), args.niter)
    net = UNet(seed=0)
    t0 = time.time()
    losses, step_ms = train(net, X, Y, args.epochs, args.batch, args.lr, log=log)
    rep["t_train_s"] = time.time() - t0
    rep["losses"] = losses
    rep["train_step_ms"] = step_ms
    H, W = X.shape[1:]
    rep["train_tflops"] = 3 * unet_flops(net, H, W) * args.batch / (step_ms / 1000.0) / 1e12
    rep["nparam"] = net.nparam
    net.save(args.out)
    log(f"saved {args.out}")
    rep["eval"] = evaluate(net, ev, args.niter, args.rtol, log=log)
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    log("done")


if __name__ == "__main__":
    main()
