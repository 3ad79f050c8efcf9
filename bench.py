"""Benchmark: static-imaging solves/s at 256x256 / ~1e5 visibilities.

Workload (the precision-path configuration): 256x256 image, 1 uas pixels,
10 stations, ~1e5 visibilities with station gain errors, data terms
amplitudes (5% error) + closure phases + log closure amplitudes,
regularizers l1 / TV / MEM = 1 / 1 / 0.1, L-BFGS-B m=5, factr=10, pgtol=0,
niter=1000 (the reference's default, smili/imaging/lbfgs.py:44-80).  Inputs
are seeded synthetic observations (no public data set exists); distinct
seeds are replicated to the batch size.

A solve runs the reference driver's iteration budget (niter iterations,
stopped like fftim2d.f90:324) and exits early once it reaches the final cost
of the plain FP64 single-problem solve of the same data x (1 + target_rtol).
L-BFGS-B on the closure terms is chaotic: a 1e-12 perturbation of the start
changes the iterates at the 1e-2 level within ten iterations, and the plain
FP64 method rerun with another reduction order reaches its own earlier final
cost in only about half of the cases.  "Equal final chi-square" is therefore
shown as a distribution: the FP32 solves' final cost / plain final cost and
target hit rate beside those of an FP64 control arm (the plain method rerun
four times per seed, in one batch).  ``value`` counts only the solves that
reached their plain solve's final cost (x (1 + target_rtol)) within its
iteration budget; ``value_all`` counts every solve of the launch.

One step = one batched FP32 solve of ``--batch`` problems with inputs
resident on the device.  The batch holds more problems than resident CTA
groups: a group whose problem reaches its target takes the next queued
problem, so early exits shorten the launch.  The group size is chosen by
``smili_b200.autotune`` from whole solves of this batch with its targets.
With the trained weights present the step is the learned warm start
(``WarmStart``): 50 FP32 iterations from the prior, the U-Net's proposal
from those images, and the remaining iterations from the proposals; the
cold arm (every problem from its prior) is timed beside it (``value_cold``).
``value`` = counted solves per second over the timed steps; ``e2e`` = the
same metric through the C ABI from host buffers (packing and upload of the
problems, the step, download of every image inside the timed region);
``plain_fp64`` reports single-problem FP64 solves/s; ``cpu_baseline`` times
the CPU restatement (one whole solve).
``--impl reference`` times only that CPU path (the reference's
Fortran/FINUFFT build is unavailable in this image).

For N > 1 (torchrun) every rank solves its own batch (replicas, no
collective on the data path); value = all ranks' solves / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes per function/gradient evaluation of the FP32 batched solver on
# this workload at the benchmark's concurrency (74 resident groups of 4
# CTAs of 512 threads): one ncu capture of ``bench.py --case traffic`` (74
# problems, 20 iterations) measured dram__bytes_read.sum +
# dram__bytes_write.sum = 70.02 + 31.74 GB over 2261 evaluations.  The
# traffic of a step scales with its evaluation count.
DRAM_BYTES_PER_EVAL_FP32 = (70.02e9 + 31.74e9) / 2261

METRIC = "imaging solves/s at 256²/1e5 vis, FP32+batched+warm-start vs plain, equal final χ²"
WORKLOAD = ("256x256 / 97 200 uv points (amp 5% + cp + lca), l1/TV/MEM = 1/1/0.1, L-BFGS-B m=5, "
            "{niter} iterations, a solve counts at the plain FP64 solve's final cost x (1 + {rtol:g})")


def make_problems(nseed, niter, truths=None):
    """The workload's seeded problems.  Model visibilities come from the
    exact DFT on the host (``synth.exact_dft``), so making them runs no
    device code and both arms solve identical inputs."""
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    kws = []
    for s in range(nseed):
        obs = synth.precision_path(seed=1000 + s, niter=niter)
        kw, _ = prepare_imaging(obs.image, amptable=obs.amptable, bstable=obs.bstable,
                                catable=obs.catable, niter=niter, **obs.reg)
        kws.append(kw)
        if truths is not None:
            truths.append(obs.truth)
    return kws


def nrmse(kw, x, truth):
    """||image - truth|| / ||truth|| with the pixel vector placed on the grid,
    after the integer-pixel shift of the image that best matches the truth
    (the peak of their circular cross-correlation): amplitudes and closure
    quantities carry no absolute position, so a solve may land shifted."""
    img = np.zeros_like(truth)
    img[np.asarray(kw["yidx"]) - 1, np.asarray(kw["xidx"]) - 1] = x / float(kw["inormfactr"])
    xc = np.fft.ifft2(np.fft.fft2(truth) * np.conj(np.fft.fft2(img))).real
    dy, dx = np.unravel_index(int(np.argmax(xc)), xc.shape)
    img = np.roll(img, (dy, dx), axis=(0, 1))
    return float(np.linalg.norm(img - truth) / np.linalg.norm(truth))


def fg_bytes(kw, s=4):
    """Compulsory bytes of one function/gradient evaluation: image in,
    gradient out, uv coordinates, data + variance + signed indices, and one
    weight image per weighted regularizer."""
    npix, nuv = int(kw["npix"]), np.asarray(kw["u"]).size
    nfcv = np.asarray(kw["uvidxfcv"]).size if kw["isfcv"] else 0
    namp = np.asarray(kw["uvidxamp"]).size if kw["isamp"] else 0
    ncp = np.asarray(kw["uvidxcp"]).shape[1] if kw["iscp"] else 0
    nca = np.asarray(kw["uvidxca"]).shape[1] if kw["isca"] else 0
    nreg = sum(1 for k in ("l1_l", "tv_l", "tsv_l", "kl_l", "gs_l") if kw[k] > 0)
    return (s * 2 * npix + s * 2 * nuv + nfcv * (3 * s + 4) + namp * (2 * s + 4)
            + ncp * (2 * s + 12) + nca * (2 * s + 16) + s * npix * nreg)


def task_histogram(codes):
    """How solves ended, from their L-BFGS-B task codes: reached the target
    cost, converged (factr / pgtol test), abnormal line-search end, iteration
    limit, error (a device wait timed out), other."""
    from smili_b200 import _lib
    names = {_lib.TASK_TARGET: "target", _lib.TASK_CONV: "converged", _lib.TASK_ABNORMAL: "abnormal",
             _lib.TASK_STOP: "iteration_limit", _lib.TASK_ERROR: "error"}
    out = {v: 0 for v in names.values()}
    for c in codes:
        k = names.get(int(c), "other")
        out[k] = out.get(k, 0) + 1
    return out


def lb_bytes_per_iteration(kw, m=5):
    """Compulsory FP64 traffic of one L-BFGS-B iteration (lbfgsb.f v3.0):
    the limited-memory matrices S and Y (2 m n doubles) read by the Cauchy
    point, formk and subspace minimisation, and about ten n-vectors (x, g,
    d, z, r, t, xp and the bounds' work) read or written: (4 m + 10) n x 8
    bytes."""
    return (4 * m + 10) * int(kw["npix"]) * 8


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device=0):
        self.samples = []
        self.stop = threading.Event()
        self.device = device

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and "Active" in s[3 + i] and "Not" not in s[3 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


NFG_FIXTURE = os.path.join(ROOT, "tests", "golden", "bench_plain_nfg.json")


def plain_nfg_table():
    """Evaluations of whole plain FP64 solves of the workload's seeds by the
    CPU restatement, by seed (``tests/golden/make_bench_nfg.py``)."""
    with open(NFG_FIXTURE) as f:
        d = json.load(f)
    return {int(r["seed"]) - 1000: int(r["nfg"]) for r in d["solves"]}, d


def cpu_sample(kw, iters):
    """Seconds per function/gradient evaluation of the CPU restatement
    (oracle, FP64, NUFFT eps 1e-6, all host threads) over the first
    ``iters`` iterations of one plain solve: (s per evaluation, evaluations,
    seconds)."""
    from oracle import oracle as O
    O.build()
    k = dict(kw)
    k["niter"] = iters
    t0 = time.perf_counter()
    _, _, info = O.imaging(k, eps=1e-6)
    dt = time.perf_counter() - t0
    return dt / max(1, info["nfg"]), info["nfg"], dt


def cpu_baseline(kw, iters, nfg_seed0):
    """The CPU restatement on the host cores: one whole plain solve of the
    first seed (``kw``, 1000 iterations), timed end to end; and, as a check
    of the reference arm's extrapolation, a sample of its first ``iters``
    iterations scaled to the whole solve's evaluation count."""
    from oracle import oracle as O
    O.build()
    t0 = time.perf_counter()
    _, terms, info = O.imaging(kw, eps=1e-6)
    whole = time.perf_counter() - t0
    per, n, dt = cpu_sample(kw, iters)
    return {"value": 1.0 / whole, "unit": "solves/s", "cores": O.lib().orc_nthreads(), "kind": "port",
            "sample": f"one whole plain solve of the first seed ({info['niter']} iterations, "
                      f"{info['nfg']} evaluations, FP64, NUFFT eps 1e-6): {whole:.1f} s",
            "whole_solve_s": whole, "whole_solve_nfg": int(info["nfg"]),
            "whole_solve_nfg_fixture": nfg_seed0,
            "extrapolated_from_sample": {"iterations": iters, "evaluations": n, "s": dt,
                                         "solves_per_s": 1.0 / (per * info["nfg"])}}


def warm_start_cfg4(nprob, niter, rtol, device=0, group=4):
    """The learned warm start on the 128x128 warm-start configuration
    (complex visibilities + closure phases, 6-12 stations, SNR 5-200).
    Held-out problems are solved:

    - by the plain method: FP64 single-problem launches from the Gaussian
      prior, niter iterations; the final cost x (1 + rtol) becomes each
      problem's target;
    - by the FP32 batched solver from the same prior, with an early exit at
      the target;
    - by the FP32 batched solver from the U-Net's proposal, with the same
      exit; its time adds the proposal: the device time of the dirty-image
      evaluation and of the network's forward pass, and the host time that
      turns the network output into starting pixel vectors.  Host packing of
      batches is outside both arms' times.

    Groups of ``group`` CTAs per problem leave fewer resident groups than
    problems, so a problem that exits early hands its CTAs to a queued one
    and the launch time follows the total work."""
    import torch
    from smili_b200.warmstart import data
    from smili_b200.warmstart.unet import UNet
    path = os.path.join(ROOT, "smili_b200", "warmstart", "unet_cfg4.npz")
    if not os.path.exists(path):
        return {"unavailable": "trained weights smili_b200/warmstart/unet_cfg4.npz missing"}
    net = UNet.load(path, device=f"cuda:{device}")
    ev = data.make_set(range(3 * 10 ** 6, 3 * 10 ** 6 + nprob), niter)
    kws = [e[0] for e in ev]
    xs_p, _, cost_p, _, _ = data.solve(kws, niter, 64, device=device)
    targets = cost_p * (1 + rtol)
    t_single = [data.solve([kws[i]], niter, 64, device=device)[4] for i in range(min(4, nprob))]
    xs_32p, inf32p, _, _, ms32p = data.solve(kws, niter, 32, targets=targets, device=device,
                                              ctas_per_problem=group)
    net.predict(data.dirty_images(kws[:8], device=device))  # first-call setup of both libraries
    ms_dirty = []
    dirty = data.dirty_images(kws, device=device, kernel_ms=ms_dirty)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    pred = net.predict(dirty)
    e1.record()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x0 = [data.warm_init(kw, pr, e[2]) for kw, pr, e in zip(kws, pred, ev)]
    t_init = time.perf_counter() - t0
    t_infer = sum(ms_dirty) / 1000.0 + e0.elapsed_time(e1) / 1000.0 + t_init
    xs_w, inf32w, _, _, ms32w = data.solve(kws, niter, 32, targets=targets, x0=x0, device=device,
                                           ctas_per_problem=group)
    nr = lambda xs: float(np.median([data.nrmse(data.to_grid(kw, x), e[1]) for kw, x, e in zip(kws, xs, ev)]))
    return {"problems": nprob, "niter": niter, "target_rtol": rtol, "ctas_per_problem": group,
            "plain_fp64_single_solves_per_s": 1000.0 / float(np.mean(t_single)),
            "fp32_batched_solves_per_s": nprob / (ms32p / 1000.0),
            "fp32_batched_warm_solves_per_s": nprob / (ms32w / 1000.0 + t_infer),
            "warm_inference_s": t_infer,
            "warm_inference_parts_s": {"dirty_images_device": sum(ms_dirty) / 1000.0,
                                       "unet_forward_device": e0.elapsed_time(e1) / 1000.0,
                                       "starting_vectors_host": t_init},
            "fp32_reached_target": int(sum(i["task"] == 8 for i in inf32p)),
            "fp32_warm_reached_target": int(sum(i["task"] == 8 for i in inf32w)),
            "fp32_iterations_mean": float(np.mean([i["niter"] for i in inf32p])),
            "fp32_warm_iterations_mean": float(np.mean([i["niter"] for i in inf32w])),
            "nrmse_truth_plain_fp64": nr(xs_p), "nrmse_truth_fp32": nr(xs_32p),
            "nrmse_truth_warm_fp32": nr(xs_w)}


UNET_FORWARD_LAUNCHES = 21  # 15 convolutions, 3 poolings, 3 upsamplings per forward pass


class WarmStart:
    """The learned warm start on this workload (``smili_b200.warmstart.closure``).

    One step: K FP32 iterations of every problem from its prior, the U-Net's
    proposal from each K-iteration image, then the remaining niter - K FP32
    iterations from the proposals, with the same targets as the cold arm.
    Both phases are launches of one device-resident batch, and the images
    never leave the device: between the launches ``Batch.images`` writes the
    K-iteration images as the network's input grid, the network runs on it,
    and ``Batch.set_starts_from_images`` turns its output into every
    problem's start image (``Batch.set_niter`` changes the iteration caps;
    ``Batch.reset_starts`` puts the priors back at the start of the next
    step).  A problem that reaches its target in the first K iterations
    counts there and restarts from its own image.  The step's time is the
    two launches' CUDA event times, the network's forward pass (CUDA events)
    and the calls around them (wall clock)."""

    def __init__(self, probs, kws, seed_of, ftarget, niter, G, device=0):
        import torch
        from smili_b200 import _lib
        from smili_b200.warmstart import closure
        from smili_b200.warmstart.unet import UNet
        self.torch, self.lib, self.closure = torch, _lib, closure
        self.net = UNet.load(WARM_WEIGHTS, device=f"cuda:{device}")
        self.K, self.niter = closure.K_DEFAULT, niter
        self.kws, self.seed_of, self.B = kws, seed_of, len(probs)
        self.b = _lib.Batch(probs, niter=niter, options=_lib.make_options(32, 1e-6, G, device))
        self.b.set_targets(ftarget)
        nx = int(kws[0]["nx"])
        self.img = torch.zeros((self.B, nx, nx), dtype=torch.float32, device=f"cuda:{device}")
        self.net.forward(self.img)  # buffers and first-call set-up
        torch.cuda.synchronize()

    def step(self):
        torch, _lib, B, b = self.torch, self.lib, self.B, self.b
        t0 = time.perf_counter()
        b.set_niter(self.K)
        b.reset_starts()
        t_host = time.perf_counter() - t0
        ms_k = b.run()
        t0 = time.perf_counter()
        early = [b.info(p) for p in range(B)]
        hit_k = np.array([e["task"] == _lib.TASK_TARGET for e in early])
        b.images(self.img)
        t_host += time.perf_counter() - t0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pred = self.net.forward(self.img)[:, :, :, 0].float()
        e1.record()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.set_starts_from_images(pred, keep=hit_k)
        b.set_niter(self.niter - self.K)
        t_host += time.perf_counter() - t0
        ms_w = b.run()
        infos = [b.info(p) for p in range(B)]
        hit = hit_k | np.array([i["task"] == _lib.TASK_TARGET for i in infos])
        ms_net = e0.elapsed_time(e1)
        return {"s": (ms_k + ms_net + ms_w) / 1000.0 + t_host, "hits": int(hit.sum()),
                "kernel_s": (ms_k + ms_w) / 1000.0,
                "nfg": int(sum(e["nfg"] for e in early) + sum(i["nfg"] for i in infos)),
                "iterations": int(sum(self.K if h else self.K + i["niter"] for h, i in zip(hit_k, infos))),
                "parts_s": {"first_K_iterations_device": ms_k / 1000.0, "unet_forward_device": ms_net / 1000.0,
                            "host": t_host, "remaining_iterations_device": ms_w / 1000.0}}

    def fetch(self, p):
        return self.b.fetch(p)

    def close(self):
        self.b.close()


WARM_WEIGHTS = os.path.join(ROOT, "smili_b200", "warmstart", "unet_closure256.npz")
WARM_K = 50  # FP32 iterations before the proposal (smili_b200.warmstart.closure.K_DEFAULT)
WARM_HELPER_LAUNCHES = 2  # smili_batch_images and smili_batch_set_starts_from_images
PROB_RESULT_BYTES = 20 * 8 + 4 * 4  # ProbResult: terms[SMILI_NTERMS3D] and four counters


def survey_cfg3(nprob, niter, device=0, nplain=8):
    """The batched survey: nprob problems with image sizes from {64, 96, 128,
    192, 256}^2, 2e3-5e4 visibilities, fcv + closure phases and (l1, tsv, mem)
    on the 8^3 log grid, solved in one launch in FP32 and in FP64, and the
    plain method (one FP64 launch per problem) on the first nplain problems."""
    from smili_b200 import _lib, synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    kws = []
    for i in range(nprob):
        obs = synth.survey_problem(i, seed=3, niter=niter, model=synth.nufft_model)
        kw, _ = prepare_imaging(obs.image, vistable=obs.vistable, bstable=obs.bstable, niter=niter, **obs.reg)
        kws.append(kw)
    probs = [_lib.Problem(k) for k in kws]
    out = {"problems": nprob, "niter": niter,
           "nx_counts": {str(n): int(sum(int(k["nx"]) == n for k in kws)) for n in (64, 96, 128, 192, 256)},
           "uv_points_median": int(np.median([np.size(k["u"]) for k in kws]))}
    cost = {}
    for prec in (32, 64):
        b = _lib.Batch(probs, niter=niter, options=_lib.make_options(prec, 1e-6, 0, device))
        ms = b.run()
        info = [b.fetch(p)[3] for p in range(nprob)]
        cost[prec] = np.array([b.fetch(p)[1]["cost"] for p in range(nprob)])
        b.close()
        out[f"fp{prec}_batched_s"] = ms / 1e3
        out[f"fp{prec}_batched_solves_per_s"] = nprob / (ms / 1e3)
        out[f"fp{prec}_iterations_mean"] = float(np.mean([i["niter"] for i in info]))
    r = cost[32] / cost[64]
    out["fp32_over_fp64_final_cost_median_p10_p90"] = [float(np.median(r)), float(np.percentile(r, 10)),
                                                       float(np.percentile(r, 90))]
    ts = []
    for p in range(min(nplain, nprob)):
        s = _lib.Batch([probs[p]], niter=niter, options=_lib.make_options(64, 1e-6, 0, device))
        ts.append(s.run())
        s.close()
    out["plain_fp64_single_solves_per_s"] = 1e3 / float(np.mean(ts))
    return out


def dynamic_cfg5(niter, device=0, cpu_evals=2):
    """Dynamic imaging (fftim3d): 64 frames of 128x128, ~6000 visibilities
    per frame from 16 stations over 24 h, a crescent rotating by 90 deg,
    complex visibilities + closure phases, l1 = tsv = 1 per frame, Rt = 1.
    One movie solve (1000 iterations) in FP64 and FP32 on the device, and
    the CPU restatement's time per evaluation (host threads) scaled to the
    FP64 solve's evaluation count."""
    from oracle import oracle as O
    from smili_b200 import synth
    from smili_b200.fortlib import fftim3d
    from smili_b200.imaging.lbfgs3d import prepare_imaging3d
    m = synth.dynamic_problem(seed=0, nframes=64, nx=128, nst=16, vis_per_frame=6000, niter=niter,
                              model=synth.nufft_model)
    kw, _ = prepare_imaging3d(m.frames, vistable=m.vistable, bstable=m.bstable, niter=niter, **m.reg)
    out = {"frames": 64, "nx": 128, "visibilities": int(len(m.vistable)), "closure_phases": int(len(m.bstable)),
           "parameters": int(np.size(kw["iin"])), "niter": niter}
    for prec in (64, 32):
        info = {}
        t0 = time.perf_counter()
        r = fftim3d.imaging(precision=prec, nufft_eps=1e-6, device=device, info=info, **kw)
        dt = time.perf_counter() - t0
        out[f"fp{prec}_solve_s"] = dt
        out[f"fp{prec}_final_cost"] = r[20]
        out[f"fp{prec}_nfg"] = info["nfg"]
    O.build()
    t0 = time.perf_counter()
    for _ in range(cpu_evals):
        O.calc_cost3d(kw, kw["iin"], eps=1e-6)
    per = (time.perf_counter() - t0) / cpu_evals
    out["cpu_port_s_per_eval"] = per
    out["cpu_port_solve_s_scaled"] = per * out["fp64_nfg"]
    out["cpu_cores"] = O.lib().orc_nthreads()
    return out


def large_cfg5(niter, device=0, cpu_evals=1):
    """Large static image: 1024x1024 (1 uas pixels), 16 stations over 24 h
    with ~5 s scans (~2e6 complex visibilities + closure phases), l1 = tsv
    = 1, 50 uas Gaussian prior.  One FP64 and one FP32 solve on the device; the CPU restatement's
    time per evaluation scaled to the FP64 evaluation count."""
    from oracle import oracle as O
    from smili_b200 import synth
    from smili_b200.fortlib import fftim2d
    from smili_b200.imaging.lbfgs import prepare_imaging
    rng = np.random.default_rng(11)
    img = synth.Image(1024, 1024, 1.0)
    truth = synth.multigauss_gp_image(img, rng, ngauss=50, flux=1.0, extent_uas=200.0)
    t = synth.observe(truth, img, rng, nst=16, dec_deg=12.0, freq_hz=230e9, hours=24.0, scan_min=5.2 / 60.0,
                      fcv=True, cp=True, model=synth.nufft_model)
    init = img.copy()
    # a 50 uas prior: from 100-200 uas priors the first line search of the
    # plain method (and of the CPU restatement) ends ABNORMAL at iteration 1
    init.data[0, 0] = synth.gaussian_image(img, 50.0, 1.0)
    kw, _ = prepare_imaging(init, vistable=t["vistable"], bstable=t["bstable"], niter=niter, l1_lambda=1.0,
                            tsv_lambda=1.0)
    out = {"nx": 1024, "visibilities": int(len(t["vistable"])), "closure_phases": int(len(t["bstable"])),
           "niter": niter}
    for prec in (64, 32):
        info = {}
        t0 = time.perf_counter()
        r = fftim2d.imaging(precision=prec, nufft_eps=1e-6, device=device, info=info, **kw)
        out[f"fp{prec}_solve_s"] = time.perf_counter() - t0
        out[f"fp{prec}_final_cost"] = r[15]
        out[f"fp{prec}_nfg"] = info["nfg"]
    O.build()
    t0 = time.perf_counter()
    for _ in range(cpu_evals):
        O.calc_cost(kw, kw["iin"], eps=1e-6)
    per = (time.perf_counter() - t0) / cpu_evals
    out["cpu_port_s_per_eval"] = per
    out["cpu_port_solve_s_scaled"] = per * out["fp64_nfg"]
    out["cpu_cores"] = O.lib().orc_nthreads()
    return out


def max_over_ranks(dist, ms_step, e2e_s, device):
    """Replicas only: every rank solves its own batch, and the job's time is
    the slowest rank's (step time and end-to-end time, all-reduced with MAX;
    the identity on one process)."""
    if dist is None:
        return ms_step, e2e_s
    import torch
    t = torch.tensor([ms_step, e2e_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0]), float(t[1])


def job_values(world, batch, reached, max_ms, e2e_s):
    """Whole-job solves/s over the slowest rank's time: every solve, the
    solves that reached their target, and every solve end to end."""
    return (world * batch / (max_ms / 1000.0), world * reached / (max_ms / 1000.0),
            world * batch / e2e_s)


def run_reference(args, rank, world):
    """The reference arm: the CPU restatement of the reference's fortlib path
    (``oracle/``, C++/OpenMP on every host thread; the reference's own
    Fortran/FINUFFT build cannot be built in this image) on the GPU arm's
    workload.  The inputs are made on the host (exact DFT) and nothing of
    this project's CUDA library is loaded.  Each step is one timed sample:
    ``--ref-iters`` iterations of the plain FP64 solve of seed (step mod
    seeds), from its prior.  A step's predicted whole-solve time is its
    seconds per evaluation times the evaluation count of that seed's whole
    plain solve by the same restatement (``tests/golden/bench_plain_nfg.json``);
    value = timed steps / the sum of those predicted times.  Under torchrun
    only rank 0 works."""
    if rank != 0:
        return
    S = args.seeds
    kws = make_problems(S, args.niter)
    nfg, fixture = plain_nfg_table()
    for _ in range(args.warmup):
        cpu_sample(kws[0], args.ref_iters)
    step_s, pred = [], []
    for k in range(args.steps):
        per, n, dt = cpu_sample(kws[k % S], args.ref_iters)
        step_s.append(dt)
        pred.append(per * nfg[k % S])
    from oracle import oracle as O
    v = args.steps / float(np.sum(pred))
    cores = O.lib().orc_nthreads()
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(step_s)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD.format(niter=args.niter, rtol=args.target_rtol),
                       "distinct_seeds": S, "parallelism": f"host threads x{cores}",
                       "step": f"one timed sample: {args.ref_iters} iterations of the plain FP64 solve "
                               "of seed (step mod distinct_seeds)"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{args.steps} samples of {args.ref_iters} iterations (FP64, NUFFT eps "
                                       "1e-6), each scaled by its seed's whole-solve evaluation count "
                                       f"(mean {fixture['nfg_mean']:.0f}, measured by whole solves of the "
                                       "same restatement)"},
            "predicted_solve_s_mean": float(np.mean(pred)),
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def profile_case(case, device=0):
    """One small launch of interest for an ncu capture (``--case``):

    - ``traffic``: the benchmark's concurrency (74 resident groups of 4 CTAs,
      74 problems of the workload) for 20 FP32 iterations;
    - ``stages``: the same launch with the stage profiler on, every group busy
      for the whole launch: the steady-state time split per evaluation;
    - ``fg``: one FP32 function/gradient evaluation of those 74 problems;
    - ``t2`` / ``t1``: one FP32 type-2 / type-1 transform of the workload's
      97 200 uv points on the 256 x 256 grid (the transform stages alone);
    - ``conv``: the U-Net convolution 32 x 64 x 64, 192 -> 192 channels,
      timed with CUDA events on the tcgen05 path and the mma.sync path;
    - ``train``: U-Net training steps (forward, backward, Adam) on 32 images
      of 128 x 128, timed with CUDA events.

    Inputs come from the library's own transform (fast), not the exact DFT."""
    from smili_b200 import _lib, synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    if case in ("traffic", "stages", "fg", "t2", "t1"):
        kws = []
        for s in range(16 if case in ("traffic", "stages", "fg") else 1):
            obs = synth.precision_path(seed=1000 + s, niter=20, model=synth.nufft_model)
            kw, _ = prepare_imaging(obs.image, amptable=obs.amptable, bstable=obs.bstable,
                                    catable=obs.catable, niter=20, **obs.reg)
            kws.append(kw)
    if case in ("traffic", "stages", "fg"):
        P = [_lib.Problem(k) for k in kws]
        b = _lib.Batch([P[i % 16] for i in range(74)], niter=1 if case == "fg" else 20,
                       options=_lib.make_options(32, 1e-6, 4, device))
        if case == "stages":
            b.run()  # warm-up
            b.profile(True)
        ms = b.run(fg_only=case == "fg")
        nfg = sum(b.fetch(p)[3]["nfg"] for p in range(74))
        out = {"case": case, "ms": ms, "evaluations": nfg}
        if case == "stages":
            st = b.stage_times()
            n0 = st.pop("n_fg")
            out["group0_us_per_evaluation"] = {k: round(1000.0 * v / n0, 1) for k, v in st.items()
                                               if k != "c_rounds"}
            out["group0_evaluations"] = n0
            b.profile(False)
        b.close()
        print(json.dumps(out))
    elif case in ("t2", "t1"):
        from smili_b200.fortlib import fftlib
        u, v = np.asarray(kws[0]["u"]), np.asarray(kws[0]["v"])
        rng = np.random.default_rng(0)
        if case == "t2":
            fftlib.nufft_fwd_real(u, v, rng.random((256, 256)), precision=32, nufft_eps=1e-6, device=device)
        else:
            c = rng.standard_normal(u.size)
            fftlib.nufft_adj_real1d(u, v, c, np.zeros_like(c), 256, 256, precision=32, nufft_eps=1e-6,
                                    device=device)
        print(json.dumps({"case": case, "uv_points": int(u.size)}))
    elif case == "conv":
        import torch
        from smili_b200.warmstart import kernels as K
        N, H, W, C = 32, 64, 64, 192
        x = torch.randn(N, H, W, C, device=f"cuda:{device}").to(torch.bfloat16)
        w = (torch.randn(C, 3, 3, C, device=f"cuda:{device}") / 20).to(torch.bfloat16)
        y = torch.zeros(N, H, W, C, device=f"cuda:{device}", dtype=torch.bfloat16)
        out = {"case": case, "gflop": 2.0 * N * H * W * C * 9 * C / 1e9}
        for path, name in ((0, "tcgen05"), (2, "tcgen05_one_tile_per_cta"), (1, "mma_sync")):
            K.set_conv_path(path)
            for _ in range(3):
                K.conv3x3(x, N, H, W, C, C, w, None, y, C, C, True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(20):
                K.conv3x3(x, N, H, W, C, C, w, None, y, C, C, True)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 20
            out[name] = {"ms": ms, "tflops": out["gflop"] / ms}
        K.set_conv_path(0)
        print(json.dumps(out))
    elif case == "train":
        import torch
        from smili_b200.warmstart.train import unet_flops
        from smili_b200.warmstart.unet import UNet
        B, H = 32, 128
        rng = np.random.default_rng(0)
        X = rng.random((B, H, H), dtype=np.float32)
        Y = rng.random((B, H, H), dtype=np.float32)
        net = UNet(seed=0, device=f"cuda:{device}")
        xt, yt = torch.as_tensor(X, device=net.device), torch.as_tensor(Y, device=net.device)

        def step():
            net.forward(xt)
            net.loss(yt)
            net.backward()
            net.adam_step(1e-4)
        for _ in range(5):
            step()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 20
        flops = 3 * unet_flops(net, H, H) * B  # forward, data gradient, weight gradient
        print(json.dumps({"case": case, "batch": B, "image": H, "ms_per_step": ms,
                          "tflops": flops / (ms / 1000.0) / 1e12, "nparam": int(net.nparam)}))
    else:
        raise SystemExit(f"unknown case {case}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=444)
    ap.add_argument("--seeds", type=int, default=16)
    ap.add_argument("--niter", type=int, default=1000)
    ap.add_argument("--ref-iters", type=int, default=60)
    ap.add_argument("--target-rtol", type=float, default=1e-4)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="automatic launch shape instead of the autotuner (fewer launches, for profiling)")
    ap.add_argument("--ctas", type=int, default=None,
                    help="fixed CTAs per problem instead of the autotuner (profiled runs: the autotuner's "
                         "timings are not meaningful under a profiler)")
    ap.add_argument("--survey", type=int, default=512,
                    help="problems of the batched survey configuration (0: skip)")
    ap.add_argument("--no-config5", dest="config5", action="store_false",
                    help="skip the 64-frame movie and the 1024x1024 / 2e6-visibility image")
    ap.add_argument("--no-warm", action="store_true",
                    help="time the cold arm (prior starts) as the headline instead of the learned warm start")
    ap.add_argument("--warm-problems", type=int, default=256,
                    help="held-out problems of the learned warm-start comparison (0: skip)")
    ap.add_argument("--case", default=None, choices=["traffic", "stages", "fg", "t2", "t1", "conv", "train"],
                    help="run one small launch for a profiler capture instead of the benchmark")
    args = ap.parse_args()
    if args.case:
        profile_case(args.case)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    from smili_b200 import _lib
    truths = []
    kws = make_problems(args.seeds, args.niter, truths)
    S = len(kws)
    B = args.batch
    P = [_lib.Problem(k) for k in kws]
    probs = [P[i % S] for i in range(B)]
    seed_of = np.arange(B) % S

    # plain FP64 single-problem solves (the drop-in path, niter iterations
    # like the reference driver), one per distinct seed
    opt64 = _lib.make_options(64, 1e-6, device=local)
    plain_ms, plain_cost, plain_nfg, plain_nrmse = [], [], [], []
    for k in range(S):
        plain = _lib.Batch([P[k]], niter=args.niter, options=opt64)
        if k == 0:
            plain.run()  # warm-up
        plain_ms.append(plain.run())
        x, t, _, i = plain.fetch(0)
        plain.close()
        plain_cost.append(t["cost"])
        plain_nfg.append(i["nfg"])
        plain_nrmse.append(nrmse(kws[k], x, truths[k]))
    plain_cost = np.asarray(plain_cost)
    targets = plain_cost * (1.0 + args.target_rtol)

    def quality(b, n, seeds):
        """Per-solve final cost / plain final cost, target hits, NRMSE, and
        how the solves ended (L-BFGS-B task codes: reached the target,
        converged by factr / pgtol, abnormal line-search end, iteration limit)."""
        ratio, hit, err, its, codes = [], 0, [], [], []
        for p in range(n):
            x, t, _, i = b.fetch(p)
            k = seeds[p]
            ratio.append(t["cost"] / plain_cost[k])
            hit += i["task"] == _lib.TASK_TARGET
            codes.append(i["task"])
            err.append(nrmse(kws[k], x, truths[k]))
            its.append(i["niter"])
        return {"reached_target": int(hit), "solves": n, "task_codes": task_histogram(codes),
                "final_cost_over_plain_median": float(np.median(ratio)),
                "final_cost_over_plain_p10_p90": [float(np.percentile(ratio, 10)),
                                                  float(np.percentile(ratio, 90))],
                "nrmse_vs_truth_median": float(np.median(err)),
                "niter_mean": float(np.mean(its)), "nfg_total": 0}

    def hits(b, n):
        return int(sum(b.fetch(p)[3]["task"] == _lib.TASK_TARGET for p in range(n)))

    # control arm: the same FP64 method once more, four batched reruns of
    # every seed (they differ from the plain solve and from each other in
    # reduction order only), same targets and iteration budget
    nctl = 4 * S
    ctl = _lib.Batch([P[i % S] for i in range(nctl)], niter=args.niter, options=opt64)
    ctl.set_targets(targets[np.arange(nctl) % S])
    ctl_ms = ctl.run()
    control = quality(ctl, nctl, np.arange(nctl) % S)
    control["ms"] = ctl_ms
    ctl.close()
    # second control: FP64 from the prior with a 1e-6 relative perturbation
    # per pixel, i.e. trajectories independent of the plain solve's after a
    # few iterations, as FP32 trajectories are from the first evaluation on
    rng = np.random.default_rng(7)
    pert = [_lib.Problem(dict(kws[i % S], iin=np.asarray(kws[i % S]["iin"]) *
                              (1.0 + 1e-6 * rng.standard_normal(np.size(kws[i % S]["iin"])))))
            for i in range(nctl)]
    ctl = _lib.Batch(pert, niter=args.niter, options=opt64)
    ctl.set_targets(targets[np.arange(nctl) % S])
    ctl_ms = ctl.run()
    control_pert = quality(ctl, nctl, np.arange(nctl) % S)
    control_pert["ms"] = ctl_ms
    ctl.close()
    del pert

    # launch shape: CTAs per problem from whole solves of this batch with
    # its targets (a group whose problem reaches its target takes the next
    # queued one, so the launch time depends on the balance)
    from smili_b200 import autotune
    if args.ctas is not None:
        tuned = {"ctas_per_problem": args.ctas, "spread_bin": 8}
    elif args.no_autotune:
        tuned = {"ctas_per_problem": 0, "spread_bin": 8}
    else:
        tuned = autotune.tune(probs, 32, niter=args.niter, repeats=1, device=local,
                              cands=[(3, 8), (4, 8)], targets=targets[seed_of])
    # FP32 batched, inputs resident on the device: the reference's iteration
    # budget with an early exit at the plain solve's final cost.  The cold
    # arm starts every problem from its prior; the warm arm (the headline
    # when the trained weights are present) from the U-Net's proposal.
    opts = _lib.make_options(32, 1e-6, tuned["ctas_per_problem"], local, spread_bin=tuned["spread_bin"])
    ftarget = targets[seed_of]
    warm = (not args.no_warm) and os.path.exists(WARM_WEIGHTS)
    batch = _lib.Batch(probs, niter=args.niter, options=opts)
    batch.set_targets(ftarget)
    cold_warmup, cold_steps = (1, 2) if warm else (args.warmup, args.steps)
    for _ in range(cold_warmup):
        batch.run()
    if dist and not warm:
        dist.barrier()
    cold_times, cold_hits = [], []
    with ClockSampler(local) as clk:
        for _ in range(cold_steps):
            cold_times.append(batch.run())
            cold_hits.append(hits(batch, B))  # between timed launches, outside the events
    cold = quality(batch, B, seed_of)
    cold_nfg = sum(batch.fetch(p)[3]["nfg"] for p in range(B))
    cold_iters = int(sum(batch.fetch(p)[3]["niter"] for p in range(B)))
    cold["nfg_total"] = int(cold_nfg)
    cold["reached_target_per_step"] = cold_hits
    cold["ms_per_step"] = float(np.mean(cold_times))
    cold["value"] = world * float(np.mean(cold_hits)) / (cold["ms_per_step"] / 1000.0)
    # stage profile of one extra (untimed) cold step
    batch.profile(True)
    batch.run()
    stages = batch.stage_times()
    batch.profile(False)
    batch.close()

    h2d_prob = sum(arr.nbytes for p in probs for arr in p.keep.values())
    npix_all = sum(p.npix for p in probs)
    if warm:
        ws = WarmStart(probs, kws, seed_of, ftarget, args.niter, tuned["ctas_per_problem"], local)
        for _ in range(args.warmup):
            ws.step()
        if dist:
            dist.barrier()
        steps = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                steps.append(ws.step())
        ms_step = 1000.0 * float(np.mean([r["s"] for r in steps]))
        kernel_s = float(np.mean([r["kernel_s"] for r in steps]))
        step_hits = [r["hits"] for r in steps]
        fp32 = quality(ws, B, seed_of)
        nfg, iters = steps[-1]["nfg"], steps[-1]["iterations"]
        fp32["nfg_total"] = int(nfg)
        fp32["reached_target_per_step"] = step_hits
        fp32["parts_s"] = {k: float(np.mean([r["parts_s"][k] for r in steps])) for k in steps[0]["parts_s"]}
        ws.close()
        launches = UNET_FORWARD_LAUNCHES + 2 + WARM_HELPER_LAUNCHES
        # end to end from host buffers: packing and upload of the problems,
        # targets, iteration caps (twice) and keep flags; per-problem results
        # read after each launch; the final images, gradients and terms
        h2d = h2d_prob + B * (8 + 2 * 4 + 1)
        d2h = sum(2 * 8 * p.npix for p in probs) + B * (15 * 8 + 2 * PROB_RESULT_BYTES)
    else:
        ms_step, kernel_s = cold["ms_per_step"], cold["ms_per_step"] / 1000.0
        step_hits, fp32 = cold_hits, cold
        nfg, iters = cold_nfg, cold_iters
        launches = 1
        h2d = h2d_prob + B * 8
        d2h = sum(2 * 8 * p.npix for p in probs) + B * (15 * 8 + PROB_RESULT_BYTES)
    reached = float(np.mean(step_hits))

    # end to end through the C ABI from host buffers
    e2e_times, e2e_hits = [], []
    for _ in range(max(0, args.e2e_steps)):
        t0 = time.perf_counter()
        if warm:
            w2 = WarmStart(probs, kws, seed_of, ftarget, args.niter, tuned["ctas_per_problem"], local)
            r = w2.step()
            for p in range(B):
                w2.fetch(p)
            w2.close()
            e2e_hits.append(r["hits"])
        else:
            b2 = _lib.Batch(probs, niter=args.niter, options=opts)
            b2.set_targets(ftarget)
            b2.run()
            got = [b2.fetch(p) for p in range(B)]
            b2.close()
            e2e_hits.append(int(sum(g[3]["task"] == _lib.TASK_TARGET for g in got)))
        e2e_times.append(time.perf_counter() - t0)

    e2e_mean = float(np.mean(e2e_times)) if e2e_times else float("nan")
    max_ms, e2e_s = max_over_ranks(dist, ms_step, e2e_mean, "cuda")
    # a solve counts when it reaches its plain FP64 solve's final cost
    # (x (1 + target_rtol)) within the plain solver's iteration budget;
    # value_all counts every solve of the launch
    value_all, value, _ = job_values(world, B, reached, max_ms, e2e_s)
    e2e_value = world * float(np.mean(e2e_hits)) / e2e_s if e2e_hits else float("nan")
    bfg = fg_bytes(kws[0], 4)
    achieved = bfg * nfg / kernel_s / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": max_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD.format(niter=args.niter, rtol=args.target_rtol),
                       "batch": B, "distinct_seeds": S,
                       "launch": {"ctas_per_problem": tuned["ctas_per_problem"],
                                  "spread_bin": tuned["spread_bin"],
                                  "chosen_by": ("fixed (--ctas)" if args.ctas is not None else
                                                "automatic" if args.no_autotune else
                                                "autotuner (whole solves of this batch with its targets)"),
                                  "autotune_ms": [r["ms"] for r in tuned.get("table", [])]},
                       "precision": "FP32 transforms + compensated chi-square, FP64 L-BFGS-B",
                       "warm_start": ("learned (smili_b200/warmstart/unet_closure256.npz): the U-Net's "
                                      f"proposal from the image after {WARM_K} FP32 iterations starts the "
                                      "remaining iterations; its time is inside value" if warm else
                                      "none (cold starts from the prior)"),
                       "l2": "inputs larger than L2 (batch footprint >> 126 MB)",
                       "parallelism": f"replicas x{world}"},
            "value_all": value_all,
            "value_cold": cold["value"],
            "quality_fp32_cold": cold,
            "plain_fp64": {"value": 1000.0 * S / float(np.sum(plain_ms)), "unit": "solves/s",
                           "ms_per_solve": float(np.mean(plain_ms)),
                           "nfg_mean": float(np.mean(plain_nfg)),
                           "nrmse_vs_truth_median": float(np.median(plain_nrmse))},
            "quality_fp32": fp32,
            "quality_fp64_control": control,
            "quality_fp64_control_perturbed_start": control_pert,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": DRAM_BYTES_PER_EVAL_FP32 * nfg / 1e9,
                         "traffic_unit": "GB per launch (ncu, scaled by evaluations)",
                         "kernel": "smili_batch_kernel<float> (persistent solve)",
                         "algorithmic_bytes_per_eval": bfg, "evals_per_step": nfg,
                         "kernel_s_per_step": kernel_s,
                         "peak_source": "measured" if peaks else "fallback"},
            "roofline_with_optimizer": {
                "bound": "hbm", "unit": "GB/s", "peak": peak,
                "achieved": (bfg * nfg + lb_bytes_per_iteration(kws[0]) * iters) / kernel_s / 1e9,
                "frac": (bfg * nfg + lb_bytes_per_iteration(kws[0]) * iters) / kernel_s / 1e9 / peak,
                "bytes_per_iteration_lbfgsb": lb_bytes_per_iteration(kws[0]), "iterations_per_launch": iters},
            "gpu_launches": launches * args.steps,
            "clocks": clk.summary(),
            "stage_ms_problem0": {k: round(v, 3) for k, v in stages.items()},
        }
        if args.config5:
            line["dynamic_cfg5"] = dynamic_cfg5(args.niter, local)
            line["large_cfg5"] = large_cfg5(args.niter, local)
        if args.survey > 0:
            line["survey_cfg3"] = survey_cfg3(args.survey, args.niter, local)
        if args.warm_problems > 0:
            line["warm_start_cfg4"] = warm_start_cfg4(args.warm_problems, args.niter, args.target_rtol, local)
        if not args.no_cpu:
            line["cpu_baseline"] = cpu_baseline(kws[0], args.ref_iters, plain_nfg_table()[0][0])
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
