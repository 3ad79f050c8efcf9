"""Launch-shape autotuner for batched solves.

Two launch parameters decide how fast a batch runs and neither has a good
closed form: how many CTAs cooperate on one problem (``ctas_per_problem``:
more CTAs shorten each problem's barrier-separated stages but leave fewer
problems resident) and the side of the spreading tiles (``spread_bin``: 8 or
16 fine-grid cells; larger tiles amortise the subgrid flush over more
points but need more shared memory and waste more lanes on sparse tiles).
``tune`` times short solves of the caller's own batch for every candidate
(device time from CUDA events, the median of ``repeats`` launches) and
returns the fastest.  Results are cached in memory by the batch's shape.

With objective ``targets`` (one per problem), problems leave the launch at
different iterations and a group that finishes takes the next queued
problem, so short solves no longer predict the launch time: the candidates
are then timed on whole solves with those targets, and the one with the
shortest launch wins.
"""
from __future__ import annotations

import numpy as np

from . import _lib

_cache: dict = {}


def _key(kws, precision):
    kws = [k.kw if isinstance(k, _lib.Problem) else k for k in kws]
    sizes = tuple(sorted((int(k["nx"]), int(np.size(k["u"])) // 10000) for k in kws))
    return (precision, len(kws), sizes[:4], sizes[-4:])


def candidates(nprob, precision, max_res=None):
    """(ctas_per_problem, spread_bin) pairs worth timing for nprob problems:
    group sizes from one CTA per problem up to the size that still keeps
    every problem resident, times both tile sides."""
    max_res = max_res or 296  # two CTAs per SM in both precisions (512 threads FP32, 256 FP64)
    gs = sorted({g for g in (1, 2, 3, 4, 6, 8, 12, 16) if g * nprob <= 2 * max_res} | {1})
    return [(g, b) for g in gs for b in (8, 16)]


def tune(kws, precision=32, niter=20, repeats=3, device=0, nufft_eps=1e-6, cands=None, verbose=False,
         targets=None):
    """Time ``niter``-iteration solves of the batch ``kws`` for each
    candidate and return {"ctas_per_problem", "spread_bin", "ms_per_problem_eval", "table"}.
    ``targets``: objective targets per problem (whole solves; the shortest
    launch wins, and no warm-up launch is made)."""
    key = _key(kws, precision)
    if cands is None and targets is None and key in _cache:
        return _cache[key]
    probs = [p if isinstance(p, _lib.Problem) else _lib.Problem(p) for p in kws]
    table = []
    for g, b in (cands or candidates(len(probs), precision)):
        opts = _lib.make_options(precision, nufft_eps, g, device, spread_bin=b)
        batch = _lib.Batch(probs, niter=niter, options=opts)
        if targets is None:
            batch.run()  # warm-up
        else:
            batch.set_targets(targets)
        times = [batch.run() for _ in range(repeats)]
        nfg = sum(batch.fetch(p)[3]["nfg"] for p in range(len(probs)))
        batch.close()
        ms = float(np.median(times))
        table.append({"ctas_per_problem": g, "spread_bin": b, "ms": ms, "ms_per_problem_eval": ms / max(nfg, 1)})
        if verbose:
            print(table[-1], flush=True)
    best = min(table, key=lambda r: r["ms"] if targets is not None else r["ms_per_problem_eval"])
    out = {"ctas_per_problem": best["ctas_per_problem"], "spread_bin": best["spread_bin"],
           "ms_per_problem_eval": best["ms_per_problem_eval"], "table": table}
    if cands is None and targets is None:
        _cache[key] = out
    return out
