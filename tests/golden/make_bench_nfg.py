"""Whole plain solves of the benchmark's seeds by the CPU restatement.

The benchmark (``bench.py``) solves 16 seeded 256x256 / 97 200-visibility
problems (``synth.precision_path(seed=1000 + s)``, amplitudes + closure
phases + log closure amplitudes, l1 / TV / MEM = 1 / 1 / 0.1, L-BFGS-B m=5,
1000 iterations, NUFFT tolerance 1e-6, FP64).  Its reference arm times
bounded samples of the CPU restatement (``oracle/``) and needs the number of
function/gradient evaluations that a whole plain solve of each seed takes to
turn seconds per evaluation into solves per second.  This script runs those
whole solves once with the oracle and writes ``bench_plain_nfg.json``:
per seed the evaluation count, iteration count, task code, final cost and
wall time, with the host thread count.

Usage::

    python tests/golden/make_bench_nfg.py [nseeds]
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main(nseed=16, niter=1000):
    from oracle import oracle as O
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    O.build()
    rows = []
    for s in range(nseed):
        obs = synth.precision_path(seed=1000 + s, niter=niter)
        kw, _ = prepare_imaging(obs.image, amptable=obs.amptable, bstable=obs.bstable,
                                catable=obs.catable, niter=niter, **obs.reg)
        t0 = time.perf_counter()
        _, terms, info = O.imaging(kw, eps=1e-6)
        dt = time.perf_counter() - t0
        rows.append({"seed": 1000 + s, "nfg": int(info["nfg"]), "niter": int(info["niter"]),
                     "task": int(info["task"]), "cost": float(terms["cost"]), "wall_s": dt})
        print(rows[-1], flush=True)
        out = {"workload": "synth.precision_path(seed=1000+s), 256x256, 97 200 uv points, amp + cp + lca, "
                           "l1/TV/MEM = 1/1/0.1, L-BFGS-B m=5, niter 1000, NUFFT eps 1e-6, FP64 (oracle)",
               "threads": int(O.lib().orc_nthreads()), "solves": rows,
               "nfg_mean": sum(r["nfg"] for r in rows) / len(rows)}
        with open(os.path.join(HERE, "bench_plain_nfg.json"), "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 16)
