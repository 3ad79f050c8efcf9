"""The roofline numerators of the benchmark line, recomputed from the
workload's data counts: the compulsory bytes of one function/gradient
evaluation in FP32 (image in and gradient out, uv coordinates, each datum's
value, variance and signed uv indices, one weight image per weighted
regularizer) and of one L-BFGS-B iteration ((4m + 10) n doubles)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_compulsory_bytes_of_the_256x256_workload():
    sys.path.insert(0, ROOT)
    import bench
    from smili_b200 import synth
    from smili_b200.imaging.lbfgs import prepare_imaging
    # the data counts do not depend on the model values: unit visibilities keep this fast
    obs = synth.precision_path(seed=1000, niter=1000,
                               model=lambda truth, im, u, v: np.ones(u.size, dtype=complex))
    kw, _ = prepare_imaging(obs.image, amptable=obs.amptable, bstable=obs.bstable, catable=obs.catable,
                            niter=1000, **obs.reg)
    npix, nuv = 256 * 256, 97200
    namp, ncp, nca = 97200, 77760, 75600
    assert int(kw["npix"]) == npix and np.size(kw["u"]) == nuv
    s = 4
    want = (s * 2 * npix + s * 2 * nuv + namp * (2 * s + 4) + ncp * (2 * s + 12) + nca * (2 * s + 16)
            + s * npix * 3)  # l1, TV and MEM weights
    assert bench.fg_bytes(kw, s) == want == 6624320
    assert bench.lb_bytes_per_iteration(kw, 5) == (4 * 5 + 10) * npix * 8 == 15728640
