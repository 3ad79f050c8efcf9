"""Record what the reference's own imaging driver passes to ``fortlib``.

Runs ``smili/imaging/lbfgs.py:imaging`` from a reference checkout (loaded by
path, see ``tests/reference_dropin.py``) on the driver cases of
``reference_dropin.cases()``.  ``fortlib.image`` is this project's mirror and
``fortlib.fftim2d.imaging`` records its keyword arguments and returns the CPU
oracle's solve at the reference's NUFFT tolerance 1e-6.  Each case is saved
as ``tests/golden/dropin_<case>.npz``: the driver's inputs, the recorded
kwargs (``kw__*``) and the image the reference's driver returned
(``out__data``).

Usage (in a container that has the reference checkout)::

    SMILI_REFERENCE_ROOT=/path/to/reference python tests/golden/make_dropin.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

import reference_dropin as R  # noqa: E402


def main():
    root = R.reference_root()
    if root is None:
        raise SystemExit(f"set ${R.ENV} to a reference checkout")
    for name, init, opts in R.cases():
        fresh = {k: (v.copy() if hasattr(v, "copy") else v) for k, v in opts.items()}
        fl = R.RecordingFortlib(R.oracle_solve(1e-6))
        with R.reference_lbfgs(root, fl) as ref:
            out = ref.imaging(init.copy(), **fresh)
        assert len(fl.calls) == 1
        path = os.path.join(HERE, f"dropin_{name}.npz")
        R.save_case(path, init, opts, fl.calls[0])
        z = dict(np.load(path))
        z["out__data"] = np.asarray(out.data)
        np.savez_compressed(path, **z)
        print(name, "npix", fl.calls[0]["npix"], "nuv", np.size(fl.calls[0]["u"]),
              os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
