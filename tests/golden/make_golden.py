"""Generate golden fixtures by running the reference's own pure-Python code.

Only ``get_uvlist`` (smili/uvdata/uvtable/tools.py:12-132) on the imaging
path is runnable here: it needs nothing but numpy.  The reference package's
``__init__`` pulls in astropy/matplotlib, which are absent, so the module is
loaded straight from its file.  Everything else on the path is Fortran plus
FINUFFT and cannot be built in this image (no Fortran compiler, no FINUFFT).

Usage (in a container that has the reference checkout)::

    python tests/golden/make_golden.py /path/to/reference

or with $SMILI_REFERENCE_ROOT set and no argument.

writes ``tests/golden/uvlist_*.npz`` (inputs and reference outputs).
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from smili_b200 import synth  # noqa: E402


def load_reference_tools(ref_root: str):
    path = os.path.join(ref_root, "smili", "uvdata", "uvtable", "tools.py")
    spec = importlib.util.spec_from_file_location("ref_uvtable_tools", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _save(name, tables, out):
    arrays = {}
    for key, tab in tables.items():
        if tab is None:
            continue
        for col in tab.columns:
            if col.startswith("u") or col.startswith("v"):
                arrays[f"{key}__{col}"] = np.asarray(tab[col], dtype=np.float64)
    u, v, ifcv, iamp, icp, ica = out
    np.savez_compressed(os.path.join(HERE, f"uvlist_{name}.npz"), u=u, v=v,
                        uvidxfcv=np.asarray(ifcv), uvidxamp=np.asarray(iamp),
                        uvidxcp=np.asarray(icp), uvidxca=np.asarray(ica), **arrays)


def main(ref_root: str):
    ref = load_reference_tools(ref_root)
    cases = {}
    # 1) small crescent: fcv + closure phases (conjugations on ~half the points)
    o = synth.small_crescent(seed=0)
    cases["fcv_cp"] = {"fcv": o.vistable.iloc[:600].reset_index(drop=True),
                       "bs": o.bstable.iloc[:400].reset_index(drop=True)}
    # 2) amplitudes + closure phases + closure amplitudes (shared uv points)
    p = synth.precision_path(seed=5, nx=32, nst=6, hours=2.0, scan_s=600.0)
    cases["amp_cp_ca"] = {"amp": p.amptable, "bs": p.bstable, "ca": p.catable}
    # 3) single-table cases and duplicated / v == 0 / v < 0 edge points
    import pandas as pd
    edge = pd.DataFrame({"u": [1.0, -1.0, 1.0, 0.0, -2.0, 2.0, 1.0],
                         "v": [2.0, -2.0, 2.0, 0.0, 0.0, -0.0, -3.0],
                         "amp": 1.0, "phase": 0.0, "sigma": 1.0})
    cases["edge_fcv"] = {"fcv": edge}
    cases["edge_amp"] = {"amp": edge}
    cases["cp_only"] = {"bs": o.bstable.iloc[:50].reset_index(drop=True)}
    cases["ca_only"] = {"ca": p.catable.iloc[:40].reset_index(drop=True)}
    for name, t in cases.items():
        out = ref.get_uvlist(fcvtable=t.get("fcv"), amptable=t.get("amp"),
                             bstable=t.get("bs"), catable=t.get("ca"))
        _save(name, t, out)
        print(name, "nuv", len(out[0]))
    # 4) movies: get_uvlist_loop (tools.py:255-335) over frame-tagged tables,
    #    frame 2 without data
    m = synth.dynamic_problem(seed=3, nframes=5, nx=32, nst=6, vis_per_frame=60)
    keep_v = m.vistable[m.vistable.frmidx != 2].reset_index(drop=True)
    keep_b = m.bstable[m.bstable.frmidx != 2].reset_index(drop=True)
    out = ref.get_uvlist_loop(Nt=5, fcvconcat=keep_v, bsconcat=keep_b)
    arrays = {}
    for key, tab in (("fcv", keep_v), ("bs", keep_b)):
        for col in tab.columns:
            if col.startswith("u") or col.startswith("v") or col == "frmidx":
                arrays[f"{key}__{col}"] = np.asarray(tab[col], dtype=np.float64)
    u, v, ifcv, iamp, icp, ica, nuvs = out
    np.savez_compressed(os.path.join(HERE, "uvlistloop_fcv_cp.npz"), u=u, v=v, uvidxfcv=np.asarray(ifcv),
                        uvidxamp=np.asarray(iamp), uvidxcp=np.asarray(icp), uvidxca=np.asarray(ica),
                        nuvs=np.asarray(nuvs), **arrays)
    print("loop nuv", len(u), "nuvs", list(nuvs))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SMILI_REFERENCE_ROOT")
    if not root:
        raise SystemExit("usage: make_golden.py REFERENCE_ROOT (or set $SMILI_REFERENCE_ROOT)")
    main(root)
