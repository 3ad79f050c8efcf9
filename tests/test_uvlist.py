"""get_uvlist against golden vectors produced by the reference's own code
(tests/golden/make_golden.py runs smili/uvdata/uvtable/tools.py)."""
import glob
import os

import numpy as np
import pandas as pd
import pytest

from smili_b200.uvdata.tools import get_uvlist

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "uvlist_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p) for p in GOLD])
def test_uvlist_matches_reference(path):
    z = np.load(path)
    tabs = {}
    for k in z.files:
        if "__" in k:
            t, c = k.split("__")
            tabs.setdefault(t, {})[c] = z[k]
    args = {name: (pd.DataFrame(tabs[key]) if key in tabs else None)
            for name, key in [("fcvtable", "fcv"), ("amptable", "amp"), ("bstable", "bs"),
                              ("catable", "ca")]}
    out = get_uvlist(**args)
    for got, name in zip(out, ["u", "v", "uvidxfcv", "uvidxamp", "uvidxcp", "uvidxca"]):
        np.testing.assert_array_equal(np.asarray(got), z[name], err_msg=name)


def test_uvlist_no_data_returns_minus_one():
    assert get_uvlist() == -1


def test_golden_fixture_count():
    assert len(GOLD) >= 6


def test_uvlist_loop_matches_reference():
    """get_uvlist_loop (movies) against the reference's output on a 5-frame
    movie whose frame 2 has no data (Nuvs[2] == 0)."""
    from smili_b200.uvdata.tools import get_uvlist_loop
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "uvlistloop_fcv_cp.npz"))
    tabs = {}
    for k in z.files:
        if "__" in k:
            t, c = k.split("__")
            tabs.setdefault(t, {})[c] = z[k]
    out = get_uvlist_loop(5, fcvconcat=pd.DataFrame(tabs["fcv"]), bsconcat=pd.DataFrame(tabs["bs"]))
    for got, name in zip(out, ["u", "v", "uvidxfcv", "uvidxamp", "uvidxcp", "uvidxca", "nuvs"]):
        np.testing.assert_array_equal(np.asarray(got), z[name], err_msg=name)
