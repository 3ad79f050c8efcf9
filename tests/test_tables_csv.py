"""uv-data tables through CSV files (read_vistable / read_bstable /
read_catable and to_csv), and the argument checks of the device uv list,
without a GPU."""
import ctypes as C
import os

import numpy as np
import pandas as pd
import pytest

from conftest import make_kw

from reference_dropin import reference_root

# the reference's example tables, when $SMILI_REFERENCE_ROOT names a checkout
EXAMPLES = os.path.join(reference_root() or "", "docs", "examples", "uvdata")


def _roundtrip(tab, reader, tmp_path, name):
    from smili_b200.uvdata import tables
    path = tmp_path / f"{name}.csv"
    tables.to_csv(tab, path)
    back = reader(path)
    assert list(back.columns) == list(tab.columns)
    for c in tab.columns:
        assert np.array_equal(np.asarray(back[c]), np.asarray(tab[c])), c  # float64 round-trips exactly
    return back


def test_csv_roundtrip_gives_the_same_imaging_inputs(crescent32, closure40, tmp_path):
    from smili_b200.imaging.lbfgs import prepare_imaging
    from smili_b200.uvdata import tables
    for name, o in (("crescent", crescent32), ("closure", closure40)):
        tabs = {}
        for key, reader, kind in (("vistable", tables.read_vistable, "vis"), ("amptable", tables.read_vistable, "amp"),
                                  ("bstable", tables.read_bstable, "bs"), ("catable", tables.read_catable, "ca")):
            tab = getattr(o, key)
            if tab is None:
                continue
            assert tables.missing_columns(tab, kind) == []
            tabs[key] = _roundtrip(tab, reader, tmp_path, f"{name}_{key}")
        kw0 = make_kw(o)
        kw1, _ = prepare_imaging(o.image, niter=50, **tabs, **o.reg)
        for k, v in kw0.items():
            if isinstance(v, np.ndarray):
                assert np.array_equal(v, kw1[k]), k
            else:
                assert v == kw1[k], k


@pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="the reference's example tables are not on this machine")
def test_reference_example_tables_read():
    """The reference's own example CSVs (3C 273 at 43 GHz) read with the
    columns the imaging path needs, and list their uv points."""
    from smili_b200.uvdata import tables, tools
    vis = tables.read_vistable(os.path.join(EXAMPLES, "visibility.csv"))
    bs = tables.read_bstable(os.path.join(EXAMPLES, "cphase.csv"))
    ca = tables.read_catable(os.path.join(EXAMPLES, "logcamp.csv"))
    assert (len(vis), len(bs), len(ca)) == (7648, 5868, 5620)
    assert list(vis.columns) == tables.VIS_COLUMNS
    assert list(bs.columns) == tables.BS_COLUMNS
    assert list(ca.columns) == tables.CA_COLUMNS
    assert pd.api.types.is_datetime64_any_dtype(vis["utc"])
    for t, kind in ((vis, "vis"), (bs, "bs"), (ca, "ca")):
        assert tables.missing_columns(t, kind) == []
    u, v, ifcv, _, icp, ica = tools.get_uvlist(fcvtable=vis, bstable=bs, catable=ca)
    assert np.all(v >= 0) and icp.shape == (3, len(bs)) and ica.shape == (4, len(ca))
    # every datum points at its own (folded) uv point
    assert np.allclose(u[np.abs(ifcv) - 1] * np.sign(ifcv), vis["u"]) and np.allclose(v[np.abs(ifcv) - 1] * np.sign(ifcv), vis["v"])


def test_device_uvlist_rejects_bad_input_without_a_device():
    from smili_b200 import _lib
    u = np.array([1.0, np.nan])
    v = np.zeros(2)
    n = C.c_int(0)
    out = np.zeros(2)
    idx = np.zeros(2, dtype=np.int32)
    args = (_lib.dptr(u), _lib.dptr(v), None, C.byref(n), _lib.dptr(out), _lib.dptr(out),
            idx.ctypes.data_as(C.POINTER(C.c_int)))
    assert _lib.lib().smili_get_uvlist(0, *args) == -1   # SMILI_ERR_ARG
    assert _lib.lib().smili_get_uvlist(2, *args) == -2   # SMILI_ERR_DATA: non-finite u
