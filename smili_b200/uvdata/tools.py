"""Non-redundant uv list and signed uv indices for the imaging data terms.

Mirrors ``get_uvlist`` (smili/uvdata/uvtable/tools.py:12-132): the uv points
of all data terms are stacked in the order fcv, amp, cp (uv12, uv23, uv31),
ca (uv1..uv4); points with v < 0 are replaced by (-u, -v) and carry sign -1;
the unique points are sorted lexicographically (u, then v) as ``np.unique``
sorts complex numbers; each datum gets ``sign * (1 + position in the unique
list)``.  Closure index arrays come back as (3, Ncp) and (4, Nca) in Fortran
order, absent tables as 1-element zero dummies, exactly like the reference.
"""
from __future__ import annotations

import numpy as np


def _fold(u: np.ndarray, v: np.ndarray):
    u = np.array(u, dtype=np.float64, copy=True)
    v = np.array(v, dtype=np.float64, copy=True)
    sign = np.ones(u.size, dtype=np.int64)
    neg = v < 0
    u[neg] *= -1
    v[neg] *= -1
    sign[neg] = -1
    return u, v, sign


def _cols(table, names):
    return [np.asarray(table[n]).astype(np.float64) for n in names]


def _unique_host(ustack, vstack):
    """Fold, list the distinct points (u, then v) and index them, in numpy."""
    ustack, vstack, sstack = _fold(ustack, vstack)
    # lexicographic unique on (u, v): the order numpy uses for complex values
    order = np.lexsort((vstack, ustack))
    us_sorted, vs_sorted = ustack[order], vstack[order]
    new = np.ones(order.size, dtype=bool)
    new[1:] = (us_sorted[1:] != us_sorted[:-1]) | (vs_sorted[1:] != vs_sorted[:-1])
    rank = np.cumsum(new) - 1
    inverse = np.empty(order.size, dtype=np.int64)
    inverse[order] = rank
    return us_sorted[new], vs_sorted[new], (inverse + 1) * sstack


def _unique_device(ustack, vstack, device):
    """The same on the GPU (smili_get_uvlist)."""
    import ctypes as C
    from .. import _lib
    u = np.ascontiguousarray(ustack, dtype=np.float64)
    v = np.ascontiguousarray(vstack, dtype=np.float64)
    n = u.size
    uo, vo = np.empty(n), np.empty(n)
    idx = np.empty(n, dtype=np.int32)
    m = C.c_int(0)
    opt = _lib.make_options(64, 0.0, 0, int(device))
    _lib.check(_lib.lib().smili_get_uvlist(n, _lib.dptr(u), _lib.dptr(v), C.byref(opt), C.byref(m),
                                           _lib.dptr(uo), _lib.dptr(vo),
                                           idx.ctypes.data_as(C.POINTER(C.c_int))))
    return uo[:m.value].copy(), vo[:m.value].copy(), idx.astype(np.int64)


def get_uvlist(fcvtable=None, amptable=None, bstable=None, catable=None, device=None):
    """Return ``(u, v, uvidxfcv, uvidxamp, uvidxcp, uvidxca)``.

    ``device``: None lists the points with numpy on the host; a CUDA device
    ordinal does the folding, sorting and indexing on that GPU
    (``smili_get_uvlist``), with identical results.  Returns -1 (after
    printing an error) when no table is given, as the reference does
    (tools.py:15-18).
    """
    if fcvtable is None and amptable is None and bstable is None and catable is None:
        print("Error: No data are input.")
        return -1
    us, vs = [], []
    counts = {"fcv": 0, "amp": 0, "cp": 0, "ca": 0}
    if fcvtable is not None:
        u, v = _cols(fcvtable, ["u", "v"])
        us.append(u)
        vs.append(v)
        counts["fcv"] = u.size
    if amptable is not None:
        u, v = _cols(amptable, ["u", "v"])
        us.append(u)
        vs.append(v)
        counts["amp"] = u.size
    if bstable is not None:
        cols = _cols(bstable, ["u12", "v12", "u23", "v23", "u31", "v31"])
        us.extend(cols[0::2])
        vs.extend(cols[1::2])
        counts["cp"] = cols[0].size
    if catable is not None:
        cols = _cols(catable, ["u1", "v1", "u2", "v2", "u3", "v3", "u4", "v4"])
        us.extend(cols[0::2])
        vs.extend(cols[1::2])
        counts["ca"] = cols[0].size

    ustack = np.concatenate(us)
    vstack = np.concatenate(vs)
    if device is None:
        u, v, uvidx = _unique_host(ustack, vstack)
    else:
        u, v, uvidx = _unique_device(ustack, vstack, device)

    nf, na, nc, nq = counts["fcv"], counts["amp"], counts["cp"], counts["ca"]
    uvidxfcv = uvidx[:nf] if fcvtable is not None else np.zeros(1, dtype=np.int32)
    uvidxamp = uvidx[nf:nf + na] if amptable is not None else np.zeros(1, dtype=np.int32)
    if bstable is not None:
        uvidxcp = uvidx[nf + na:nf + na + 3 * nc].reshape([nc, 3], order="F").transpose()
    else:
        uvidxcp = np.zeros([3, 1], dtype=np.int32, order="F")
    if catable is not None:
        s0 = nf + na + 3 * nc
        uvidxca = uvidx[s0:s0 + 4 * nq].reshape([nq, 4], order="F").transpose()
    else:
        uvidxca = np.zeros([4, 1], dtype=np.int32, order="F")
    return (u, v, uvidxfcv, uvidxamp, uvidxcp, uvidxca)


def get_uvlist_loop(Nt, fcvconcat=None, ampconcat=None, bsconcat=None, caconcat=None):
    """Per-frame uv lists of a movie, concatenated (tools.py:255-335).

    Every table carries a ``frmidx`` column; frame i's rows go through
    ``get_uvlist`` on their own and the frame's indices are offset by the
    number of uv points of the frames before it.  Returns ``(u, v, uvidxfcv,
    uvidxamp, uvidxcp, uvidxca, Nuvs)``; the data rows must be ordered by
    frame, as the index arrays are concatenated frame by frame.
    """
    if fcvconcat is None and ampconcat is None and bsconcat is None and caconcat is None:
        print("Error: No data are input.")
        return -1
    u, v = [], []
    idx = {"fcv": [], "amp": [], "cp": [], "ca": []}
    Nuvs = []
    offset = 0
    for i in range(Nt):
        parts = {}
        for key, tab in (("fcv", fcvconcat), ("amp", ampconcat), ("cp", bsconcat), ("ca", caconcat)):
            if tab is None:
                continue
            rows = np.where(np.asarray(tab["frmidx"]) == i)[0]
            if rows.size:
                parts[key] = tab.iloc[rows]
        if not parts:
            Nuvs.append(0)
            continue
        u0, v0, ifcv, iamp, icp, ica = get_uvlist(fcvtable=parts.get("fcv"), amptable=parts.get("amp"),
                                                  bstable=parts.get("cp"), catable=parts.get("ca"))
        u.append(u0)
        v.append(v0)
        Nuvs.append(len(u0))
        for key, arr in (("fcv", ifcv), ("amp", iamp), ("cp", icp), ("ca", ica)):
            if key in parts:
                idx[key].append(np.sign(arr) * (np.abs(arr) + offset))
        offset += len(u0)
    u = np.concatenate(u)
    v = np.concatenate(v)
    uvidxfcv = np.concatenate(idx["fcv"]) if fcvconcat is not None else np.zeros(1, dtype=np.int32)
    uvidxamp = np.concatenate(idx["amp"]) if ampconcat is not None else np.zeros(1, dtype=np.int32)
    uvidxcp = np.hstack(idx["cp"]) if bsconcat is not None else np.zeros([3, 1], dtype=np.int32, order="F")
    uvidxca = np.hstack(idx["ca"]) if caconcat is not None else np.zeros([4, 1], dtype=np.int32, order="F")
    return u, v, uvidxfcv, uvidxamp, uvidxcp, uvidxca, np.asarray(Nuvs)
