"""``fortlib.coord``: baseline vectors to uvw (src/fortlib/coord.f90:9-60)."""
from __future__ import annotations

import numpy as np


def calc_uvw(gst, alpha, delta, dx, dy, dz, Ndata=None):
    """(u, v, w) of baseline vectors (dx, dy, dz) in the Earth-fixed frame at
    Greenwich sidereal time ``gst`` (hours) toward (alpha, delta) (rad):
    the baseline is rotated by the hour angle gst pi / 12 - alpha, then
    u = y, v = -x sin(delta) + z cos(delta), w = x cos(delta) + z sin(delta)."""
    arrs = [np.asarray(a, dtype=np.float64) for a in (gst, alpha, delta, dx, dy, dz)]
    if Ndata is not None:
        arrs = [a[:int(Ndata)] if a.ndim else a for a in arrs]
    gst, alpha, delta, dx, dy, dz = arrs
    gh = gst * np.pi / 12 - alpha
    cosgh, singh = np.cos(gh), np.sin(gh)
    blx = cosgh * dx - singh * dy
    bly = singh * dx + cosgh * dy
    blz = dz
    return bly, -blx * np.sin(delta) + blz * np.cos(delta), blx * np.cos(delta) + blz * np.sin(delta)
