"""Seeded synthetic VLBI observations for the static-imaging workloads.

There is no public data set behind the imaging benchmark, so every workload
is generated here from a seed.  The conventions follow SMILI:

* station positions are random points on a 6371 km sphere (ECEF metres);
* u, v come from the baseline vector rotated by the Greenwich hour angle
  exactly as ``calc_uvw`` does it (src/fortlib/coord.f90:37-59);
* the image grid follows IMFITS: ``dx < 0`` (RA grows to the left), pixel
  ``(ix, iy)`` (1-based) sits at ``x = dx*(ix - nxref)``, ``y = dy*(iy - nyref)``
  with ``nxref = (nx+1)/2`` (smili/imdata/imdata.py:151-162);
* visibilities use the "+" Fourier sign of fortlib
  (V = sum I exp(+2 pi i (u x + v y)); src/wrapfinufft/wrapfinufft.f90:114-124);
* closure phases use independent triangles (0, i, j) with uv31 = -uv13 and
  sigma_cp = amp_B * sqrt(sum (sigma/amp)^2)
  (smili/uvdata/uvtable/vistable.py:925-930, 949-952);
* log closure amplitudes use N(N-3)/2 independent quadrangles with
  logsigma = sqrt(sum 1/rho^2), rho^2 = max(1, snr^2 - 1)
  (vistable.py:1769-1779).

Model visibilities are an exact DFT of the pixelised truth computed with a
numpy GEMM, so the generator depends on neither the oracle nor the kernels.
Tables are pandas DataFrames carrying the column names SMILI's VisTable,
BSTable and CATable use, so they feed the ``imaging`` driver unchanged.
"""
from __future__ import annotations

import dataclasses
import itertools
import math
from typing import Optional

import numpy as np
import pandas as pd

C_LIGHT = 299792458.0
EARTH_R = 6371e3
UAS = np.deg2rad(1.0 / 3600.0 / 1e6)  # one micro-arcsecond in radians


# ----------------------------------------------------------------------------
# image container (the subset of IMFITS that the imaging driver touches)
# ----------------------------------------------------------------------------
class Image:
    """Minimal stand-in for ``smili.imdata.IMFITS`` used by ``imaging``.

    ``data`` has IMFITS' shape ``[nstokes, nfreq, ny, nx]``; ``header`` holds
    ``nx, ny, nxref, nyref`` and ``dx, dy`` in degrees (dx negative).
    """

    def __init__(self, nx: int, ny: int, dx_uas: float, dy_uas: Optional[float] = None,
                 nxref: Optional[float] = None, nyref: Optional[float] = None):
        if dy_uas is None:
            dy_uas = dx_uas
        self.angunit = "uas"
        self.header = {
            "nx": int(nx), "ny": int(ny),
            "nxref": float((nx + 1) / 2.0 if nxref is None else nxref),
            "nyref": float((ny + 1) / 2.0 if nyref is None else nyref),
            "dx": -abs(dx_uas) / 3600.0 / 1e6,
            "dy": abs(dy_uas) / 3600.0 / 1e6,
        }
        self.data = np.zeros((1, 1, ny, nx), dtype=np.float64)

    def angconv(self, unit1: str, unit2: str) -> float:
        scale = {"deg": 1.0, "rad": 180.0 / np.pi, "uas": 1.0 / 3600.0 / 1e6,
                 "mas": 1.0 / 3600.0 / 1e3, "arcsec": 1.0 / 3600.0}
        return scale[unit1] / scale[unit2]

    def get_xygrid(self, twodim: bool = False, angunit: str = "rad"):
        h = self.header
        conv = self.angconv("deg", angunit)
        x = h["dx"] * conv * (np.arange(h["nx"]) + 1 - h["nxref"])
        y = h["dy"] * conv * (np.arange(h["ny"]) + 1 - h["nyref"])
        if twodim:
            return np.meshgrid(x, y)
        return x, y

    def update_fits(self) -> None:  # IMFITS keeps a FITS HDU in sync; nothing to do here
        return None

    def copy(self) -> "Image":
        out = Image(self.header["nx"], self.header["ny"], 1.0)
        out.header = dict(self.header)
        out.data = self.data.copy()
        out.angunit = self.angunit
        return out

    def __deepcopy__(self, memo):
        return self.copy()


def xy_rad(img: Image):
    """Pixel-centre coordinates (radians) as 2-D arrays ``(x, y)`` of shape (ny, nx)."""
    return img.get_xygrid(twodim=True, angunit="rad")


# ----------------------------------------------------------------------------
# truth images
# ----------------------------------------------------------------------------
def gaussian_image(img: Image, fwhm_uas: float, flux: float,
                   x0_uas: float = 0.0, y0_uas: float = 0.0) -> np.ndarray:
    x, y = xy_rad(img)
    sig = fwhm_uas * UAS / math.sqrt(8 * math.log(2))
    g = np.exp(-((x - x0_uas * UAS) ** 2 + (y - y0_uas * UAS) ** 2) / (2 * sig * sig))
    return g * (flux / g.sum())


def _gauss_blur(a: np.ndarray, sigma_pix: float) -> np.ndarray:
    ny, nx = a.shape
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.fftfreq(nx)[None, :]
    h = np.exp(-2 * np.pi ** 2 * sigma_pix ** 2 * (kx ** 2 + ky ** 2))
    return np.real(np.fft.ifft2(np.fft.fft2(a) * h))


def crescent_image(img: Image, r_out_uas: float = 22.0, r_in_uas: float = 15.0,
                   shift_uas: float = 5.0, flux: float = 0.6, blur_fwhm_uas: float = 5.0,
                   angle: float = 0.0, supersample: int = 4) -> np.ndarray:
    """Uniform disk minus an offset inner disk, blurred by a Gaussian."""
    h = img.header
    nx, ny = h["nx"], h["ny"]
    pix = abs(h["dx"]) * 3600e6
    s = supersample
    off = (np.arange(s) + 0.5) / s - 0.5
    ix = (np.arange(nx)[:, None] + 1 - h["nxref"] + off[None, :]).reshape(-1)
    iy = (np.arange(ny)[:, None] + 1 - h["nyref"] + off[None, :]).reshape(-1)
    X, Y = np.meshgrid(-ix * pix, iy * pix)  # RA offset grows to the left
    cx, cy = shift_uas * math.cos(angle), shift_uas * math.sin(angle)
    inside = (X ** 2 + Y ** 2 <= r_out_uas ** 2) & ((X - cx) ** 2 + (Y - cy) ** 2 > r_in_uas ** 2)
    a = inside.astype(np.float64).reshape(ny, s, nx, s).mean(axis=(1, 3))
    if blur_fwhm_uas > 0:
        a = np.clip(_gauss_blur(a, blur_fwhm_uas / pix / math.sqrt(8 * math.log(2))), 0, None)
    return a * (flux / a.sum())


def multigauss_gp_image(img: Image, rng: np.random.Generator, ngauss: int = 50,
                        flux: float = 1.0, extent_uas: float = 60.0,
                        gp_corr_uas: float = 10.0, gp_frac: float = 0.2) -> np.ndarray:
    """Sum of seeded elliptical Gaussians plus a log-normal GP background.

    The background is exp() of a squared-exponential Gaussian process
    (correlation length ``gp_corr_uas``) under a broad envelope, scaled to
    ``gp_frac`` of the total flux.
    """
    x, y = xy_rad(img)
    xu, yu = x / UAS, y / UAS
    out = np.zeros_like(xu)
    for _ in range(ngauss):
        x0, y0 = rng.uniform(-extent_uas, extent_uas, 2)
        maj = rng.uniform(3.0, 20.0)
        mnr = maj * rng.uniform(0.3, 1.0)
        pa = rng.uniform(0, np.pi)
        f = 10 ** rng.uniform(-2, 0)
        c, s = math.cos(pa), math.sin(pa)
        dxu, dyu = xu - x0, yu - y0
        a = (c * dxu + s * dyu) / (maj / 2.3548)
        b = (-s * dxu + c * dyu) / (mnr / 2.3548)
        g = np.exp(-0.5 * (a * a + b * b))
        if g.sum() > 0:
            out += f * g / g.sum()
    pix = abs(img.header["dx"]) * 3600e6
    field = _gauss_blur(rng.standard_normal(xu.shape), gp_corr_uas / pix)
    field = (field - field.mean()) / (field.std() + 1e-30)
    env = np.exp(-(xu ** 2 + yu ** 2) / (2 * (1.5 * extent_uas) ** 2))
    bg = np.exp(0.8 * field) * env
    out = out * ((1 - gp_frac) * flux / out.sum()) + bg * (gp_frac * flux / bg.sum())
    return out


# ----------------------------------------------------------------------------
# arrays and uv coverage
# ----------------------------------------------------------------------------
def random_stations(rng: np.random.Generator, n: int) -> np.ndarray:
    """ECEF positions (m) of ``n`` stations at seeded lat/lon on a sphere."""
    lat = np.arcsin(rng.uniform(-0.9, 0.9, n))
    lon = rng.uniform(-np.pi, np.pi, n)
    return EARTH_R * np.stack([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)], 1)


def calc_uvw(gst_hour, alpha, delta, bx, by, bz):
    """Baseline vector -> (u, v, w) (``fortlib.coord.calc_uvw``)."""
    from .fortlib.coord import calc_uvw as _calc_uvw
    return _calc_uvw(gst_hour, alpha, delta, bx, by, bz)


def exact_dft(img_data: np.ndarray, img: Image, u: np.ndarray, v: np.ndarray,
              chunk: int = 8192) -> np.ndarray:
    """V(u,v) = sum_pix I exp(+2 pi i (u x + v y)), u, v in wavelengths.

    Separable form: V_j = sum_y e^{2 pi i v_j y} sum_x I(y, x) e^{2 pi i u_j x},
    evaluated as real GEMMs in chunks of ``chunk`` uv points.
    """
    xv, yv = img.get_xygrid(twodim=False, angunit="rad")
    out = np.empty(u.size, dtype=np.complex128)
    I = np.asarray(img_data, dtype=np.float64)
    for s in range(0, u.size, chunk):
        uu = u[s:s + chunk, None] * (2 * np.pi) * xv[None, :]
        vv = v[s:s + chunk, None] * (2 * np.pi) * yv[None, :]
        cu, su = np.cos(uu), np.sin(uu)
        ar = cu @ I.T
        ai = su @ I.T
        cv, sv = np.cos(vv), np.sin(vv)
        out[s:s + chunk] = (ar * cv - ai * sv).sum(1) + 1j * (ai * cv + ar * sv).sum(1)
    return out


def _independent_quads(nst: int):
    """A maximal independent set of N(N-3)/2 closure-amplitude quadrangles.

    Quadrangle (a,b,c,d) gives log|V_ab| + log|V_cd| - log|V_ac| - log|V_bd|;
    candidates are taken greedily while they raise the rank of the
    baseline-incidence matrix.
    """
    bls = list(itertools.combinations(range(nst), 2))
    bidx = {b: i for i, b in enumerate(bls)}
    rows, quads = [], []
    target = nst * (nst - 3) // 2
    for a, b, c, d in itertools.permutations(range(nst), 4):
        if not (a < b and c < d and a < c and a < d):
            continue
        e = [(a, b, 1), (c, d, 1), (a, c, -1), (b, d, -1)]
        row = np.zeros(len(bls))
        ok = True
        for s, t, sg in e:
            key = (min(s, t), max(s, t))
            if key not in bidx:
                ok = False
                break
            row[bidx[key]] += sg
        if not ok or not np.any(row):
            continue
        cand = np.array(rows + [row])
        if np.linalg.matrix_rank(cand) > len(rows):
            rows.append(row)
            quads.append((a, b, c, d))
        if len(quads) == target:
            break
    return quads


@dataclasses.dataclass
class Observation:
    """One synthetic data set plus its imaging set-up."""
    image: Image                  # grid description (data = initial image)
    truth: np.ndarray             # (ny, nx) truth on the imaging grid
    vistable: Optional[pd.DataFrame]
    amptable: Optional[pd.DataFrame]
    bstable: Optional[pd.DataFrame]
    catable: Optional[pd.DataFrame]
    reg: dict                     # regularizer lambdas for ``imaging``
    niter: int
    totalflux: float


def observe(truth: np.ndarray, img: Image, rng: np.random.Generator, nst: int,
            dec_deg: float, freq_hz: float, hours: float, scan_min: float,
            snr_range=(5.0, 200.0), gain_amp: float = 0.0, gain_phase: bool = False,
            fcv: bool = True, amp: bool = False, cp: bool = True, ca: bool = False,
            amp_frac_err: float = 0.0, tint_s: float = 10.0, model=None, stations=None,
            gst_start=None):
    """Simulate a VLBI track of ``truth`` and form the requested tables.

    ``model(truth, img, u, v)`` returns the model visibilities; the default is
    the exact DFT ``exact_dft``.  ``stations`` (ECEF positions) and
    ``gst_start`` (hours) fix the array and the track start instead of drawing
    them, so that consecutive frames of a movie share one array.  Every baseline is observed in every scan, so
    row ``scan * Nbl + b`` of the visibility table is baseline ``b``.
    """
    lam = C_LIGHT / freq_hz
    pos = random_stations(rng, nst) if stations is None else np.asarray(stations)
    nscan = max(1, int(round(hours * 60.0 / scan_min)))
    gst = np.linspace(0.0, hours, nscan, endpoint=False) + (rng.uniform(0, 24) if gst_start is None
                                                             else gst_start)
    dec = np.deg2rad(dec_deg)
    bls = list(itertools.combinations(range(nst), 2))
    nbl = len(bls)
    bidx = {b: i for i, b in enumerate(bls)}
    ba = np.array([a for a, _ in bls])
    bb = np.array([b for _, b in bls])
    dvec = pos[bb] - pos[ba]                                   # (nbl, 3)
    T = np.repeat(gst, nbl)
    D = np.tile(dvec, (nscan, 1))
    u, v, _ = calc_uvw(T, 0.0, dec, D[:, 0], D[:, 1], D[:, 2])
    tab = pd.DataFrame({"scan": np.repeat(np.arange(nscan), nbl), "st1": np.tile(ba, nscan),
                        "st2": np.tile(bb, nscan), "u": u / lam, "v": v / lam})
    V = (model or exact_dft)(truth, img, tab["u"].values, tab["v"].values)
    snr = 10 ** rng.uniform(np.log10(snr_range[0]), np.log10(snr_range[1]), V.size)
    sigma = np.abs(V) / snr
    if gain_amp > 0 or gain_phase:
        ga = 1 + rng.uniform(-gain_amp, gain_amp, (nscan, nst))
        gp = rng.uniform(-np.pi, np.pi, (nscan, nst)) if gain_phase else np.zeros((nscan, nst))
        g = ga * np.exp(1j * gp)
        s, a_, b_ = tab["scan"].values, tab["st1"].values, tab["st2"].values
        V = V * g[s, a_] * np.conj(g[s, b_])
        sigma = sigma * np.abs(g[s, a_] * g[s, b_])
    Vn = V + sigma * (rng.standard_normal(V.size) + 1j * rng.standard_normal(V.size))
    tab["amp"] = np.abs(Vn)
    tab["phase"] = np.rad2deg(np.angle(Vn))
    tab["sigma"] = sigma
    tab["gsthour"] = gst[tab["scan"].values]
    out = {"vistable": tab.copy() if fcv else None, "amptable": None,
           "bstable": None, "catable": None}
    if amp:
        at = tab.copy()
        if amp_frac_err > 0:
            at["sigma"] = np.sqrt(at["sigma"] ** 2 + (amp_frac_err * at["amp"]) ** 2)
        out["amptable"] = at
    U, Vv = tab["u"].values, tab["v"].values
    A, P, S = tab["amp"].values, np.deg2rad(tab["phase"].values), tab["sigma"].values
    base = (np.arange(nscan) * nbl)[:, None]
    if cp:
        tri = [(0, i, j) for i in range(1, nst) for j in range(i + 1, nst)]
        k1 = (base + np.array([bidx[(0, i)] for _, i, _ in tri])[None, :]).ravel()
        k2 = (base + np.array([bidx[(i, j)] for _, i, j in tri])[None, :]).ravel()
        k3 = (base + np.array([bidx[(0, j)] for _, _, j in tri])[None, :]).ravel()
        bamp = A[k1] * A[k2] * A[k3]
        ph = P[k1] + P[k2] - P[k3]
        out["bstable"] = pd.DataFrame({
            "u12": U[k1], "v12": Vv[k1], "u23": U[k2], "v23": Vv[k2], "u31": -U[k3], "v31": -Vv[k3],
            "amp": bamp, "phase": np.rad2deg(np.angle(np.exp(1j * ph))),
            "sigma": bamp * np.sqrt((S[k1] / A[k1]) ** 2 + (S[k2] / A[k2]) ** 2 + (S[k3] / A[k3]) ** 2)})
    if ca:
        quads = _independent_quads(nst)
        ks = []
        for pair_sel in range(4):
            col = []
            for (a, b, c, d) in quads:
                pr = ((a, b), (c, d), (a, c), (b, d))[pair_sel]
                col.append(bidx[tuple(sorted(pr))])
            ks.append((base + np.array(col)[None, :]).ravel())
        rho2 = [np.maximum(1.0, (A[k] / S[k]) ** 2 - 1) for k in ks]
        lamp = np.log(A[ks[0]]) + np.log(A[ks[1]]) - np.log(A[ks[2]]) - np.log(A[ks[3]])
        lsig = np.sqrt(sum(1.0 / r for r in rho2))
        out["catable"] = pd.DataFrame({
            "u1": U[ks[0]], "v1": Vv[ks[0]], "u2": U[ks[1]], "v2": Vv[ks[1]],
            "u3": U[ks[2]], "v3": Vv[ks[2]], "u4": U[ks[3]], "v4": Vv[ks[3]],
            "amp": np.exp(lamp), "logamp": lamp, "logsigma": lsig})
    return out


# ----------------------------------------------------------------------------
# the named workloads
# ----------------------------------------------------------------------------
def small_crescent(seed: int = 0, nx: int = 64, niter: int = 1000, model=None) -> Observation:
    """64x64, 2 uas pixels, blurred crescent, 8 stations, fcv + cp, l1 = tsv = 1."""
    rng = np.random.default_rng(seed)
    img = Image(nx, nx, 2.0)
    truth = crescent_image(img)
    t = observe(truth, img, rng, nst=8, dec_deg=12.0, freq_hz=230e9, hours=12.0,
                scan_min=10.0, fcv=True, cp=True, model=model)
    init = img.copy()
    init.data[0, 0] = gaussian_image(img, 20.0, 0.6)
    return Observation(init, truth, t["vistable"], None, t["bstable"], None,
                       {"l1_lambda": 1.0, "tsv_lambda": 1.0}, niter, 0.6)


def precision_path(seed: int = 1, nx: int = 256, nst: int = 10, hours: float = 12.0,
                   scan_s: float = 20.0, niter: int = 1000, model=None) -> Observation:
    """256x256, 1 uas, 50 Gaussians + GP, 10 stations, ~1e5 vis with gain errors;
    log closure amplitudes + closure phases + 5% amplitudes; l1/TV/MEM = 1/1/0.1."""
    rng = np.random.default_rng(seed)
    img = Image(nx, nx, 1.0)
    truth = multigauss_gp_image(img, rng)
    t = observe(truth, img, rng, nst=nst, dec_deg=12.0, freq_hz=230e9, hours=hours,
                scan_min=scan_s / 60.0, gain_amp=0.1, gain_phase=True, fcv=False,
                amp=True, cp=True, ca=True, amp_frac_err=0.05, model=model)
    init = img.copy()
    tf = float(t["amptable"]["amp"].max())
    init.data[0, 0] = gaussian_image(img, 60.0, tf)
    return Observation(init, truth, None, t["amptable"], t["bstable"], t["catable"],
                       {"l1_lambda": 1.0, "tv_lambda": 1.0, "kl_lambda": 0.1}, niter, tf)


def survey_problem(index: int, seed: int = 3, niter: int = 1000, model=None) -> Observation:
    """One problem of the hyper-parameter survey: N in {64..256}, Nvis log-uniform
    2e3-5e4, 6-12 stations, (l1, tsv, mem) on an 8x8x8 log grid 1e-2..1e2."""
    rng = np.random.default_rng([seed, index])
    nx = int(rng.choice([64, 96, 128, 192, 256]))
    nst = int(rng.integers(6, 13))
    nvis = 10 ** rng.uniform(np.log10(2e3), np.log10(5e4))
    nbl = nst * (nst - 1) // 2
    nscan = max(4, int(round(nvis / nbl)))
    hours = 12.0
    pix = 160.0 / nx  # same field of view for every grid size
    img = Image(nx, nx, pix)
    kind = index % 3
    if kind == 0:
        truth = crescent_image(img, flux=0.6)
    elif kind == 1:
        truth = multigauss_gp_image(img, rng, ngauss=10, extent_uas=40.0)
    else:
        truth = gaussian_image(img, 30.0, 0.8, 5.0, -3.0)
    t = observe(truth, img, rng, nst=nst, dec_deg=float(rng.uniform(-30, 60)), freq_hz=230e9,
                hours=hours, scan_min=hours * 60.0 / nscan, fcv=True, cp=True, model=model)
    grid = np.logspace(-2, 2, 8)
    li = np.unravel_index(index % 512, (8, 8, 8))
    init = img.copy()
    tf = float(t["vistable"]["amp"].max())
    init.data[0, 0] = gaussian_image(img, 40.0, tf)
    return Observation(init, truth, t["vistable"], None, t["bstable"], None,
                       {"l1_lambda": float(grid[li[0]]), "tsv_lambda": float(grid[li[1]]),
                        "kl_lambda": float(grid[li[2]])}, niter, tf)


def warmstart_problem(seed: int, nx: int = 128, niter: int = 1000, model=None) -> Observation:
    """One problem of the learned-warm-start set: 1 uas pixels; truth a
    crescent, ring, multi-Gaussian or GP-texture source (by seed mod 4) with
    seeded shape and total flux; 6-12 seeded stations, 12 h track with 10 min
    scans, SNR log-uniform 5-200; complex visibilities + closure phases;
    l1 = tsv = 1; a 20 uas Gaussian prior with the zero-spacing flux."""
    rng = np.random.default_rng([seed, 44])
    img = Image(nx, nx, 1.0)
    flux = float(10 ** rng.uniform(np.log10(0.3), np.log10(1.5)))
    kind = seed % 4
    if kind in (0, 1):
        r_out = float(rng.uniform(15.0, 30.0))
        truth = crescent_image(img, r_out_uas=r_out, r_in_uas=r_out * float(rng.uniform(0.5, 0.8)),
                               shift_uas=0.0 if kind == 1 else float(rng.uniform(2.0, 0.3 * r_out)),
                               flux=flux, blur_fwhm_uas=float(rng.uniform(3.0, 8.0)),
                               angle=float(rng.uniform(0, 2 * np.pi)))
    elif kind == 2:
        truth = multigauss_gp_image(img, rng, ngauss=int(rng.integers(3, 13)), flux=flux,
                                    extent_uas=25.0, gp_frac=0.05)
    else:
        truth = multigauss_gp_image(img, rng, ngauss=int(rng.integers(2, 6)), flux=flux,
                                    extent_uas=20.0, gp_corr_uas=float(rng.uniform(5.0, 12.0)),
                                    gp_frac=float(rng.uniform(0.6, 0.9)))
    nst = int(rng.integers(6, 13))
    t = observe(truth, img, rng, nst=nst, dec_deg=float(rng.uniform(-30, 60)), freq_hz=230e9,
                hours=12.0, scan_min=10.0, fcv=True, cp=True, model=model)
    tf = float(t["vistable"]["amp"].max())
    init = img.copy()
    init.data[0, 0] = gaussian_image(img, 20.0, tf)
    return Observation(init, truth, t["vistable"], None, t["bstable"], None,
                       {"l1_lambda": 1.0, "tsv_lambda": 1.0}, niter, tf)


@dataclasses.dataclass
class MovieObservation:
    """A synthetic movie data set: per-frame initial images and truths, and
    tables with a ``frmidx`` column, ordered by frame."""
    frames: list                  # initial Image of every frame
    truths: list                  # (ny, nx) truth of every frame
    vistable: Optional[pd.DataFrame]
    bstable: Optional[pd.DataFrame]
    reg: dict
    niter: int
    totalflux: float


def dynamic_problem(seed: int = 0, nframes: int = 64, nx: int = 128, nst: int = 16, hours: float = 24.0,
                    vis_per_frame: int = 6000, niter: int = 1000, model=None) -> MovieObservation:
    """Dynamic imaging: ``nframes`` frames of nx x nx (1 uas pixels) over a
    ``hours`` track, ~``vis_per_frame`` visibilities per frame from ``nst``
    seeded stations; the truth is a crescent rotating by 90 deg over the
    sequence; complex visibilities + closure phases per frame; l1 = tsv = 1
    per frame and the inter-frame squared difference Rt = 1."""
    rng = np.random.default_rng([seed, 55])
    img = Image(nx, nx, 1.0)
    pos = random_stations(rng, nst)
    dec = float(rng.uniform(-30, 60))
    gst0 = float(rng.uniform(0, 24))
    window = hours / nframes
    nbl = nst * (nst - 1) // 2
    nscan = max(1, int(round(vis_per_frame / nbl)))
    angle0 = float(rng.uniform(0, 2 * np.pi))
    truths, vis, bs = [], [], []
    for z in range(nframes):
        ang = angle0 + 0.5 * np.pi * z / max(1, nframes - 1)
        truth = crescent_image(img, r_out_uas=22.0, r_in_uas=15.0, shift_uas=5.0, flux=0.6,
                               blur_fwhm_uas=5.0, angle=ang)
        t = observe(truth, img, rng, nst=nst, dec_deg=dec, freq_hz=230e9, hours=window,
                    scan_min=window * 60.0 / nscan, fcv=True, cp=True, model=model, stations=pos,
                    gst_start=gst0 + z * window)
        t["vistable"]["frmidx"] = z
        t["bstable"]["frmidx"] = z
        truths.append(truth)
        vis.append(t["vistable"])
        bs.append(t["bstable"])
    vistable = pd.concat(vis, ignore_index=True)
    bstable = pd.concat(bs, ignore_index=True)
    tf = 0.6
    frames = []
    for z in range(nframes):
        f = img.copy()
        f.data[0, 0] = gaussian_image(img, 20.0, tf)
        frames.append(f)
    return MovieObservation(frames, truths, vistable, bstable,
                            {"l1_lambda": 1.0, "tsv_lambda": 1.0, "rt_lambda": 1.0}, niter, tf)


def nufft_model(truth: np.ndarray, img: Image, u: np.ndarray, v: np.ndarray,
                eps: float = 1e-12) -> np.ndarray:
    """Model visibilities through the library's own type-2 NUFFT (GPU).

    Same convention as ``exact_dft``: the NUFFT phase origin is pixel
    nx/2+1, so the result is rotated to the reference pixel nxref.
    """
    from .fortlib import fftlib
    h = img.header
    up = u * (2 * np.pi * np.deg2rad(h["dx"]))
    vp = v * (2 * np.pi * np.deg2rad(h["dy"]))
    vr, vi = fftlib.nufft_fwd_real(up, vp, np.asarray(truth).T, nufft_eps=eps)
    dix = h["nx"] // 2 + 1 - h["nxref"]
    diy = h["ny"] // 2 + 1 - h["nyref"]
    return (vr + 1j * vi) * np.exp(1j * (up * dix + vp * diy))
