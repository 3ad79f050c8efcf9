"""Static imaging driver: the host side of ``smili.imaging.lbfgs.imaging``.

``prepare_imaging`` restates the body of ``imaging`` up to the single f2py
call (smili/imaging/lbfgs.py:185-489): sanity checks, total-flux guess,
intensity normalisation, regularizer weights, data arrays and the uv list.
It returns the keyword arguments of ``fortlib.fftim2d.imaging`` with the
names the reference passes (lbfgs.py:492-564).  ``imaging`` then makes that
call against this package's CUDA-backed ``fortlib`` and rebuilds the image
(lbfgs.py:565-576).  Images are duck-typed IMFITS (``.data``, ``.header``,
``.get_xygrid``, ``.angconv``); tables are pandas DataFrames with SMILI's
VisTable / BSTable / CATable columns.
"""
from __future__ import annotations

import copy

import numpy as np

from .. import fortlib
from ..uvdata import tools

# L-BFGS-B defaults (lbfgs.py:34-38)
lbfgsbprms = {"m": 5, "factr": 1e1, "pgtol": 0.0}


def _uvdist(tab, u, v):
    return np.hypot(np.asarray(tab[u], dtype=np.float64), np.asarray(tab[v], dtype=np.float64))


def deburr_vistable(vistable, fwhm=1, angunit=None, angconv=None):
    """Divide amplitudes and sigmas by a Gaussian pulse's visibility (lbfgs.py:1114-1134)."""
    out = copy.deepcopy(vistable)
    fr = angconv(angunit, "rad") * fwhm
    k = np.exp(-(np.pi ** 2 * (fr * _uvdist(out, "u", "v")) ** 2 / (4.0 * np.log(2))))
    out["amp"] = out["amp"] / k
    out["sigma"] = out["sigma"] / k
    return out


def deburr_bstable(bstable, fwhm=1, angunit=None, angconv=None):
    """Same for bispectra (lbfgs.py:1137-1163)."""
    out = copy.deepcopy(bstable)
    fr = angconv(angunit, "rad") * fwhm
    k = 1.0
    for a, b in (("u12", "v12"), ("u23", "v23"), ("u31", "v31")):
        k = k * np.exp(-(np.pi ** 2 * (fr * _uvdist(out, a, b)) ** 2 / (4.0 * np.log(2))))
    out["amp"] = out["amp"] / k
    out["sigma"] = out["sigma"] / k
    return out


def deburr_catable(catable, fwhm=1, angunit=None, angconv=None):
    """Same for closure amplitudes (lbfgs.py:1166-1194)."""
    out = copy.deepcopy(catable)
    fr = angconv(angunit, "rad") * fwhm
    ks = [np.exp(-(np.pi ** 2 * (fr * _uvdist(out, f"u{i}", f"v{i}")) ** 2 / (4.0 * np.log(2))))
          for i in (1, 2, 3, 4)]
    k = ks[0] * ks[1] / ks[2] / ks[3]
    out["amp"] = out["amp"] / k
    out["logamp"] = out["logamp"] - np.log(k)
    out["sigma"] = out["sigma"] / k
    return out


def prepare_imaging(initimage, imregion=None, vistable=None, amptable=None, bstable=None,
                    catable=None, w_vis=1, w_amp=1, w_bs=1, w_ca=1, l1_lambda=-1.,
                    l1_prior=None, l1_noise=1e-2, tv_lambda=-1, tv_prior=None, tsv_lambda=-1,
                    tsv_prior=None, kl_lambda=-1, kl_prior=None, gs_lambda=-1, gs_prior=None,
                    tfd_lambda=-1, tfd_tgterror=0.01, cen_lambda=-1, cen_alpha=3, sm_lambda=-1,
                    sm_maj=0., sm_min=0., sm_phi=0., pulse_fwhm=-1, niter=1000, nonneg=True,
                    nprint=500, totalflux=None, inorm=1., istokes=0, ifreq=0, verbose=False,
                    uvlist_device=None):
    """Return ``(kwargs, meta)``: the fftim2d.imaging kwargs and what is needed
    to rebuild the output image, or ``-1`` on the reference's input errors.
    ``uvlist_device``: a CUDA device ordinal lists the uv points on that GPU
    (``get_uvlist(device=...)``); None does it with numpy."""
    say = print if verbose else (lambda *a, **k: None)
    # Sanity checks (lbfgs.py:185-201)
    if vistable is None and amptable is None and bstable is None and catable is None:
        print("Error: No data are input.")
        return -1
    if vistable is None and amptable is None and totalflux is None:
        print("Error: No absolute amplitude information in the input data.")
        print("       You need to set the total flux constraint by totalflux / tfd_lambda")
        return -1
    elif vistable is None and amptable is None and (totalflux is None or tfd_lambda < 0):
        print("Warning: No absolute amplitude information in the input data.")
        print("         The total flux must be constrained")
        return -1
    if totalflux is None:  # lbfgs.py:203-210
        tf = []
        if vistable is not None:
            tf.append(np.asarray(vistable["amp"]).max())
        if amptable is not None:
            tf.append(np.asarray(amptable["amp"]).max())
        totalflux = float(np.max(tf))
    say("Total flux: %g Jy" % totalflux)

    Iin = np.float64(initimage.data[istokes, ifreq])
    Nx = int(initimage.header["nx"])
    Ny = int(initimage.header["ny"])
    Nyx = Nx * Ny
    xidx, yidx = np.meshgrid(np.arange(Nx) + 1, np.arange(Ny) + 1)
    Nxref = initimage.header["nxref"]
    Nyref = initimage.header["nyref"]
    dx_rad = np.deg2rad(initimage.header["dx"])
    dy_rad = np.deg2rad(initimage.header["dy"])

    if imregion is None:  # lbfgs.py:226-249
        Iin = Iin.reshape(Nyx)
        xidx = xidx.reshape(Nyx)
        yidx = yidx.reshape(Nyx)
        winidx = None
    else:
        if isinstance(imregion, np.ndarray):  # a (ny, nx) mask (ndarray also has .data)
            imagewin = imregion.astype(bool)
        elif hasattr(imregion, "imagewin"):
            imagewin = imregion.imagewin(initimage, istokes, ifreq)
        elif hasattr(imregion, "data"):
            imagewin = imregion.data[0, 0] > 0.5
        else:
            imagewin = np.asarray(imregion, dtype=bool)
        winidx = np.where(imagewin)
        Iin = Iin[winidx]
        xidx = xidx[winidx]
        yidx = yidx[winidx]
    Npix = len(Iin)

    if inorm < 0:  # lbfgs.py:252-260
        inormfactr = 1.0
    elif Iin.sum() != 0:
        inormfactr = inorm / Iin.max()
    else:
        inormfactr = inorm / (totalflux / Npix)
    totalflux_scaled = totalflux * inormfactr

    def prior_array(prior):
        # The reference takes the prior's pixels as a view of prior.data when
        # there is no window (lbfgs.py:275, 298, 328, 357, 380) and then
        # normalises it in place, so a prior image shared by several
        # regularizers reaches the later ones already normalised (and the
        # caller's image is changed).  Kept for identical weights.
        if imregion is None:
            return prior.data[0, 0].reshape(Nyx)
        return prior.data[0, 0][winidx]

    # A 0-d float64, as np.float64(np.asarray([0])) gives in the reference
    # (lbfgs.py:265, 287, 317, 347, 370); f2py broadcasts it to length 1.
    zero = np.float64(0.0)

    # regularizers (lbfgs.py:264-414)
    if l1_lambda <= 0:
        l1_wgt, l1_nwgt, l1_l = zero, 1, -1
    else:
        if l1_prior is None:
            pr = np.full(Npix, totalflux_scaled / Npix)
        else:
            pr = prior_array(l1_prior)
            amax = np.abs(pr).max()
            pr[np.where(np.abs(pr) < amax * l1_noise)] = amax * l1_noise
        pr *= totalflux_scaled / pr.sum()
        l1_wgt = fortlib.image.init_l1reg(pr)
        l1_nwgt, l1_l = len(l1_wgt), l1_lambda
    if tv_lambda <= 0:
        tv_wgt, tv_nwgt, tv_l = zero, 1, -1
    else:
        if tv_prior is None:
            pr, flat = np.full(Npix, totalflux_scaled / Npix), True
        else:
            pr, flat = prior_array(tv_prior), False
        pr *= totalflux_scaled / pr.sum()
        tv_wgt = fortlib.image.init_tvreg(xidx=xidx, yidx=yidx, nx=Nx, ny=Ny, tv_isflat=flat,
                                          tv_prior=pr)
        tv_nwgt, tv_l = len(tv_wgt), tv_lambda
    if tsv_lambda <= 0:
        tsv_wgt, tsv_nwgt, tsv_l = zero, 1, -1
    else:
        if tsv_prior is None:
            pr, flat = np.full(Npix, totalflux_scaled / Npix), True
        else:
            pr, flat = prior_array(tsv_prior), False
        pr *= totalflux_scaled / pr.sum()
        tsv_wgt = fortlib.image.init_tsvreg(xidx=xidx, yidx=yidx, nx=Nx, ny=Ny,
                                            tsv_isflat=flat, tsv_prior=pr)
        tsv_nwgt, tsv_l = len(tsv_wgt), tsv_lambda
    if kl_lambda <= 0:
        kl_wgt, kl_nwgt, kl_l = zero, 1, -1
    else:
        pr = np.full(Npix, totalflux_scaled / Npix) if kl_prior is None else prior_array(kl_prior)
        pr *= totalflux_scaled / pr.sum()
        kl_l, kl_wgt = fortlib.image.init_klreg(kl_l_in=kl_lambda, kl_prior=pr)
        kl_nwgt = len(kl_wgt)
    if gs_lambda <= 0:
        gs_wgt, gs_nwgt, gs_l = zero, 1, -1
    else:
        pr = np.full(Npix, totalflux_scaled / Npix) if gs_prior is None else prior_array(gs_prior)
        pr *= totalflux_scaled / pr.sum()
        gs_wgt = fortlib.image.init_gsreg(gs_prior=pr)
        gs_nwgt, gs_l = len(gs_wgt), gs_lambda
    if tfd_lambda <= 0:
        tfd_l, tfd_tgtfd = -1, 1
    else:
        tfd_tgtfd = np.float64(totalflux_scaled)
        tfd_l = fortlib.image.init_tfdreg(tfd_l_in=tfd_lambda, tfd_tgtfd=tfd_tgtfd,
                                          tfd_tgter=tfd_tgterror)
    if cen_lambda <= 0:
        cen_l, cen_alpha = -1, 1
    else:
        cen_l = cen_lambda
    if sm_lambda <= 0:
        sm_l = -1
    else:
        sm_l = sm_lambda
        dtheta = np.abs(initimage.angconv("deg", initimage.angunit) * initimage.header["dx"])
        sm_maj = (sm_maj / dtheta) ** 2 / (8. * np.log(2.))
        sm_min = (sm_min / dtheta) ** 2 / (8. * np.log(2.))
        sm_phi = -sm_phi / 180. * np.pi

    dummy = zero  # dammyreal, lbfgs.py:425
    conv = getattr(initimage, "angconv", None)
    if vistable is None:  # lbfgs.py:421-480
        isfcv, vfcvr, vfcvi, varfcv = False, dummy, dummy, dummy
    else:
        isfcv = True
        if pulse_fwhm > 0:
            vistable = deburr_vistable(vistable, pulse_fwhm, initimage.angunit, conv)
        phase = np.deg2rad(np.asarray(vistable["phase"], dtype=np.float64))
        amp = np.asarray(vistable["amp"], dtype=np.float64) * inormfactr
        vfcvr = amp * np.cos(phase)
        vfcvi = amp * np.sin(phase)
        varfcv = np.square(np.asarray(vistable["sigma"], dtype=np.float64)) * inormfactr ** 2
    if amptable is None:
        isamp, vamp, varamp = False, dummy, dummy
    else:
        isamp = True
        if pulse_fwhm > 0:
            amptable = deburr_vistable(amptable, pulse_fwhm, initimage.angunit, conv)
        vamp = np.asarray(amptable["amp"], dtype=np.float64) * inormfactr
        varamp = np.square(np.asarray(amptable["sigma"], dtype=np.float64)) * inormfactr ** 2
    if bstable is None:
        iscp, cp, varcp = False, dummy, dummy
    else:
        iscp = True
        if pulse_fwhm > 0:
            bstable = deburr_bstable(bstable, pulse_fwhm, initimage.angunit, conv)
        cp = np.deg2rad(np.asarray(bstable["phase"], dtype=np.float64))
        varcp = np.square(np.asarray(bstable["sigma"], dtype=np.float64) /
                          np.asarray(bstable["amp"], dtype=np.float64))
    if catable is None:
        isca, ca, varca = False, dummy, dummy
    else:
        isca = True
        if pulse_fwhm > 0:
            catable = deburr_catable(catable, pulse_fwhm, initimage.angunit, conv)
        ca = np.asarray(catable["logamp"], dtype=np.float64)
        varca = np.square(np.asarray(catable["logsigma"], dtype=np.float64))

    u, v, uvidxfcv, uvidxamp, uvidxcp, uvidxca = tools.get_uvlist(
        fcvtable=vistable, amptable=amptable, bstable=bstable, catable=catable, device=uvlist_device)
    u = u * (2 * np.pi * dx_rad)
    v = v * (2 * np.pi * dy_rad)

    kw = dict(
        iin=np.float64(Iin * inormfactr), xidx=np.int32(xidx), yidx=np.int32(yidx),
        nxref=np.float64(Nxref), nyref=np.float64(Nyref), nx=np.int32(Nx), ny=np.int32(Ny),
        u=u, v=v, niter=np.int32(niter), nonneg=bool(nonneg), nprint=np.int32(nprint),
        l1_l=np.float64(l1_l), l1_wgt=np.asarray(l1_wgt, dtype=np.float64), l1_nwgt=np.int32(l1_nwgt),
        tv_l=np.float64(tv_l), tv_wgt=np.asarray(tv_wgt, dtype=np.float64), tv_nwgt=np.int32(tv_nwgt),
        tsv_l=np.float64(tsv_l), tsv_wgt=np.asarray(tsv_wgt, dtype=np.float64), tsv_nwgt=np.int32(tsv_nwgt),
        kl_l=np.float64(kl_l), kl_wgt=np.asarray(kl_wgt, dtype=np.float64), kl_nwgt=np.int32(kl_nwgt),
        gs_l=np.float64(gs_l), gs_wgt=np.asarray(gs_wgt, dtype=np.float64), gs_nwgt=np.int32(gs_nwgt),
        tfd_l=np.float64(tfd_l), tfd_tgtfd=np.float64(tfd_tgtfd),
        cen_l=np.float64(cen_l), cen_alpha=np.float64(cen_alpha),
        sm_l=np.float64(sm_l), sm_maj=np.float64(sm_maj), sm_min=np.float64(sm_min),
        sm_phi=np.float64(sm_phi),
        isfcv=isfcv, uvidxfcv=np.int32(uvidxfcv), vfcvr=np.asarray(vfcvr, dtype=np.float64),
        vfcvi=np.asarray(vfcvi, dtype=np.float64), varfcv=np.asarray(varfcv, dtype=np.float64), wfcv=np.float64(w_vis),
        isamp=isamp, uvidxamp=np.int32(uvidxamp), vamp=np.asarray(vamp, dtype=np.float64),
        varamp=np.asarray(varamp, dtype=np.float64), wamp=np.float64(w_amp),
        iscp=iscp, uvidxcp=np.int32(uvidxcp), cp=np.asarray(cp, dtype=np.float64), varcp=np.asarray(varcp, dtype=np.float64),
        wcp=np.float64(w_bs),
        isca=isca, uvidxca=np.int32(uvidxca), ca=np.asarray(ca, dtype=np.float64), varca=np.asarray(varca, dtype=np.float64),
        wca=np.float64(w_ca),
        inormfactr=np.float64(inormfactr),
        m=np.int32(lbfgsbprms["m"]), factr=np.float64(lbfgsbprms["factr"]),
        pgtol=np.float64(lbfgsbprms["pgtol"]), npix=xidx.shape[0],
    )
    meta = {"xidx": xidx, "yidx": yidx, "inormfactr": inormfactr, "istokes": istokes,
            "ifreq": ifreq, "pulse_fwhm": pulse_fwhm}
    return kw, meta


def finish_imaging(initimage, output, meta):
    """Scatter Iout/inormfactr into a copy of the initial image (lbfgs.py:565-576)."""
    Iout = output[0] / meta["inormfactr"]
    outimage = copy.deepcopy(initimage)
    outimage.data[meta["istokes"], meta["ifreq"]] = 0.
    outimage.data[meta["istokes"], meta["ifreq"], meta["yidx"] - 1, meta["xidx"] - 1] = Iout
    outimage.update_fits()
    if meta["pulse_fwhm"] > 0 and hasattr(outimage, "convolve_gauss"):
        outimage = copy.deepcopy(outimage.convolve_gauss(meta["pulse_fwhm"],
                                                         angunit=outimage.angunit,
                                                         save_totalflux=True))
    return outimage


def imaging(initimage, **kwargs):
    """Drop-in for ``smili.imaging.lbfgs.imaging``: same keywords, same return."""
    prep = prepare_imaging(initimage, **kwargs)
    if isinstance(prep, int):
        return prep
    kw, meta = prep
    output = fortlib.fftim2d.imaging(**kw)
    return finish_imaging(initimage, output, meta)


# ---------------------------------------------------------------------------
# statistics (lbfgs.py:578-755) and the chi-squares behind it
# ---------------------------------------------------------------------------
def _image_grid(image, mask, istokes, ifreq):
    """Pixel vector, 1-based pixel indices, phase centre and uv scaling of an
    image, windowed by ``mask`` (vistable.py:435-495)."""
    Iin = np.float64(image.data[istokes, ifreq])
    Nx, Ny = int(image.header["nx"]), int(image.header["ny"])
    xidx, yidx = np.meshgrid(np.arange(Nx) + 1, np.arange(Ny) + 1)
    if mask is None:
        Iin, xidx, yidx = Iin.reshape(-1), xidx.reshape(-1), yidx.reshape(-1)
    else:
        idx = np.where(mask)
        Iin, xidx, yidx = Iin[idx], xidx[idx], yidx[idx]
    return (Iin, np.int32(xidx), np.int32(yidx), float(image.header["nxref"]), float(image.header["nyref"]),
            Nx, Ny, np.deg2rad(image.header["dx"]), np.deg2rad(image.header["dy"]))


def chisq_image(table, kind, image, mask=None, istokes=0, ifreq=0, **opt):
    """``chisq_image`` of a VisTable (kind "fcv" or "amp"), BSTable ("cp")
    or CATable ("ca") for an image (vistable.py:416-433, bstable.py:300-330,
    catable.py:260-290): (chisq, reduced chisq) from model_fcv / amp / cp /
    ca on the GPU, with the table's own values (no intensity normalisation)."""
    Iin, xidx, yidx, nxref, nyref, Nx, Ny, dx, dy = _image_grid(image, mask, istokes, ifreq)
    args = dict(fcvtable=None, amptable=None, bstable=None, catable=None)
    args[{"fcv": "fcvtable", "amp": "amptable", "cp": "bstable", "ca": "catable"}[kind]] = table
    u, v, ifcv, iamp, icp, ica = tools.get_uvlist(**args)
    u = u * (2 * np.pi * dx)
    v = v * (2 * np.pi * dy)
    base = (Iin, xidx, yidx, nxref, nyref, Nx, Ny, u, v)
    if kind == "fcv":
        ph = np.deg2rad(np.asarray(table["phase"], dtype=np.float64))
        amp = np.asarray(table["amp"], dtype=np.float64)
        out = fortlib.fftlib.model_fcv(*base, ifcv, amp * np.cos(ph), amp * np.sin(ph),
                                       np.square(np.asarray(table["sigma"], dtype=np.float64)), **opt)
        n = 2 * len(table)
    elif kind == "amp":
        out = fortlib.fftlib.model_amp(*base, iamp, np.asarray(table["amp"], dtype=np.float64),
                                       np.square(np.asarray(table["sigma"], dtype=np.float64)), **opt)
        n = len(table)
    elif kind == "cp":
        out = fortlib.fftlib.model_cp(*base, icp, np.deg2rad(np.asarray(table["phase"], dtype=np.float64)),
                                      np.square(np.asarray(table["sigma"], dtype=np.float64)
                                                / np.asarray(table["amp"], dtype=np.float64)), **opt)
        n = len(table)
    else:
        out = fortlib.fftlib.model_ca(*base, ica, np.asarray(table["logamp"], dtype=np.float64),
                                      np.square(np.asarray(table["logsigma"], dtype=np.float64)), **opt)
        n = len(table)
    return out[0], out[0] / n


def image_costs(image, istokes=0, ifreq=0):
    """(l1, tv, tsv) of an image: the per-pixel functions l1_e, tv_e and
    tsv_e of image.f90:245-257, 477-520, 678-720 summed over all pixels.
    (The reference's ``imagecost`` calls fortlib.image.i2d_l1 / i2d_tv /
    i2d_tsv, which its Fortran sources do not define; these sums are what
    their names and the per-pixel functions describe.)"""
    I = np.float64(image.data[istokes, ifreq])
    l1 = float(np.sum(np.sqrt(I * I + 1e-10)))
    dIx = np.zeros_like(I)
    dIy = np.zeros_like(I)
    dIx[:, :-1] = I[:, 1:] - I[:, :-1]
    dIy[:-1, :] = I[1:, :] - I[:-1, :]
    return l1, float(np.sum(np.sqrt(dIx * dIx + dIy * dIy))), float(np.sum(dIx * dIx + dIy * dIy))


def statistics(initimage, imregion=None, vistable=None, amptable=None, bstable=None, catable=None,
               lambl1=-1., lambtv=-1., lambtsv=-1., lambmem=-1., lambcom=-1., normlambda=True,
               reweight=False, dyrange=1e6, niter=1000, nonneg=True, compower=1., totalflux=None,
               fluxconst=False, istokes=0, ifreq=0, **opt):
    """Chi-squares and regularization costs of an image (lbfgs.py:578-755):
    the same OrderedDict of keys.  ``opt`` passes precision / nufft_eps /
    device to the GPU evaluations."""
    import collections
    if vistable is None and amptable is None and bstable is None and catable is None:
        print("Error: No data are input.")
        return -1
    imagewin = imregion.imagewin(initimage, istokes, ifreq) if imregion is not None else None
    if totalflux is None:
        tf = []
        if vistable is not None:
            tf.append(np.asarray(vistable["amp"]).max())
        if amptable is not None:
            tf.append(np.asarray(amptable["amp"]).max())
        totalflux = np.max(tf)
    Ndata = 0
    res = {}
    for key, table, kind, nd in (("fcv", vistable, "fcv", 2), ("amp", amptable, "amp", 1),
                                 ("cp", bstable, "cp", 1), ("ca", catable, "ca", 1)):
        if table is None:
            res[key] = (False, 0., 0.)
        else:
            c, rc = chisq_image(table, kind, initimage, imagewin, istokes, ifreq, **opt)
            res[key] = (True, c, rc)
            Ndata += len(table) * nd
    Nx, Ny = int(initimage.header["nx"]), int(initimage.header["ny"])
    Nyx = Nx * Ny
    if normlambda:
        fluxscale = np.abs(np.float64(totalflux)) / Nyx
        lambl1_sim = lambl1 / (fluxscale * Nyx)
        lambtv_sim = lambtv / (4 * fluxscale * Nyx)
        lambtsv_sim = lambtsv / (4 * fluxscale ** 2 * Nyx)
    else:
        lambl1_sim, lambtv_sim, lambtsv_sim = lambl1, lambtv, lambtsv
    l1, tv, tsv = image_costs(initimage, istokes, ifreq)
    if lambl1 > 0:
        l1cost = l1 * lambl1_sim
    else:
        lambl1 = lambl1_sim = l1cost = 0.
    if lambtv > 0:
        tvcost = tv * lambtv_sim
    else:
        lambtv = lambtv_sim = tvcost = 0.
    if lambtsv > 0:
        tsvcost = tsv * lambtsv_sim
    else:
        lambtsv = lambtsv_sim = tsvcost = 0.
    stats = collections.OrderedDict()
    stats["cost"] = l1cost + tvcost + tsvcost
    stats["chisq"] = res["fcv"][1] + res["amp"][1] + res["cp"][1] + res["ca"][1]
    stats["rchisq"] = stats["chisq"] / Ndata
    stats["cost"] += stats["rchisq"]
    for key in ("fcv", "amp", "cp", "ca"):
        stats["is" + key] = res[key][0]
    for key in ("fcv", "amp", "cp", "ca"):
        stats["chisq" + key] = res[key][1]
    for key in ("fcv", "amp", "cp", "ca"):
        stats["rchisq" + key] = res[key][2]
    stats["lambl1"], stats["lambl1_sim"], stats["l1"], stats["l1cost"] = lambl1, lambl1_sim, l1, l1cost
    stats["lambtv"], stats["lambtv_sim"], stats["tv"], stats["tvcost"] = lambtv, lambtv_sim, tv, tvcost
    stats["lambtsv"], stats["lambtsv_sim"], stats["tsv"], stats["tsvcost"] = lambtsv, lambtsv_sim, tsv, tsvcost
    return stats
