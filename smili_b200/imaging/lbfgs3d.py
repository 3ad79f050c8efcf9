"""Drop-in host side of ``smili.imaging.lbfgs3d.imaging3d`` (dynamic imaging).

``prepare_imaging3d`` restates the preparation of lbfgs3d.py:280-730 (total
flux, normalisation, per-frame windows, regularizer weights, light curve,
Rt / Ri / Rs / Rf weights, data arrays, ``get_uvlist_loop``) and returns the
keyword arguments of ``fortlib.fftim3d.imaging``; ``imaging3d`` runs them
through the B200 library and returns the frames' images.

Two inputs on which the reference raises instead of imaging are given a
result here: ``l1_lambda > 0`` without ``l1_prior`` (the reference leaves
``l1_l`` and ``l1_wgt`` unset, lbfgs3d.py:388-393) uses the flat prior as
the 2D path does, and ``tfd_lambda <= 0`` without ``lc_array`` (the
reference takes ``len(None)``, lbfgs3d.py:517) uses the unit target.
"""
from __future__ import annotations

import copy

import numpy as np

from .. import fortlib
from ..uvdata import tools
from .lbfgs import lbfgsbprms


def prepare_imaging3d(initmovie, imregion=None, vistable=None, amptable=None, bstable=None, catable=None,
                      w_vis=1, w_amp=1, w_bs=1, w_ca=1, l1_lambda=-1., l1_prior=None, l1_noise=1e-2,
                      l1_type=1, l1_floor=1e-1, sm_lambda=-1, sm_maj=50., sm_min=50., sm_phi=0.,
                      tv_lambda=-1., tv_prior=None, tsv_lambda=-1., tsv_prior=None, kl_lambda=-1.,
                      kl_prior=None, gs_lambda=-1, gs_prior=None, tfd_lambda=-1, tfd_tgterror=0.01,
                      lc_lambda=-1, lc_array=None, lc_tgterror=0.01, lc_normalize=False, cen_lambda=-1,
                      cen_alpha=3, rt_lambda=-1., rt_prior=None, ri_lambda=-1., ri_prior=None, rs_lambda=-1,
                      rs_prior=None, rf_lambda=-1, rf_prior=None, niter=1000, nonneg=True, nprint=500,
                      totalflux=None, inorm=1., istokes=0, ifreq=0):
    """Return ``(kwargs, meta)`` for fortlib.fftim3d.imaging, or -1 on the
    reference's input errors.  ``initmovie`` is a list of images (one per
    frame) or an object with ``.images``."""
    frames = list(getattr(initmovie, "images", initmovie))
    Nt = len(frames)
    if vistable is None and amptable is None and bstable is None and catable is None:
        print("Error: No data are input.")
        return -1
    if totalflux is None and lc_array is not None:  # lbfgs3d.py:280-294
        totalflux = float(np.median(lc_array))
    elif totalflux is None:
        tf = []
        if vistable is not None:
            tf.append(np.asarray(vistable["amp"]).max())
        if amptable is not None:
            tf.append(np.asarray(amptable["amp"]).max())
        if not tf:
            print("Error: No absolute amplitude information in the input data.")
            return -1
        totalflux = float(np.max(tf))

    init0 = frames[0]
    Iin = [np.float64(f.data[istokes, ifreq]) for f in frames]
    Nx, Ny = int(init0.header["nx"]), int(init0.header["ny"])
    Nyx = Nx * Ny
    xidx, yidx = np.meshgrid(np.arange(Nx) + 1, np.arange(Ny) + 1)
    Nxref, Nyref = init0.header["nxref"], init0.header["nyref"]
    dx_rad = np.deg2rad(init0.header["dx"])
    dy_rad = np.deg2rad(init0.header["dy"])
    if imregion is None:
        Iin = [I.reshape(Nyx) for I in Iin]
        xidx, yidx = xidx.reshape(Nyx), yidx.reshape(Nyx)
        winidx = None
    else:
        if isinstance(imregion, np.ndarray):  # a (ny, nx) mask (ndarray also has .data)
            imagewin = imregion.astype(bool)
        elif hasattr(imregion, "imagewin"):
            imagewin = imregion.imagewin(init0, istokes, ifreq)
        elif hasattr(imregion, "data"):
            imagewin = imregion.data[0, 0] > 0.5
        else:
            imagewin = np.asarray(imregion, dtype=bool)
        winidx = np.where(imagewin)
        Iin = [I[winidx] for I in Iin]
        xidx, yidx = xidx[winidx], yidx[winidx]
    Npix = len(Iin[0])
    allI = np.concatenate(Iin)
    if inorm < 0:  # lbfgs3d.py:346-353
        inormfactr = 1.0
    elif np.sum(allI) != 0:
        inormfactr = inorm / np.max(allI)
    else:
        inormfactr = inorm / (totalflux / Npix)
    totalflux_scaled = totalflux * inormfactr

    def prior_array(prior):
        if imregion is None:
            return np.array(prior.data[0, 0], dtype=np.float64).reshape(Nyx)
        return np.array(prior.data[0, 0], dtype=np.float64)[winidx]

    img = fortlib.image
    if l1_lambda <= 0:  # lbfgs3d.py:357-402
        l1_wgt, l1_nwgt, l1_l = np.float64([0]), 1, -1
    else:
        if l1_prior is None:
            pr = np.full(Npix, totalflux_scaled / Npix)
        else:
            pr = prior_array(l1_prior)
            amax = np.abs(pr).max()
            if l1_type == 1:
                pr[np.where(np.abs(pr) < amax * l1_noise)] = amax * l1_noise
                pr *= totalflux_scaled / pr.sum()
            else:
                pr *= totalflux_scaled / np.sum(pr)
                pr[np.where(np.abs(pr) < np.abs(pr).max() * l1_noise)] = np.abs(pr).max() * l1_floor
        l1_wgt = img.init_l1reg(pr)
        l1_nwgt, l1_l = len(l1_wgt), l1_lambda
    if sm_lambda <= 0:  # lbfgs3d.py:405-418
        sm_l = -1
    else:
        sm_l = sm_lambda
        dtheta = np.abs(init0.angconv("deg", init0.angunit) * init0.header["dx"])
        sm_maj = (sm_maj / dtheta) ** 2 / (8. * np.log(2.))
        sm_min = (sm_min / dtheta) ** 2 / (8. * np.log(2.))
        sm_phi = sm_phi / 180. * np.pi
    if tv_lambda <= 0:
        tv_wgt, tv_nwgt, tv_l = np.float64([0]), 1, -1
    else:
        if tv_prior is None:
            pr, flat = np.full(Npix, totalflux_scaled / Npix), True
        else:
            pr, flat = prior_array(tv_prior), False
        pr *= totalflux_scaled / pr.sum()
        tv_wgt = img.init_tvreg(xidx=xidx, yidx=yidx, nx=Nx, ny=Ny, tv_isflat=flat, tv_prior=pr)
        tv_nwgt, tv_l = len(tv_wgt), tv_lambda
    if tsv_lambda <= 0:
        tsv_wgt, tsv_nwgt, tsv_l = np.float64([0]), 1, -1
    else:
        if tsv_prior is None:
            pr, flat = np.full(Npix, totalflux_scaled / Npix), True
        else:
            pr, flat = prior_array(tsv_prior), False
        pr *= totalflux_scaled / pr.sum()
        tsv_wgt = img.init_tsvreg(xidx=xidx, yidx=yidx, nx=Nx, ny=Ny, tsv_isflat=flat, tsv_prior=pr)
        tsv_nwgt, tsv_l = len(tsv_wgt), tsv_lambda
    if kl_lambda <= 0:
        kl_wgt, kl_nwgt, kl_l = np.float64([0]), 1, -1
    else:
        pr = np.full(Npix, totalflux_scaled / Npix) if kl_prior is None else prior_array(kl_prior)
        pr *= totalflux_scaled / pr.sum()
        kl_l, kl_wgt = img.init_klreg(kl_l_in=kl_lambda, kl_prior=pr)
        kl_nwgt = len(kl_wgt)
    if gs_lambda <= 0:
        gs_wgt, gs_nwgt, gs_l = np.float64([0]), 1, -1
    else:
        pr = np.full(Npix, totalflux_scaled / Npix) if gs_prior is None else prior_array(gs_prior)
        pr *= totalflux_scaled / pr.sum()
        gs_wgt = img.init_gsreg(gs_prior=pr)
        gs_nwgt, gs_l = len(gs_wgt), gs_lambda
    if tfd_lambda <= 0:  # lbfgs3d.py:513-526
        tfd_l, tfd_tgtfd = -1, 1.0
        if lc_array is not None and len(lc_array) > 0 and lc_normalize in ("static", "both"):
            tfd_tgtfd = float(np.mean(lc_array)) * inormfactr
    else:
        tfd_tgtfd = np.float64(totalflux_scaled)
        tfd_l = img.init_tfdreg(tfd_l_in=tfd_lambda, tfd_tgtfd=tfd_tgtfd, tfd_tgter=tfd_tgterror)
    lc_nidx = -1  # lbfgs3d.py:527-551
    if lc_lambda <= 0:
        lc_l = np.zeros(Nt) - 1.
        lc_tgtfd = np.zeros(Nt) + 1.
    else:
        if lc_array is None or len(lc_array) != Nt:
            print("Error: Length of light array is inconsistent with time bin of the movie")
            return -1
        lc_tgtfd = np.float64(lc_array) * inormfactr
        lc_l = lc_lambda / (lc_tgterror * lc_tgtfd) ** 2
        lc_nidx = {"static": 1, "dynamic": 2, "both": 3}.get(lc_normalize, -1)
    if cen_lambda <= 0:
        cen_l, cen_alpha = -1, 1
    else:
        cen_l = cen_lambda

    def dyn_weights(lam, prior, eps2, flat_value, norm_sum, sq):
        """Rt / Ri / Rs / Rf weights 1 / (Nt Npix prior) (lbfgs3d.py:559-660)."""
        if lam <= 0:
            return np.float64([0]), 1, -1
        if prior is None:
            pr = np.full(Npix, flat_value)
        else:
            pr = prior_array(prior)
            pr *= norm_sum / pr.sum()
            pr = np.sqrt(np.float64(pr ** 2 + (eps2 ** 2 if sq else eps2)))
        return 1. / (Nt * Npix * pr), Npix, lam

    rt_wgt, rt_nwgt, _ = dyn_weights(rt_lambda, rt_prior, 1e-5, 1. / Npix, 1.0, True)
    ri_wgt, ri_nwgt, _ = dyn_weights(ri_lambda, ri_prior, 1e-5, 1. / Npix, 1.0, True)
    if rs_lambda <= 0:
        rs_wgt, rs_nwgt = np.float64([0]), 1
    else:
        pr = np.full(Npix, totalflux_scaled / Npix) if rs_prior is None else prior_array(rs_prior)
        if rs_prior is not None:
            pr *= totalflux_scaled / pr.sum()
            pr = np.sqrt(np.float64(pr ** 2 + 1e-10))
        pr /= pr.sum()
        rs_wgt, rs_nwgt = 1. / (Nt * Npix * pr), Npix
    rf_wgt, rf_nwgt, _ = dyn_weights(rf_lambda, rf_prior, 1e-10, totalflux_scaled / Npix, totalflux_scaled,
                                     False)

    dummy = np.float64([0.])
    if vistable is None:
        isfcv, vfcvr, vfcvi, varfcv = False, dummy, dummy, dummy
    else:
        isfcv = True
        phase = np.deg2rad(np.asarray(vistable["phase"], dtype=np.float64))
        amp = np.asarray(vistable["amp"], dtype=np.float64) * inormfactr
        vfcvr, vfcvi = amp * np.cos(phase), amp * np.sin(phase)
        varfcv = np.square(np.asarray(vistable["sigma"], dtype=np.float64)) * inormfactr ** 2
    if amptable is None:
        isamp, vamp, varamp = False, dummy, dummy
    else:
        isamp = True
        vamp = np.asarray(amptable["amp"], dtype=np.float64) * inormfactr
        varamp = np.square(np.asarray(amptable["sigma"], dtype=np.float64)) * inormfactr ** 2
    if bstable is None:
        iscp, cp, varcp = False, dummy, dummy
    else:
        iscp = True
        cp = np.deg2rad(np.asarray(bstable["phase"], dtype=np.float64))
        varcp = np.square(np.asarray(bstable["sigma"], dtype=np.float64) / np.asarray(bstable["amp"], dtype=np.float64))
    if catable is None:
        isca, ca, varca = False, dummy, dummy
    else:
        isca = True
        ca = np.asarray(catable["logamp"], dtype=np.float64)
        varca = np.square(np.asarray(catable["logsigma"], dtype=np.float64))
    if Nt > 1:  # lbfgs3d.py:712-722
        u, v, uvidxfcv, uvidxamp, uvidxcp, uvidxca, Nuvs = tools.get_uvlist_loop(
            Nt=Nt, fcvconcat=vistable, ampconcat=amptable, bsconcat=bstable, caconcat=catable)
    else:
        u, v, uvidxfcv, uvidxamp, uvidxcp, uvidxca = tools.get_uvlist(
            fcvtable=vistable, amptable=amptable, bstable=bstable, catable=catable)
        Nuvs = np.array([len(u)])
    u = u * (2 * np.pi * dx_rad)
    v = v * (2 * np.pi * dy_rad)
    f64 = lambda a: np.asarray(a, dtype=np.float64)
    kw = dict(
        iin=np.float64(allI * inormfactr), xidx=np.int32(xidx), yidx=np.int32(yidx),
        nxref=np.float64(Nxref), nyref=np.float64(Nyref), nx=np.int32(Nx), ny=np.int32(Ny), nz=np.int32(Nt),
        u=u, v=v, nuvs=np.int32(Nuvs), niter=np.int32(niter), nonneg=bool(nonneg), nprint=np.int32(nprint),
        l1_l=np.float64(l1_l), l1_wgt=f64(l1_wgt), l1_nwgt=np.int32(l1_nwgt),
        sm_l=np.float64(sm_l), sm_maj=np.float64(sm_maj), sm_min=np.float64(sm_min), sm_phi=np.float64(sm_phi),
        tv_l=np.float64(tv_l), tv_wgt=f64(tv_wgt), tv_nwgt=np.int32(tv_nwgt),
        tsv_l=np.float64(tsv_l), tsv_wgt=f64(tsv_wgt), tsv_nwgt=np.int32(tsv_nwgt),
        kl_l=np.float64(kl_l), kl_wgt=f64(kl_wgt), kl_nwgt=np.int32(kl_nwgt),
        gs_l=np.float64(gs_l), gs_wgt=f64(gs_wgt), gs_nwgt=np.int32(gs_nwgt),
        tfd_l=np.float64(tfd_l), tfd_tgtfd=np.float64(tfd_tgtfd),
        lc_l=f64(lc_l), lc_tgtfd=f64(lc_tgtfd), lc_nidx=np.int32(lc_nidx),
        cen_l=np.float64(cen_l), cen_alpha=np.float64(cen_alpha),
        rt_l=np.float64(rt_lambda), rt_wgt=f64(rt_wgt), rt_nwgt=np.int32(rt_nwgt),
        ri_l=np.float64(ri_lambda), ri_wgt=f64(ri_wgt), ri_nwgt=np.int32(ri_nwgt),
        rs_l=np.float64(rs_lambda), rs_wgt=f64(rs_wgt), rs_nwgt=np.int32(rs_nwgt),
        rf_l=np.float64(rf_lambda), rf_wgt=f64(rf_wgt), rf_nwgt=np.int32(rf_nwgt),
        isfcv=isfcv, uvidxfcv=np.int32(uvidxfcv), vfcvr=f64(vfcvr), vfcvi=f64(vfcvi), varfcv=f64(varfcv),
        wfcv=np.float64(w_vis),
        isamp=isamp, uvidxamp=np.int32(uvidxamp), vamp=f64(vamp), varamp=f64(varamp), wamp=np.float64(w_amp),
        iscp=iscp, uvidxcp=np.int32(uvidxcp), cp=f64(cp), varcp=f64(varcp), wcp=np.float64(w_bs),
        isca=isca, uvidxca=np.int32(uvidxca), ca=f64(ca), varca=f64(varca), wca=np.float64(w_ca),
        inormfactr=np.float64(inormfactr),
        m=np.int32(lbfgsbprms["m"]), factr=np.float64(lbfgsbprms["factr"]),
        pgtol=np.float64(lbfgsbprms["pgtol"]), npix=xidx.shape[0],
    )
    meta = {"xidx": xidx, "yidx": yidx, "inormfactr": inormfactr, "istokes": istokes, "ifreq": ifreq,
            "nt": Nt}
    return kw, meta


def finish_imaging3d(initmovie, output, meta):
    """Frames of Iout / inormfactr in copies of the initial frames
    (lbfgs3d.py:786-791)."""
    frames = list(getattr(initmovie, "images", initmovie))
    Iout = np.asarray(output[0]) / meta["inormfactr"]
    Npix = len(meta["xidx"])
    out = []
    for it, f in enumerate(frames):
        g = copy.deepcopy(f)
        g.data[meta["istokes"], meta["ifreq"], meta["yidx"] - 1, meta["xidx"] - 1] = Iout[it * Npix:(it + 1) * Npix]
        if hasattr(g, "update_fits"):
            g.update_fits()
        out.append(g)
    return out


def imaging3d(initmovie, precision=64, nufft_eps=0.0, device=0, **kwargs):
    """Dynamic imaging on the GPU with the arguments of lbfgs3d.imaging3d;
    returns the list of output frames."""
    prep = prepare_imaging3d(initmovie, **kwargs)
    if isinstance(prep, int):
        return prep
    kw, meta = prep
    out = fortlib.fftim3d.imaging(precision=precision, nufft_eps=nufft_eps, device=device, **kw)
    return finish_imaging3d(initmovie, out, meta)
