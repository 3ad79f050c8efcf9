// CPU oracle, part 4: dynamic (movie) imaging (test infrastructure only).
//
// Restates src/fortlib/fftlib3d.f90:14-205 (calc_chisq3d: per-frame NUFFTs
// over the frame's slice of the uv list, chi-square terms over all data,
// per-frame adjoints), src/fortlib/image3d.f90:15-425 (calc_cost_reg3d:
// the static regularizers per frame divided by Nz, the light-curve variant,
// and the dynamic Rt / Ri terms of calc_cost_dynamical) and
// src/fortlib/fftim3d.f90:11-614 (imaging, calc_cost).  Reference behaviour
// kept as is: only Rt and Ri are evaluated (rs_cost, rf_cost and cen_cost
// stay 0, the centroid term is switched off per frame), the Rt gradient is
// added only for frames iz < Nz, and the returned image is thresholded at
// zeroeps after the final summary (fftim3d.f90:466).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "oracle_internal.h"

using namespace orc;

namespace {

// Rt / Ri (image3d.f90:280-441)
void cost_dynamical(const orc_args3d* a, const double* x, double& rt_cost, double& ri_cost, double* grad) {
  const int N = a->npix, Nz = a->nz;
  rt_cost = ri_cost = 0.0;
  std::vector<double> iavg(N, 0.0);
  for (int iz = 0; iz < Nz; ++iz)
    for (int i = 0; i < N; ++i) iavg[i] += x[(size_t)iz * N + i] / a->lc_tgtfd[iz] / Nz;
  for (int iz = 0; iz < Nz; ++iz) {
    for (int i = 0; i < N; ++i) {
      const double II = x[(size_t)iz * N + i] / a->lc_tgtfd[iz];
      const double Iu = iz + 1 < Nz ? x[(size_t)(iz + 1) * N + i] / a->lc_tgtfd[iz + 1] : 0.0;
      const double Il = iz > 0 ? x[(size_t)(iz - 1) * N + i] / a->lc_tgtfd[iz - 1] : 0.0;
      if (a->rt_l > 0 && iz + 1 < Nz) {
        rt_cost += a->rt_l * a->rt_wgt[i] * (Iu - II) * (Iu - II);
        // rt_grade (image3d.f90:409-421): iz is never Nz here
        const double ge = (iz == 0) ? 2.0 * (II - Iu) : 2.0 * (2.0 * II - Il - Iu);
        grad[(size_t)iz * N + i] += a->rt_l * a->rt_wgt[i] * ge / a->lc_tgtfd[iz];
      }
      if (a->ri_l > 0) {
        ri_cost += a->ri_l * a->ri_wgt[i] * (II - iavg[i]) * (II - iavg[i]);
        grad[(size_t)iz * N + i] += a->ri_l * a->ri_wgt[i] * 2.0 * (II - iavg[i]) / a->lc_tgtfd[iz];
      }
    }
  }
}

}  // namespace

// calc_cost (fftim3d.f90:473-614); terms[20] in the fftim3d.imaging order
extern "C" int orc_calc_cost3d(const orc_args3d* a, const double* vre_s, const double* vim_s, double wfcv,
                               double wamp, double wcp, double wca, const double* x, double eps,
                               double* terms, double* grad) {
  const int N = a->npix, nx = a->nx, ny = a->ny, Nz = a->nz, nuv = a->nuv;
  std::vector<int> off(Nz, 0);
  for (int z = 1; z < Nz; ++z) off[z] = off[z - 1] + a->nuvs[z - 1];
  // forward transforms per frame
  std::vector<cplx> V(std::max(nuv, 1));
  for (int z = 0; z < Nz; ++z) {
    const int n = a->nuvs[z];
    if (!n) continue;
    std::vector<double> I2d((size_t)nx * ny, 0.0), vr(n), vi(n);
    for (int i = 0; i < N; ++i) I2d[(size_t)(a->yidx[i] - 1) * nx + (a->xidx[i] - 1)] = x[(size_t)z * N + i];
    orc_nufft2d2(n, a->u + off[z], a->v + off[z], nx, ny, I2d.data(), eps, vr.data(), vi.data());
    for (int j = 0; j < n; ++j) V[off[z] + j] = cplx(vr[j], vi[j]);
  }
  std::vector<double> rre(std::max(nuv, 1), 0.0), rim(std::max(nuv, 1), 0.0);
  double chisq = 0, cfcv = 0, camp = 0, ccp = 0, cca = 0;
  if (a->isfcv) {
    std::vector<cplx> Vd(a->nfcv);
    for (int i = 0; i < a->nfcv; ++i) Vd[i] = cplx(vre_s[i], vim_s[i]);
    chisq_fcv(V.data(), a->uvidxfcv, Vd.data(), a->varfcv, wfcv, a->nfcv, cfcv, rre.data(), rim.data());
    chisq += cfcv;
    cfcv = cfcv / wfcv / (2 * a->nfcv);
  }
  if (a->isamp) {
    chisq_amp(V.data(), a->uvidxamp, a->vamp, a->varamp, wamp, a->namp, camp, rre.data(), rim.data());
    chisq += camp;
    camp = camp / wamp / a->namp;
  }
  if (a->isca) {
    chisq_ca(V.data(), a->uvidxca, a->ca, a->varca, wca, a->nca, cca, rre.data(), rim.data());
    chisq += cca;
    cca = cca / wca / a->nca;
  }
  if (a->iscp) {
    chisq_cp(V.data(), a->uvidxcp, a->cp, a->varcp, wcp, a->ncp, ccp, rre.data(), rim.data());
    chisq += ccp;
    ccp = ccp / wcp / a->ncp;
  }
  // adjoints per frame (NUFFT_adj_resid on the frame's slice)
  std::vector<double> gchi((size_t)N * Nz, 0.0);
  for (int z = 0; z < Nz; ++z) {
    const int n = a->nuvs[z];
    if (!n) continue;
    std::vector<double> zero(n, 0.0), g1r((size_t)nx * ny), g1i((size_t)nx * ny), g2r((size_t)nx * ny),
        g2i((size_t)nx * ny);
    orc_nufft2d1(n, a->u + off[z], a->v + off[z], rre.data() + off[z], zero.data(), nx, ny, eps, g1r.data(),
                 g1i.data());
    orc_nufft2d1(n, a->u + off[z], a->v + off[z], rim.data() + off[z], zero.data(), nx, ny, eps, g2r.data(),
                 g2i.data());
    for (int i = 0; i < N; ++i) {
      const size_t p = (size_t)(a->yidx[i] - 1) * nx + (a->xidx[i] - 1);
      gchi[(size_t)z * N + i] = g1r[p] + g2i[p];
    }
  }
  // static regularizers per frame (image3d.f90:163-257)
  double l1c = 0, smc = 0, tvc = 0, tsvc = 0, klc = 0, gsc = 0, tfdc = 0, lcc = 0, regs = 0;
  std::vector<double> greg((size_t)N * Nz, 0.0), gfrm(N);
  double lcsum = 0;
  for (int z = 0; z < Nz; ++z) lcsum += a->lc_l[z];
  const bool lc_on = lcsum > 0;
  std::vector<double> w1(N), wtv(N), wtsv(N), wkl(N), wgs(N);
  for (int z = 0; z < Nz; ++z) {
    orc_args f;
    std::memset(&f, 0, sizeof(f));
    f.npix = N;
    f.nx = nx;
    f.ny = ny;
    f.xidx = a->xidx;
    f.yidx = a->yidx;
    f.nxref = a->nxref;
    f.nyref = a->nyref;
    f.l1_l = a->l1_l;
    f.tv_l = a->tv_l;
    f.tsv_l = a->tsv_l;
    f.kl_l = a->kl_l;
    f.gs_l = a->gs_l;
    f.l1_wgt = a->l1_wgt;
    f.tv_wgt = a->tv_wgt;
    f.tsv_wgt = a->tsv_wgt;
    f.kl_wgt = a->kl_wgt;
    f.gs_wgt = a->gs_wgt;
    f.cen_l = -1.0;
    f.cen_alpha = 1.0;
    f.sm_l = a->sm_l;
    f.sm_maj = a->sm_maj;
    f.sm_min = a->sm_min;
    f.sm_phi = a->sm_phi;
    if (lc_on) {
      if (a->lc_nidx == 1 || a->lc_nidx == 3) {
        const double c = a->tfd_tgtfd / a->lc_tgtfd[z];
        for (int i = 0; i < N; ++i) {
          if (a->l1_l > 0) w1[i] = a->l1_wgt[i] * c;
          if (a->tv_l > 0) wtv[i] = a->tv_wgt[i] * c;
          if (a->tsv_l > 0) wtsv[i] = a->tsv_wgt[i] * c * c;
          if (a->kl_l > 0) wkl[i] = a->kl_wgt[i] * c;
          if (a->gs_l > 0) wgs[i] = a->gs_wgt[i] * c;
        }
        f.l1_wgt = w1.data();
        f.tv_wgt = wtv.data();
        f.tsv_wgt = wtsv.data();
        f.kl_wgt = wkl.data();
        f.gs_wgt = wgs.data();
      }
      f.tfd_l = a->lc_l[z];
      f.tfd_tgtfd = a->lc_tgtfd[z];
    } else {
      f.tfd_l = a->tfd_l;
      f.tfd_tgtfd = a->tfd_tgtfd;
    }
    double r[9];
    calc_cost_reg(&f, x + (size_t)z * N, r, gfrm.data());
    if (lc_on) lcc += r[6] / Nz;
    else tfdc += r[6] / Nz;
    l1c += r[1] / Nz;
    smc += r[8] / Nz;
    tvc += r[2] / Nz;
    tsvc += r[3] / Nz;
    klc += r[4] / Nz;
    gsc += r[5] / Nz;
    regs += r[0] / Nz;
    for (int i = 0; i < N; ++i) greg[(size_t)z * N + i] = gfrm[i] / Nz;
  }
  double rtc = 0, ric = 0;
  if (a->cen_l > 0 || a->rt_l > 0 || a->ri_l > 0 || a->rs_l > 0) {
    cost_dynamical(a, x, rtc, ric, greg.data());
    regs += rtc + ric;
  }
  for (size_t i = 0; i < (size_t)N * Nz; ++i) grad[i] = gchi[i] + greg[i];
  const double t[20] = {chisq, cfcv, camp, ccp, cca, regs, l1c, smc, tvc, tsvc,
                        klc, gsc, tfdc, lcc, 0.0, rtc, ric, 0.0, 0.0, chisq + regs};
  std::memcpy(terms, t, sizeof(t));
  return 0;
}

// fftim3d.imaging (fftim3d.f90:11-467)
extern "C" int orc_imaging3d(const orc_args3d* a, int niter, int nonneg, int nprint, int m, double factr,
                             double pgtol, double eps, double* iout, double* terms, double* trace, int* nfg_out,
                             int* niter_out, int* task_out) {
  (void)nprint;
  const int n = a->npix * a->nz;
  double wtotal = 0;
  if (a->isfcv) wtotal += 2 * a->nfcv * a->wfcv;
  if (a->isamp) wtotal += a->namp * a->wamp;
  if (a->iscp) wtotal += a->ncp * a->wcp;
  if (a->isca) wtotal += a->nca * a->wca;
  const double wfcv_n = a->isfcv ? a->wfcv / wtotal : 0;
  const double wamp_n = a->isamp ? a->wamp / wtotal : 0;
  const double wcp_n = a->iscp ? a->wcp / wtotal : 0;
  const double wca_n = a->isca ? a->wca / wtotal : 0;
  std::memcpy(iout, a->iin, sizeof(double) * n);
  std::vector<double> vr(std::max(a->nfcv, 1), 0.0), vi(std::max(a->nfcv, 1), 0.0);
  if (a->isfcv) {
    const double dix = a->nxref - a->nx / 2.0 - 1, diy = a->nyref - a->ny / 2.0 - 1;
    for (int i = 0; i < a->nfcv; ++i) {
      const int k = std::abs(a->uvidxfcv[i]) - 1, s = isign(a->uvidxfcv[i]);
      const double ut = a->u[k] * s, vt = a->v[k] * s;
      const cplx out = cplx(a->vfcvr[i], a->vfcvi[i]) * std::exp(cplx(0.0, ut * dix + vt * diy));
      vr[i] = out.real();
      vi[i] = out.imag();
    }
  }
  std::vector<double> g(n), lo(n, 0.0);
  std::vector<int> nbd(n, nonneg ? 1 : 0);
  double t20[20];
  orc_calc_cost3d(a, vr.data(), vi.data(), wfcv_n, wamp_n, wcp_n, wca_n, iout, eps, t20, g.data());
  void* h = orc_lbfgsb_new(n, m, lo.data(), nullptr, nbd.data(), factr, pgtol);
  double cost = t20[19];
  int task = orc_lbfgsb_step(h, iout, cost, g.data());
  int nfg = 1;
  while (task == ORC_TASK_FG || task == ORC_TASK_NEW_X) {
    if (task == ORC_TASK_FG) {
      orc_calc_cost3d(a, vr.data(), vi.data(), wfcv_n, wamp_n, wcp_n, wca_n, iout, eps, t20, g.data());
      cost = t20[19];
      ++nfg;
    } else {
      int it = 0;
      orc_lbfgsb_info(h, &it, nullptr, nullptr, nullptr, nullptr);
      if (trace && it - 1 <= niter) trace[it - 1] = cost;
      if (it > niter) {
        task = ORC_TASK_STOP;
        break;
      }
    }
    task = orc_lbfgsb_step(h, iout, cost, g.data());
  }
  int it = 0;
  orc_lbfgsb_info(h, &it, nullptr, nullptr, nullptr, nullptr);
  orc_lbfgsb_free(h);
  orc_calc_cost3d(a, vr.data(), vi.data(), wfcv_n, wamp_n, wcp_n, wca_n, iout, eps, terms, g.data());
  for (int i = 0; i < n; ++i)
    if (std::fabs(iout[i]) < kZeroEps) iout[i] = 0.0;  // fftim3d.f90:466
  if (nfg_out) *nfg_out = nfg;
  if (niter_out) *niter_out = it;
  if (task_out) *task_out = task;
  return 0;
}
