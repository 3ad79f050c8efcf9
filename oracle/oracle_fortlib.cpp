// CPU oracle, part 3: chi-square terms, regularizers, calc_cost and the
// fftim2d.imaging driver (test infrastructure only).
//
// Restates src/fortlib/fftlib.f90:250-655 (calc_chisq and the four chi-square
// kernels), src/fortlib/image.f90:12-200 + the per-pixel functions
// (calc_cost_reg, l1/kl/gs/tv/tsv/tfd/cen/sm) and
// src/fortlib/fftim2d.f90:11-607 (imaging, calc_cost).  The arithmetic and
// the evaluation order follow the Fortran statement by statement, including
// its quirks (tv_grade resetting the accumulated gradient, 2(1-cos r) closure
// phase chi-square, smabs epsilon 1e-10).  Loops that the reference runs
// under OpenMP array reductions are summed here in a fixed order so the oracle
// is deterministic.
#include "oracle.h"
#include "oracle_internal.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

namespace orc {

const double kZeroEps = 1e-10;  // image.f90:7

inline double smabs_diff(double x) { return x / smabs(x); }

// --------------------------- chi-square terms ------------------------------
// fftlib.f90:384-439
void chisq_fcv(const cplx* V, const int* uvidx, const cplx* Vd, const double* var, double fnorm,
               int n, double& chisq, double* rre, double* rim) {
  for (int i = 0; i < n; ++i) {
    const int k = std::abs(uvidx[i]) - 1;
    const cplx model = uvidx[i] > 0 ? V[k] : std::conj(V[k]);
    const cplx resid = Vd[i] - model;
    chisq += std::norm(resid) / var[i] * fnorm;
    const double factor = -2.0 / var[i] * fnorm;
    rre[k] += factor * resid.real();
    rim[k] += factor * resid.imag() * isign(uvidx[i]);
  }
}

// fftlib.f90:442-493
void chisq_amp(const cplx* V, const int* uvidx, const double* A, const double* var, double fnorm,
               int n, double& chisq, double* rre, double* rim) {
  for (int i = 0; i < n; ++i) {
    const int k = std::abs(uvidx[i]) - 1;
    const double model = std::abs(V[k]);
    const double resid = A[i] - model;
    chisq += resid * resid / var[i] * fnorm;
    const double factor = -2.0 * resid / var[i] / model * fnorm;
    rre[k] += factor * V[k].real();
    rim[k] += factor * V[k].imag();
  }
}

// fftlib.f90:496-573
void chisq_ca(const cplx* V, const int* uvidx, const double* CA, const double* var, double fnorm,
              int n, double& chisq, double* rre, double* rim) {
  for (int i = 0; i < n; ++i) {
    int k[4];
    cplx Vk[4];
    double a[4];
    for (int q = 0; q < 4; ++q) {
      k[q] = std::abs(uvidx[4 * i + q]) - 1;
      Vk[q] = V[k[q]];
      a[q] = std::abs(Vk[q]);
    }
    const double model = std::log(a[0]) + std::log(a[1]) - std::log(a[2]) - std::log(a[3]);
    const double resid = CA[i] - model;
    chisq += resid * resid / var[i] * fnorm;
    const double factor = -2.0 * resid / var[i] * fnorm;
    rre[k[0]] += factor / (a[0] * a[0]) * Vk[0].real();
    rre[k[1]] += factor / (a[1] * a[1]) * Vk[1].real();
    rre[k[2]] -= factor / (a[2] * a[2]) * Vk[2].real();
    rre[k[3]] -= factor / (a[3] * a[3]) * Vk[3].real();
    rim[k[0]] += factor / (a[0] * a[0]) * Vk[0].imag();
    rim[k[1]] += factor / (a[1] * a[1]) * Vk[1].imag();
    rim[k[2]] -= factor / (a[2] * a[2]) * Vk[2].imag();
    rim[k[3]] -= factor / (a[3] * a[3]) * Vk[3].imag();
  }
}

// fftlib.f90:576-655
void chisq_cp(const cplx* V, const int* uvidx, const double* CP, const double* var, double fnorm,
              int n, double& chisq, double* rre, double* rim) {
  for (int i = 0; i < n; ++i) {
    int k[3], s[3];
    cplx Vk[3];
    double a2[3];
    for (int q = 0; q < 3; ++q) {
      k[q] = std::abs(uvidx[3 * i + q]) - 1;
      s[q] = isign(uvidx[3 * i + q]);
      Vk[q] = V[k[q]];
      a2[q] = std::norm(Vk[q]);
    }
    double model = std::atan2(Vk[0].imag(), Vk[0].real()) * s[0];
    model = std::atan2(Vk[1].imag(), Vk[1].real()) * s[1] + model;
    model = std::atan2(Vk[2].imag(), Vk[2].real()) * s[2] + model;
    const double resid = CP[i] - model;
    chisq += 2.0 * (1.0 - std::cos(resid)) / var[i] * fnorm;
    const double factor = -2.0 * std::sin(resid) / var[i] * fnorm;
    for (int q = 0; q < 3; ++q) rre[k[q]] -= factor / a2[q] * Vk[q].imag() * s[q];
    for (int q = 0; q < 3; ++q) rim[k[q]] += factor / a2[q] * Vk[q].real() * s[q];
  }
}

// ----------------------------- regularizers --------------------------------
// I2d is (Nx,Ny) Fortran order: I2d(i,j) = img[(j-1)*Nx + (i-1)]
struct Img2 {
  const double* a;
  int nx, ny;
  double operator()(int i, int j) const { return a[(size_t)(j - 1) * nx + (i - 1)]; }
};

double tv_e(int i1, int j1, const Img2& I) {  // image.f90:477-508
  const int i2 = i1 + 1, j2 = j1 + 1;
  const double dIx = (i2 > I.nx) ? 0.0 : I(i2, j1) - I(i1, j1);
  const double dIy = (j2 > I.ny) ? 0.0 : I(i1, j2) - I(i1, j1);
  return std::sqrt(dIx * dIx + dIy * dIy);
}

double tv_grade(int i1, int j1, const Img2& I) {  // image.f90:512-612
  double g = 0.0;
  const int i0 = i1 - 1, j0 = j1 - 1, i2 = i1 + 1, j2 = j1 + 1;
  double dIx = (i2 > I.nx) ? 0.0 : I(i2, j1) - I(i1, j1);
  double dIy = (j2 > I.ny) ? 0.0 : I(i1, j2) - I(i1, j1);
  double e = std::sqrt(dIx * dIx + dIy * dIy);
  if (e > kZeroEps) g -= (dIx + dIy) / e;
  if (i0 > 0) {
    dIx = I(i1, j1) - I(i0, j1);
    dIy = (j2 > I.ny) ? 0.0 : I(i0, j2) - I(i0, j1);
    e = std::sqrt(dIx * dIx + dIy * dIy);
    if (e > kZeroEps)
      g += dIx / e;
    else
      g = 0.0;  // reference resets the accumulated gradient (image.f90:577-578)
  }
  if (j0 > 0) {
    dIy = I(i1, j1) - I(i1, j0);
    dIx = (i2 > I.nx) ? 0.0 : I(i2, j0) - I(i1, j0);
    e = std::sqrt(dIx * dIx + dIy * dIy);
    if (e > kZeroEps)
      g += dIy / e;
    else
      g = 0.0;  // image.f90:603-604
  }
  return g;
}

double tsv_e(int i1, int j1, const Img2& I) {  // image.f90:678-711
  const int i2 = i1 + 1, j2 = j1 + 1;
  const double dIx = (i2 > I.nx) ? 0.0 : I(i2, j1) - I(i1, j1);
  const double dIy = (j2 > I.ny) ? 0.0 : I(i1, j2) - I(i1, j1);
  return dIx * dIx + dIy * dIy;
}

double tsv_grade(int i1, int j1, const Img2& I) {  // image.f90:715-754
  double g = 0.0;
  const int i0 = i1 - 1, j0 = j1 - 1, i2 = i1 + 1, j2 = j1 + 1;
  if (i2 <= I.nx) g -= 2 * (I(i2, j1) - I(i1, j1));
  if (j2 <= I.ny) g -= 2 * (I(i1, j2) - I(i1, j1));
  if (i0 > 0) g += 2 * (I(i1, j1) - I(i0, j1));
  if (j0 > 0) g += 2 * (I(i1, j1) - I(i1, j0));
  return g;
}

inline double kl_e(double I, double P) {
  const double a = smabs(I);
  return a * std::log(a / P) + P / M_E;
}
inline double kl_grade(double I, double P) { return smabs_diff(I) * (std::log(smabs(I) / P) + 1); }
inline double gs_e(double I, double P) {
  const double a = smabs(I);
  return a * (std::log(a / P) - 1) + P;
}
inline double gs_grade(double I, double P) { return smabs_diff(I) * std::log(smabs(I) / P); }

// second moment helpers (image.f90:964-1138)
void sigma_prior(double maj, double mnr, double phi, double* sp) {
  sp[0] = mnr * std::cos(phi) * std::cos(phi) + maj * std::sin(phi) * std::sin(phi);
  sp[1] = mnr * std::sin(phi) * std::sin(phi) + maj * std::cos(phi) * std::cos(phi);
  sp[2] = (maj - mnr) * std::sin(phi) * std::cos(phi);
}

void xy_cen(const double* I, const int* x, const int* y, int n, double& xc, double& yc) {
  xc = yc = 0.0;
  double tot = 0.0;
  for (int i = 0; i < n; ++i) {
    xc += x[i] * I[i];
    yc += y[i] * I[i];
    tot += std::fabs(I[i]);
  }
  xc /= tot;
  yc /= tot;
}

// calc_cost_reg (image.f90:12-200).  reg[9] = cost, l1, tv, tsv, kl, gs, tfd, cen, sm
void calc_cost_reg(const orc_args* a, const double* I1d, double* reg, double* grad) {
  const int N = a->npix;
  double l1c = 0, tvc = 0, tsvc = 0, gsc = 0, klc = 0, tfdc = 0, cenc = 0, smc = 0;
  std::fill(grad, grad + N, 0.0);
  if (a->tfd_l > 0) {  // calc_tfdreg (image.f90:777-787)
    double s = 0;
    for (int i = 0; i < N; ++i) s += I1d[i];
    const double resid = s - a->tfd_tgtfd;
    tfdc = a->tfd_l * resid * resid;
    for (int i = 0; i < N; ++i) grad[i] += a->tfd_l * 2 * resid;
  }
  if (a->cen_l > 0) {  // calc_cenreg (image.f90:793-863)
    const double alpha = a->cen_alpha;
    double sx = 0, sy = 0, sI = kZeroEps;
    for (int i = 0; i < N; ++i) {
      const double dix = a->xidx[i] - a->nxref, diy = a->yidx[i] - a->nyref;
      const double Ip = std::fabs(alpha - 1) < kZeroEps ? smabs(I1d[i]) : std::pow(smabs(I1d[i]), alpha);
      sx += Ip * dix;
      sy += Ip * diy;
      sI += Ip;
    }
    sx /= sI;
    sy /= sI;
    const double c = std::sqrt(sx * sx + sy * sy + kZeroEps);
    cenc = a->cen_l * c;
    for (int i = 0; i < N; ++i) {
      const double dix = a->xidx[i] - a->nxref, diy = a->yidx[i] - a->nyref;
      const double gIp = std::fabs(alpha - 1) < kZeroEps
                             ? smabs_diff(I1d[i])
                             : smabs_diff(I1d[i]) * alpha * std::pow(smabs(I1d[i]), alpha - 1);
      grad[i] += a->cen_l * ((sx * (dix - sx) + sy * (diy - sy)) / sI / c * gIp);
    }
  }
  double Isum = 0, xcen = 0, ycen = 0, Sg[3] = {0, 0, 0}, mom[2] = {0, 0}, Sp[3] = {0, 0, 0};
  if (a->sm_l > 0) {
    for (int i = 0; i < N; ++i) Isum += std::fabs(I1d[i]);
    xy_cen(I1d, a->xidx, a->yidx, N, xcen, ycen);
    for (int i = 0; i < N; ++i) {
      const double dx = a->xidx[i] - xcen, dy = a->yidx[i] - ycen;
      Sg[0] += I1d[i] * dx * dx / Isum;
      Sg[1] += I1d[i] * dy * dy / Isum;
      Sg[2] += I1d[i] * dx * dy / Isum;
    }
    double xc2, yc2;
    xy_cen(I1d, a->xidx, a->yidx, N, xc2, yc2);
    for (int i = 0; i < N; ++i) {
      mom[0] += (a->xidx[i] - xc2) * I1d[i];
      mom[1] += (a->yidx[i] - yc2) * I1d[i];
    }
    sigma_prior(a->sm_maj, a->sm_min, a->sm_phi, Sp);
    double e = 0;
    for (int q = 0; q < 2; ++q) e += (Sg[q] - Sp[q]) * (Sg[q] - Sp[q]);
    e += 2. * (Sg[2] - Sp[2]) * (Sg[2] - Sp[2]);
    smc += a->sm_l * e;
  }
  std::vector<double> I2d;
  Img2 im{nullptr, a->nx, a->ny};
  if (a->tv_l > 0 || a->tsv_l > 0) {
    I2d.assign((size_t)a->nx * a->ny, 0.0);
    for (int i = 0; i < N; ++i) I2d[(size_t)(a->yidx[i] - 1) * a->nx + (a->xidx[i] - 1)] = I1d[i];
    im.a = I2d.data();
  }
  for (int i = 0; i < N; ++i) {
    const double I = I1d[i];
    if (a->l1_l > 0) {
      l1c += a->l1_l * a->l1_wgt[i] * smabs(I);
      grad[i] += a->l1_l * a->l1_wgt[i] * smabs_diff(I);
    }
    if (a->kl_l > 0) {
      klc += a->kl_l * kl_e(I, a->kl_wgt[i]);
      grad[i] += a->kl_l * kl_grade(I, a->kl_wgt[i]);
    }
    if (a->gs_l > 0) {
      gsc += a->gs_l * gs_e(I, a->gs_wgt[i]);
      grad[i] += a->gs_l * gs_grade(I, a->gs_wgt[i]);
    }
    if (a->tv_l > 0) {
      tvc += a->tv_l * a->tv_wgt[i] * tv_e(a->xidx[i], a->yidx[i], im);
      grad[i] += a->tv_l * a->tv_wgt[i] * tv_grade(a->xidx[i], a->yidx[i], im);
    }
    if (a->tsv_l > 0) {
      tsvc += a->tsv_l * a->tsv_wgt[i] * tsv_e(a->xidx[i], a->yidx[i], im);
      grad[i] += a->tsv_l * a->tsv_wgt[i] * tsv_grade(a->xidx[i], a->yidx[i], im);
    }
    if (a->sm_l > 0) {  // sm_grade (image.f90:883-925)
      const double xg = (a->xidx[i] - xcen) / Isum, yg = (a->yidx[i] - ycen) / Isum;
      const double dx = a->xidx[i] - xcen, dy = a->yidx[i] - ycen;
      double Sgg[3];
      Sgg[0] = ((dx * dx - 2. * xg * mom[0]) - Sg[0]) / Isum;
      Sgg[1] = ((dy * dy - 2. * yg * mom[1]) - Sg[1]) / Isum;
      Sgg[2] = (dx * dy - xg * mom[1] - yg * mom[0] - Sg[2]) / Isum;
      grad[i] += a->sm_l * (2. * (Sg[0] - Sp[0]) * Sgg[0] + 2. * (Sg[1] - Sp[1]) * Sgg[1] +
                            4. * (Sg[2] - Sp[2]) * Sgg[2]);
    }
  }
  reg[1] = l1c;
  reg[2] = tvc;
  reg[3] = tsvc;
  reg[4] = klc;
  reg[5] = gsc;
  reg[6] = tfdc;
  reg[7] = cenc;
  reg[8] = smc;
  reg[0] = l1c + tvc + tsvc + klc + gsc + tfdc + cenc + smc;
}

}  // namespace orc

using namespace orc;

// calc_cost (fftim2d.f90:387-607) = calc_chisq (fftlib.f90:250-382) + calc_cost_reg
extern "C" int orc_calc_cost(const orc_args* a, const double* vre_s, const double* vim_s,
                             double wfcv, double wamp, double wcp, double wca, const double* x,
                             double eps, double* terms, double* grad) {
  const int N = a->npix, nx = a->nx, ny = a->ny, nuv = a->nuv;
  std::vector<double> I2d((size_t)nx * ny, 0.0);
  for (int i = 0; i < N; ++i) I2d[(size_t)(a->yidx[i] - 1) * nx + (a->xidx[i] - 1)] = x[i];
  std::vector<double> vr(nuv), vi(nuv);
  orc_nufft2d2(nuv, a->u, a->v, nx, ny, I2d.data(), eps, vr.data(), vi.data());
  std::vector<cplx> V(nuv);
  for (int j = 0; j < nuv; ++j) V[j] = cplx(vr[j], vi[j]);
  std::vector<double> rre(nuv, 0.0), rim(nuv, 0.0);
  double chisq = 0, cfcv = 0, camp = 0, ccp = 0, cca = 0;
  if (a->isfcv) {
    std::vector<cplx> Vd(a->nfcv);
    for (int i = 0; i < a->nfcv; ++i) Vd[i] = cplx(vre_s[i], vim_s[i]);
    chisq_fcv(V.data(), a->uvidxfcv, Vd.data(), a->varfcv, wfcv, a->nfcv, cfcv, rre.data(),
              rim.data());
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
  // NUFFT_adj_resid (fftlib.f90:152-174): two type-1 transforms, Re + Im
  std::vector<double> zero(nuv, 0.0), g1r((size_t)nx * ny), g1i((size_t)nx * ny),
      g2r((size_t)nx * ny), g2i((size_t)nx * ny);
  orc_nufft2d1(nuv, a->u, a->v, rre.data(), zero.data(), nx, ny, eps, g1r.data(), g1i.data());
  orc_nufft2d1(nuv, a->u, a->v, rim.data(), zero.data(), nx, ny, eps, g2r.data(), g2i.data());
  std::vector<double> greg(N);
  double reg[9];
  calc_cost_reg(a, x, reg, greg.data());
  for (int i = 0; i < N; ++i) {
    const size_t p = (size_t)(a->yidx[i] - 1) * nx + (a->xidx[i] - 1);
    grad[i] = (g1r[p] + g2i[p]) + greg[i];
  }
  terms[0] = chisq;
  terms[1] = cfcv;
  terms[2] = camp;
  terms[3] = ccp;
  terms[4] = cca;
  for (int q = 0; q < 9; ++q) terms[5 + q] = reg[q];
  terms[14] = chisq + reg[0];
  return 0;
}

// fftim2d.imaging (fftim2d.f90:11-382)
extern "C" int orc_imaging(const orc_args* a, int niter, int nonneg, int nprint, int m,
                           double factr, double pgtol, double eps, double* iout, double* terms,
                           double* trace, int* nfg_out, int* niter_out, int* task_out) {
  (void)nprint;  // the nprint summaries re-evaluate calc_cost at the same x: no effect on x
  const int N = a->npix;
  double wtotal = 0;
  if (a->isfcv) wtotal += 2 * a->nfcv * a->wfcv;
  if (a->isamp) wtotal += a->namp * a->wamp;
  if (a->iscp) wtotal += a->ncp * a->wcp;
  if (a->isca) wtotal += a->nca * a->wca;
  const double wfcv_n = a->isfcv ? a->wfcv / wtotal : 0;
  const double wamp_n = a->isamp ? a->wamp / wtotal : 0;
  const double wcp_n = a->iscp ? a->wcp / wtotal : 0;
  const double wca_n = a->isca ? a->wca / wtotal : 0;
  std::memcpy(iout, a->iin, sizeof(double) * N);
  // phashift_r2c of the data (fftim2d.f90:224-241, fftlib.f90:223-244)
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
  } else {
    for (int i = 0; i < std::max(a->nfcv, 1); ++i) {
      vr[i] = a->vfcvr[i];
      vi[i] = a->vfcvi[i];
    }
  }
  std::vector<double> g(N), lo(N, 0.0);
  std::vector<int> nbd(N, nonneg ? 1 : 0);
  double t15[15];
  orc_calc_cost(a, vr.data(), vi.data(), wfcv_n, wamp_n, wcp_n, wca_n, iout, eps, t15, g.data());
  void* h = orc_lbfgsb_new(N, m, lo.data(), nullptr, nbd.data(), factr, pgtol);
  double cost = t15[14];
  int task = orc_lbfgsb_step(h, iout, cost, g.data());  // START -> FG
  int nfg = 1;
  while (task == ORC_TASK_FG || task == ORC_TASK_NEW_X) {
    if (task == ORC_TASK_FG) {
      orc_calc_cost(a, vr.data(), vi.data(), wfcv_n, wamp_n, wcp_n, wca_n, iout, eps, t15, g.data());
      cost = t15[14];
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
  // final summary (fftim2d.f90:356-376)
  orc_calc_cost(a, vr.data(), vi.data(), wfcv_n, wamp_n, wcp_n, wca_n, iout, eps, terms, g.data());
  if (nfg_out) *nfg_out = nfg;
  if (niter_out) *niter_out = it;
  if (task_out) *task_out = task;
  return 0;
}
