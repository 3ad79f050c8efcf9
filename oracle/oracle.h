/* CPU oracle for the SMILI static-imaging hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against and the timed CPU baseline; the product never links,
 * loads or calls it.
 *
 * Parity status: the reference's own path (Fortran fortlib + FINUFFT + FFTW)
 * cannot be built in this image, and the reference ships no tests or golden
 * vectors for it.  The oracle is therefore a restatement:
 *   - get_uvlist is pinned bit-exactly against the reference's own Python
 *     (tests/golden/uvlist_*.npz);
 *   - L-BFGS-B is pinned against scipy's L-BFGS-B (the same v3.0 algorithm
 *     as src/lbfgsb/lbfgsb.f) on identical objectives;
 *   - the NUFFT is pinned against the exact DFT (its mathematical definition,
 *     src/wrapfinufft/wrapfinufft.f90:94-206) and the chi-square and
 *     regularizer gradients against finite differences;
 *   - the chi-square/regularizer arithmetic itself is "parity unpinned": it is
 *     restated line by line from src/fortlib/fftlib.f90 and image.f90 with no
 *     reference output to compare against.
 */
#ifndef SMILI_ORACLE_H
#define SMILI_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Arguments of fortlib.fftim2d.imaging / calc_cost (fftim2d.f90:11-34,387-410).
 * Arrays follow the Fortran layouts: uvidxcp is (3,Ncp) column-major, i.e.
 * the three indices of closure phase i are contiguous. */
typedef struct {
  int npix, nx, ny;
  const double* iin;
  const int* xidx;
  const int* yidx;
  double nxref, nyref;
  int nuv;
  const double* u;
  const double* v;
  double l1_l;  const double* l1_wgt;  int l1_nwgt;
  double tv_l;  const double* tv_wgt;  int tv_nwgt;
  double tsv_l; const double* tsv_wgt; int tsv_nwgt;
  double kl_l;  const double* kl_wgt;  int kl_nwgt;
  double gs_l;  const double* gs_wgt;  int gs_nwgt;
  double tfd_l, tfd_tgtfd;
  double cen_l, cen_alpha;
  double sm_l, sm_maj, sm_min, sm_phi;
  int isfcv, nfcv; const int* uvidxfcv; const double* vfcvr; const double* vfcvi; const double* varfcv; double wfcv;
  int isamp, namp; const int* uvidxamp; const double* vamp; const double* varamp; double wamp;
  int iscp, ncp;   const int* uvidxcp;  const double* cp;   const double* varcp;  double wcp;
  int isca, nca;   const int* uvidxca;  const double* ca;   const double* varca;  double wca;
  double inormfactr;
} orc_args;

/* terms[15] = chisq, chisqfcv, chisqamp, chisqcp, chisqca, reg, l1, tv, tsv,
 * kl, gs, tfd, cen, sm, cost (the intent(out) order of fftim2d.imaging). */

/* NUFFT with the exponential-of-semicircle kernel at tolerance eps
 * (eps <= 0 selects the exact direct DFT).  Image (nx,ny) in Fortran order. */
int orc_nufft2d2(int nuv, const double* u, const double* v, int nx, int ny,
                 const double* img, double eps, double* vre, double* vim);
int orc_nufft2d1(int nuv, const double* u, const double* v, const double* cre,
                 const double* cim, int nx, int ny, double eps, double* ore, double* oim);

/* One function/gradient evaluation: calc_cost (fftim2d.f90:387-607) with the
 * visibilities already phase-shifted (Vfcv as passed to calc_cost) and the
 * normalised data weights. */
int orc_calc_cost(const orc_args* a, const double* vfcv_shifted_re, const double* vfcv_shifted_im,
                  double wfcv_n, double wamp_n, double wcp_n, double wca_n,
                  const double* x, double eps, double* terms, double* grad);

/* fortlib.fftim2d.imaging (fftim2d.f90:11-382).  trace (optional, length
 * >= niter+1) receives the cost at every NEW_X; nfg/niter_done/task report
 * the solver's counters and its final task code. */
int orc_imaging(const orc_args* a, int niter, int nonneg, int nprint, int m, double factr,
                double pgtol, double eps, double* iout, double* terms, double* trace,
                int* nfg, int* niter_done, int* task);

/* Arguments of fortlib.fftim3d.imaging / calc_cost (fftim3d.f90:11-44,
 * 473-498): a movie of nz frames of npix pixels (frame-major), u/v the
 * concatenation of the frames' uv lists with nuvs[nz] points per frame. */
typedef struct {
  int npix, nx, ny, nz;
  const double* iin;
  const int* xidx;
  const int* yidx;
  double nxref, nyref;
  int nuv;
  const double* u;
  const double* v;
  const int* nuvs;
  double l1_l;  const double* l1_wgt;
  double tv_l;  const double* tv_wgt;
  double tsv_l; const double* tsv_wgt;
  double kl_l;  const double* kl_wgt;
  double gs_l;  const double* gs_wgt;
  double tfd_l, tfd_tgtfd;
  const double* lc_l;
  const double* lc_tgtfd;
  int lc_nidx;
  double cen_l, cen_alpha;
  double sm_l, sm_maj, sm_min, sm_phi;
  double rt_l; const double* rt_wgt;
  double ri_l; const double* ri_wgt;
  double rs_l, rf_l;
  int isfcv, nfcv; const int* uvidxfcv; const double* vfcvr; const double* vfcvi; const double* varfcv; double wfcv;
  int isamp, namp; const int* uvidxamp; const double* vamp; const double* varamp; double wamp;
  int iscp, ncp;   const int* uvidxcp;  const double* cp;   const double* varcp;  double wcp;
  int isca, nca;   const int* uvidxca;  const double* ca;   const double* varca;  double wca;
  double inormfactr;
} orc_args3d;

/* terms[20] = chisq, chisqfcv, chisqamp, chisqcp, chisqca, reg, l1, sm, tv,
 * tsv, kl, gs, tfd, lc, cen, rt, ri, rs, rf, cost (fftim3d.imaging order). */
int orc_calc_cost3d(const orc_args3d* a, const double* vfcv_shifted_re, const double* vfcv_shifted_im,
                    double wfcv_n, double wamp_n, double wcp_n, double wca_n,
                    const double* x, double eps, double* terms, double* grad);
int orc_imaging3d(const orc_args3d* a, int niter, int nonneg, int nprint, int m, double factr,
                  double pgtol, double eps, double* iout, double* terms, double* trace,
                  int* nfg, int* niter_done, int* task);

/* Reverse-communication L-BFGS-B restatement (src/lbfgsb/lbfgsb.f).
 * nbd: 0 none, 1 lower, 2 both, 3 upper.  Returns a task code
 * (see ORC_TASK_*). */
enum { ORC_TASK_FG = 1, ORC_TASK_NEW_X = 2, ORC_TASK_CONV = 3, ORC_TASK_ABNORMAL = 4,
       ORC_TASK_ERROR = 5, ORC_TASK_STOP = 6 };
void* orc_lbfgsb_new(int n, int m, const double* l, const double* u, const int* nbd,
                     double factr, double pgtol);
int orc_lbfgsb_step(void* h, double* x, double f, const double* g);
int orc_lbfgsb_info(void* h, int* iter, int* nfgv, int* col, double* theta, double* sbgnrm);
void orc_lbfgsb_free(void* h);

int orc_nthreads(void);
#ifdef __cplusplus
}
#endif
#endif
