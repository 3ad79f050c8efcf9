// Persistent batched solver kernel and the C ABI (include/smili_b200.h).
//
// One cooperative launch solves a whole batch: the CTAs are split into groups
// of G; a group takes the next unsolved problem from a queue and runs
// function/gradient evaluation (fg.cuh) and L-BFGS-B (lbfgsb.cuh) until the
// problem stops, then takes the next one.  Stages inside a group are
// separated by group barriers (common.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/smili_b200.h"
#include "common.cuh"
#include "fft.cuh"
#include "fg.cuh"
#include "layout.h"
#include "lbfgsb.cuh"

#define SMILI_VERSION 1
#define SMILI_SMEM_CPX 2048   // complex elements per FFT buffer
#define SMILI_DYN_CPX 6144    // complex elements of dynamic shared memory (96 KB FP64)

enum { MODE_SOLVE = 0, MODE_FG = 1, MODE_T2 = 2, MODE_T1 = 3, MODE_BARRIER = 4, MODE_WAIT_LIMIT = 5 };

// polls of a group-barrier wait in the wait-limit check (MODE_WAIT_LIMIT):
// about 10 ms, instead of the seconds a real barrier may wait
#define SMILI_TEST_SPIN_LIMIT (1LL << 14)

struct BatchArgs {
  char* arena;
  const ProbDesc* descs;
  int nprob, G, mode;
  int* queue;
  unsigned* bars;      // [ngroups][2]
  double* red_part;    // [ngroups][G][SMILI_REDK]
  double* red_out;     // [ngroups][SMILI_REDK]
  int* grp_prob;       // [ngroups]
  int* abort_flag;
  ProbResult* results; // [nprob]
  unsigned long long* prof;  // [PR_NSTAGE] stage times (ns) or null
};

// ---------------------------------------------------------------------------
// one function/gradient evaluation by the group (stages F1..F8)
// ---------------------------------------------------------------------------
// Stages F1-F8 of one evaluation of a 2D problem by group g: per-thread
// partial sums acc[0..3] = chi-square terms (weighted), acc[4..11] = the
// per-pixel regularizers (l1, tv, tsv, kl, gs, -, -, -), acc[12] = g.d,
// acc[13] = projected-gradient max, and the image moments rm.  opt_terms
// false leaves acc[12..13] alone (a movie frame).  A frame without data
// (nuv == 0) only evaluates its regularizers.
template <typename R>
__device__ bool fg_stages(FgCtx<R>& fc, GroupCtx& g, int lo, int hi, double* red, unsigned char* ops,
                          double* scratch, double (&acc)[16], RegMoments& rm, int mode, bool opt_terms,
                          Prof& pf) {
  const ProbDesc& P = *fc.P;
  memset(&rm, 0, sizeof(rm));
  double chi[4] = {0, 0, 0, 0};
  if (P.nuv > 0) {
    double mom[10];
    for (int k = 0; k < 10; ++k) mom[k] = 0.0;
    fg_t2_rows(fc, g, mom);
    if (P.has_tfd || P.has_cen || P.has_sm) {
      for (int k = threadIdx.x; k < 10; k += blockDim.x) ops[k] = RED_SUM;
      __syncthreads();
      block_reduce_arr(mom, ops, 10, red, scratch);
      if (!group_reduce(g, red, ops, 10)) return false;
      double mm[10];
      for (int k = 0; k < 10; ++k) mm[k] = red[k];
      reg_moments(P, mm, rm);
      __syncthreads();
    } else if (!group_sync(g)) {
      return false;
    }
    pf.mark(PR_F1);
    fg_t2_cols(fc, g);
    if (!group_sync(g)) return false;
    pf.mark(PR_F2);
    fg_interp(fc, g, mode != MODE_T1);
    if (!group_sync(g)) return false;
    pf.mark(PR_F3);
    if (mode == MODE_T2) return true;
    if (mode != MODE_T1) {
      fg_chisq(fc, g, chi);
      if (!group_sync(g)) return false;
    }
    pf.mark(PR_F4);
    fg_spread(fc, g);
    if (!group_sync(g)) return false;
    pf.mark(PR_F5);
    fg_t1_rows(fc, g);
    if (!group_sync(g)) return false;
    pf.mark(PR_F6);
    fg_t1_cols(fc, g);
    if (!group_sync(g)) return false;
    pf.mark(PR_F7);
    if (mode == MODE_T1) return true;
  } else if (P.has_tfd || P.has_sm) {
    double mom[10];
    for (int k = 0; k < 10; ++k) mom[k] = 0.0;
    frame_moments(P, fc.base, mom);
    for (int k = threadIdx.x; k < 10; k += blockDim.x) ops[k] = RED_SUM;
    __syncthreads();
    block_reduce_arr(mom, ops, 10, red, scratch);
    double mm[10];
    for (int k = 0; k < 10; ++k) mm[k] = red[k];
    reg_moments(P, mm, rm);
    __syncthreads();
  }
  double reg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  fg_reg_grad<R>(P, fc.base, g, rm, lo, hi, reg, acc[12], acc[13], opt_terms);
  for (int k = 0; k < 4; ++k) acc[k] += chi[k];
  for (int k = 0; k < 8; ++k) acc[4 + k] += reg[k];
  return true;
}

// global-sum regularizers of one 2D image (image.f90:108-135) from its moments
__device__ __forceinline__ void global_regs(const ProbDesc& P, const RegMoments& rm, double& tfd, double& cen,
                                            double& sm) {
  tfd = P.has_tfd ? P.tfd_l * rm.tfd_resid * rm.tfd_resid : 0.0;
  cen = P.has_cen ? P.cen_l * rm.cen_cost : 0.0;
  sm = 0.0;
  if (P.has_sm) {
    double e = 0;
    for (int q = 0; q < 2; ++q) e += (rm.Sg[q] - rm.Sp[q]) * (rm.Sg[q] - rm.Sp[q]);
    e += 2. * (rm.Sg[2] - rm.Sp[2]) * (rm.Sg[2] - rm.Sp[2]);
    sm = P.sm_l * e;
  }
}

// One evaluation of a 2D problem: f, g.d, projected-gradient norm and the
// 15 cost terms (fftim2d.f90:387-607).
template <typename R>
__device__ bool group_fg(FgCtx<R>& fc, GroupCtx& g, LbCtxT<R>& lc, double* red, unsigned char* ops,
                         double* scratch, double& f, double& gd, double& sbg, double* terms,
                         int mode) {
  const ProbDesc& P = *fc.P;
  Prof& pf = *lc.prof;
  pf.mark(PR_OTHER);
  double acc[16];
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  RegMoments rm;
  if (!fg_stages(fc, g, lc.lo, lc.hi, red, ops, scratch, acc, rm, mode, true, pf)) return false;
  if (mode == MODE_T1 || mode == MODE_T2) return true;
  for (int k = threadIdx.x; k < 14; k += blockDim.x) ops[k] = (k == 13) ? RED_MAX : RED_SUM;
  __syncthreads();
  block_reduce_arr(acc, ops, 14, red, scratch);
  if (!group_reduce(g, red, ops, 14)) return false;
  double r[14];
  for (int k = 0; k < 14; ++k) r[k] = red[k];
  __syncthreads();
  pf.mark(PR_F8);
  pf.count(PR_COUNT);
  global_regs(P, rm, r[4 + 5], r[4 + 6], r[4 + 7]);
  const double chisq = r[0] + r[1] + r[2] + r[3];
  double regs = 0;
  for (int k = 0; k < 8; ++k) regs += r[4 + k];
  f = chisq + regs;
  gd = r[12];
  sbg = r[13];
  if (threadIdx.x == 0) {
    terms[0] = chisq;
    terms[1] = P.nfcv ? r[0] / P.wfcv / (2.0 * P.nfcv) : 0.0;
    terms[2] = P.namp ? r[1] / P.wamp / P.namp : 0.0;
    terms[3] = P.ncp ? r[2] / P.wcp / P.ncp : 0.0;
    terms[4] = P.nca ? r[3] / P.wca / P.nca : 0.0;
    terms[5] = regs;
    for (int k = 0; k < 8; ++k) terms[6 + k] = r[4 + k];
    terms[14] = f;
  }
  __syncthreads();
  return true;
}

// One evaluation of a movie (fftim3d.f90:473-614, fftlib3d.f90:14-205,
// image3d.f90:15-425).  Every frame is a complete 2D evaluation run by one
// CTA (frames z = rank, rank + G, ...) with the frame's regularizer weights
// already divided by the frame count; after a group barrier the movie pass
// adds the Rt / Ri gradients (image3d.f90:280-392, Rt only for frames
// iz < Nz as the reference does) and forms g.d and the projected gradient
// over the whole vector.  terms[20] follow the fftim3d.imaging order.
template <typename R>
__device__ bool movie_fg(FgCtx<R>& fc, GroupCtx& g, LbCtxT<R>& lc, double* red, unsigned char* ops,
                         double* scratch, double& f, double& gd, double& sbg, double* terms) {
  const ProbDesc& M = *fc.P;
  char* base = fc.base;
  Prof& pf = *lc.prof;
  pf.mark(PR_OTHER);
  const ProbDesc* frames = at<ProbDesc>(base, M.o_frames);
  double acc[16];
  for (int k = 0; k < 16; ++k) acc[k] = 0.0;
  GroupCtx g1 = g;  // one CTA per frame: G == 1 barriers are block barriers
  g1.rank = 0;
  g1.G = 1;
  for (int z = g.rank; z < M.nframes; z += g.G) {
    FgCtx<R> fz = fc;
    fz.P = &frames[z];
    RegMoments rm;
    if (!fg_stages(fz, g1, 0, frames[z].npix, red, ops, scratch, acc, rm, MODE_FG, false, pf)) return false;
    if (threadIdx.x == 0) {
      double tfd, cen, sm;
      global_regs(frames[z], rm, tfd, cen, sm);
      acc[4 + 5] += tfd;  // the light-curve term when M.has_lc
      acc[4 + 7] += sm;
    }
    __syncthreads();
  }
  if (!group_sync(g)) return false;
  const int N = M.frame_npix, Nz = M.nframes;
  const double* x = lc.x;
  double* gv = lc.gv;
  const double* d = lc.d;
  const double* lcf = at<double>(base, M.o_lcf);
  double* iavg = M.has_ri ? at<double>(base, M.o_iavg) : nullptr;
  if (M.has_ri) {
    const int chunk = (N + g.G - 1) / g.G;
    const int p0 = min(N, g.rank * chunk), p1 = min(N, p0 + chunk);
    for (int i = p0 + threadIdx.x; i < p1; i += blockDim.x) {
      double s = 0.0;
      for (int z = 0; z < Nz; ++z) s += x[(size_t)z * N + i] / lcf[z] / Nz;
      iavg[i] = s;
    }
    if (!group_sync(g)) return false;
  }
  const double* rtw = M.has_rt ? at<double>(base, M.o_rtw) : nullptr;
  const double* riw = M.has_ri ? at<double>(base, M.o_riw) : nullptr;
  for (int idx = lc.lo + threadIdx.x; idx < lc.hi; idx += blockDim.x) {
    const int z = idx / N, i = idx - z * N;
    const double II = x[idx] / lcf[z];
    double gr = 0.0;
    if (M.has_rt && z + 1 < Nz) {
      const double Iu = x[idx + N] / lcf[z + 1];
      acc[14] += M.rt_l * rtw[i] * (Iu - II) * (Iu - II);
      const double ge = (z == 0) ? 2.0 * (II - Iu) : 2.0 * (2.0 * II - x[idx - N] / lcf[z - 1] - Iu);
      gr += M.rt_l * rtw[i] * ge / lcf[z];
    }
    if (M.has_ri) {
      acc[15] += M.ri_l * riw[i] * (II - iavg[i]) * (II - iavg[i]);
      gr += M.ri_l * riw[i] * 2.0 * (II - iavg[i]) / lcf[z];
    }
    const double gi_full = gv[idx] + gr;
    gv[idx] = gi_full;
    acc[12] += gi_full * d[idx];
    double gi = gi_full;
    if (M.nonneg && gi >= 0.0) gi = fmin(x[idx], gi);
    acc[13] = fmax(acc[13], fabs(gi));
  }
  for (int k = threadIdx.x; k < 16; k += blockDim.x) ops[k] = (k == 13) ? RED_MAX : RED_SUM;
  __syncthreads();
  block_reduce_arr(acc, ops, 16, red, scratch);
  if (!group_reduce(g, red, ops, 16)) return false;
  double r[16];
  for (int k = 0; k < 16; ++k) r[k] = red[k];
  __syncthreads();
  pf.mark(PR_F8);
  pf.count(PR_COUNT);
  const double chisq = r[0] + r[1] + r[2] + r[3];
  double regs = r[14] + r[15];
  for (int k = 0; k < 8; ++k) regs += r[4 + k];
  f = chisq + regs;
  gd = r[12];
  sbg = r[13];
  if (threadIdx.x == 0) {
    terms[0] = chisq;
    terms[1] = M.nfcv ? r[0] / M.wfcv / (2.0 * M.nfcv) : 0.0;
    terms[2] = M.namp ? r[1] / M.wamp / M.namp : 0.0;
    terms[3] = M.ncp ? r[2] / M.wcp / M.ncp : 0.0;
    terms[4] = M.nca ? r[3] / M.wca / M.nca : 0.0;
    terms[5] = regs;
    terms[6] = r[4];                        // l1
    terms[7] = r[4 + 7];                    // sm
    terms[8] = r[5];                        // tv
    terms[9] = r[6];                        // tsv
    terms[10] = r[7];                       // kl
    terms[11] = r[8];                       // gs
    terms[12] = M.has_lc ? 0.0 : r[4 + 5];  // tfd
    terms[13] = M.has_lc ? r[4 + 5] : 0.0;  // lc
    terms[14] = 0.0;                        // cen (not evaluated for movies)
    terms[15] = r[14];                      // rt
    terms[16] = r[15];                      // ri
    terms[17] = 0.0;                        // rs (not evaluated by the reference)
    terms[18] = 0.0;                        // rf (not evaluated by the reference)
    terms[19] = f;
  }
  __syncthreads();
  return true;
}

template <typename R>
__global__ void __launch_bounds__(Shape<R>::threads, Shape<R>::min_blocks) smili_batch_kernel(BatchArgs a) {
  extern __shared__ __align__(16) char dyn[];
  __shared__ LbState S;
  __shared__ double red[SMILI_REDK];
  __shared__ unsigned char ops[SMILI_REDK];
  __shared__ double scratch[Shape<R>::warps * SMILI_REDK];
  __shared__ int prob_s;
  const int grp = blockIdx.x / a.G, rank = blockIdx.x % a.G;
  Prof prof;
  prof.acc = (blockIdx.x == 0 && threadIdx.x == 0) ? a.prof : nullptr;
  prof.t = 0;
  prof.start();
  GroupCtx g;
  g.rank = rank;
  g.G = a.G;
  g.bar = a.bars + 2 * grp;
  g.red_part = a.red_part + (size_t)grp * a.G * SMILI_REDK;
  g.red_out = a.red_out + (size_t)grp * SMILI_REDK;
  g.abort_flag = a.abort_flag;
  g.spin_limit = SMILI_SPIN_LIMIT;
  if (a.mode == MODE_BARRIER) {  // cost of the group barrier: 1000 waits
    for (int i = 0; i < 1000; ++i)
      if (!group_sync(g)) return;
    return;
  }
  if (a.mode == MODE_WAIT_LIMIT) {
    // check of the bounded waits: rank 0 of every group never arrives at the
    // barrier, so the others' waits run out after a short limit, set the
    // abort flag and return; the host then reports SMILI_ERR_TIMEOUT
    g.spin_limit = SMILI_TEST_SPIN_LIMIT;
    if (rank != 0) group_sync(g);
    return;
  }
  while (true) {
    if (rank == 0 && threadIdx.x == 0) {
      const int p = atomicAdd(a.queue, 1);
      a.grp_prob[grp] = p;
      __threadfence();
    }
    if (!group_sync(g)) return;
    if (threadIdx.x == 0) prob_s = ((volatile int*)a.grp_prob)[grp];
    __syncthreads();
    const int p = prob_s;
    if (p >= a.nprob) return;
    const ProbDesc& P = a.descs[p];
    char* base = a.arena;
    FgCtx<R> fc;
    fc.P = &P;
    fc.base = base;
    fc.sbuf = reinterpret_cast<cpx<R>*>(dyn);
    fc.swork = fc.sbuf + SMILI_SMEM_CPX;
    fc.smem_cpx = SMILI_SMEM_CPX;
    fc.dyn_cpx = SMILI_DYN_CPX;
    LbCtxT<R> lc;
    lc.P = &P;
    lc.base = base;
    lc.g = &g;
    lc.S = &S;
    lc.n = P.npix;
    lc.m = P.m;
    const int chunk = ((P.npix + a.G - 1) / a.G + 31) / 32 * 32;
    lc.lo = min(P.npix, rank * chunk);
    lc.hi = min(P.npix, lc.lo + chunk);
    lc.x = at<double>(base, P.o_x);
    lc.gv = at<double>(base, P.o_g);
    lc.z = at<double>(base, P.o_z);
    lc.r = at<double>(base, P.o_r);
    lc.d = at<double>(base, P.o_d);
    lc.t = at<double>(base, P.o_t);
    lc.xp = at<double>(base, P.o_xp);
    lc.ws = at<R>(base, P.o_ws);  // S and Y in the kernel's precision
    lc.wy = at<R>(base, P.o_wy);
    lc.iwh = at<signed char>(base, P.o_iwh);
    lc.freef = at<unsigned char>(base, P.o_free);
    lc.bkey = at<unsigned long long>(base, P.o_bkey);
    lc.lred = at<double>(base, P.o_lred);
    lc.trace = at<double>(base, P.o_trace);
    lc.red = red;
    lc.ops = ops;
    lc.scratch = scratch;
    lc.dyn = dyn;
    lc.prof = &prof;
    const double* x0 = at<double>(base, P.o_x0);
    if (a.mode == MODE_SOLVE) {
      lb_init(lc, x0);
      if (rank == 0)
        for (int i = threadIdx.x; i < P.niter + 2; i += blockDim.x) lc.trace[i] = __longlong_as_double(0x7ff8000000000000LL);
    } else {
      // evaluation modes: x as given, no projection
      for (int i = lc.lo + threadIdx.x; i < lc.hi; i += blockDim.x) {
        lc.x[i] = x0[i];
        if (P.o_d) lc.d[i] = 0.0;
      }
      if (threadIdx.x == 0) {
        S.task = LB_TASK_FG_ONLY;
        S.done = 0;
        S.error = 0;
        S.iter = 0;
        S.nfg_total = 0;
      }
      __syncthreads();
    }
    bool ok = group_sync(g);
    prof.mark(PR_INIT);
    while (ok) {
      double f = 0, gd = 0, sbg = 0;
      const bool okf = P.nframes > 0 ? movie_fg<R>(fc, g, lc, red, ops, scratch, f, gd, sbg, S.terms)
                                     : group_fg<R>(fc, g, lc, red, ops, scratch, f, gd, sbg, S.terms, a.mode);
      if (!okf) {
        ok = false;
        break;
      }
      if (a.mode != MODE_SOLVE) {
        if (threadIdx.x == 0) S.nfg_total = 1;
        break;
      }
      const int rr = lb_after_fg(lc, f, gd, sbg);
      if (S.error) ok = false;
      if (rr != LB_RET_FG) break;
      if (!group_sync(g)) ok = false;
      prof.mark(PR_LB_POST);
    }
    if (ok && a.mode == MODE_SOLVE) {
      // final summary evaluation at the returned image (fftim2d.f90:356-376)
      if (!group_sync(g)) ok = false;
      double f = 0, gd = 0, sbg = 0;
      if (ok && !(P.nframes > 0 ? movie_fg<R>(fc, g, lc, red, ops, scratch, f, gd, sbg, S.terms)
                                : group_fg<R>(fc, g, lc, red, ops, scratch, f, gd, sbg, S.terms, MODE_FG)))
        ok = false;
      if (threadIdx.x == 0) S.nfg_total++;
    }
    __syncthreads();
    if (rank == 0 && threadIdx.x == 0) {
      ProbResult& res = a.results[p];
      for (int k = 0; k < SMILI_NTERMS3D; ++k) res.terms[k] = S.terms[k];
      res.task = ok ? S.task : LB_TASK_ERROR;
      res.iter = S.iter;
      res.nfg = S.nfg_total;
      res.error = ok ? S.error : 1;
    }
    if (!ok) return;
    if (!group_sync(g)) return;
  }
}

// ===========================================================================
// host side
// ===========================================================================
namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CUDA_TRY(expr)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(SMILI_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));   \
  } while (0)

int next235even(int n) {
  if (n <= 2) return 2;
  if (n % 2) n += 1;
  for (int m = n;; m += 2) {
    int k = m;
    for (int p : {2, 3, 5})
      while (k % p == 0) k /= p;
    if (k == 1) return m;
  }
}

void es_params(double eps, int& w, double& beta) {
  w = (int)std::ceil(std::log10(10.0 / eps));
  w = std::max(2, std::min(SMILI_MAXW, w));
  double c = 2.30;
  if (w == 2) c = 2.20;
  else if (w == 3) c = 2.26;
  else if (w == 4) c = 2.38;
  beta = c * w;
}

// Gauss-Legendre nodes on (0, 1] of a q-point rule on [-1, 1]
void gl_positive(int q, std::vector<double>& x, std::vector<double>& wt) {
  x.clear();
  wt.clear();
  for (int i = 0; i < q; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (q + 0.5));
    double dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= q; ++k) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = q * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= q; ++k) {
      const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = q * (z * p1 - p0) / (z * z - 1.0);
    if (z > 0) {
      x.push_back(z);
      wt.push_back(2.0 / ((1 - z * z) * dp * dp));
    }
  }
}

// 1 / psi_hat(k) for the N modes k = -N/2..(N-1)/2 on a fine grid of nf cells
std::vector<double> deconv_factors(int N, int nf, int w, double beta) {
  std::vector<double> gx, gw;
  gl_positive(80, gx, gw);
  std::vector<double> out(N);
  for (int i = 0; i < N; ++i) {
    const int k = i - N / 2;
    double acc = 0;
    for (size_t q = 0; q < gx.size(); ++q) {
      const double z = gx[q], s = 1.0 - z * z;
      const double phi = s > 0 ? std::exp(beta * (std::sqrt(s) - 1.0)) : 0.0;
      acc += gw[q] * phi * std::cos(M_PI * k * w * z / nf);
    }
    out[i] = 1.0 / (w * acc);
  }
  return out;
}

// Dynamic shared memory per CTA: the FFT/spread staging buffers, at least
// 48 KB, and never less than the Cauchy scan's layout.
template <typename R>
size_t dyn_smem_bytes() {
  size_t b = std::max((size_t)SMILI_DYN_CPX * sizeof(cpx<R>), (size_t)48 * 1024);
  b = std::max(b, (SMILI_CAUCHY_SMEM + 1023) / 1024 * 1024);
  return b;
}

struct Arena {
  size_t bytes = 0;
  int64_t take(size_t nbytes) {
    const int64_t off = (int64_t)bytes;
    bytes += (nbytes + 255) / 256 * 256;
    return off;
  }
};

bool finite_all(const double* p, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// Host image of one problem: descriptor + the byte blobs to upload
struct HostProb {
  ProbDesc d;
  std::vector<std::pair<int64_t, std::vector<char>>> blobs;
  // one copy of the bytes (no zero fill first)
  template <typename T>
  void put(int64_t off, const T* p, size_t n) {
    const char* c = reinterpret_cast<const char*>(p);
    blobs.emplace_back(off, std::vector<char>(c, c + n * sizeof(T)));
  }
  template <typename T>
  void put(int64_t off, const std::vector<T>& v) {
    put(off, v.data(), v.size());
  }
};

// PK_FRAME: one frame of a movie; PK_MODEL: one evaluation that also returns per-datum models
enum { PK_SOLVE = 0, PK_FG = 1, PK_T2 = 2, PK_T1 = 3, PK_FRAME = 4, PK_MODEL = 5 };

// The order of [0, n) by key(i) in [0, nkey), ties in index order: a
// counting sort, the same order as std::stable_sort by key in O(n + nkey).
template <class K>
std::vector<int> counting_order(int n, int nkey, K key) {
  std::vector<int> start((size_t)nkey + 1, 0), ord(n);
  for (int i = 0; i < n; ++i) ++start[key(i) + 1];
  for (int k = 0; k < nkey; ++k) start[k + 1] += start[k];
  for (int i = 0; i < n; ++i) ord[start[key(i)]++] = i;
  return ord;
}

// A regularizer whose per-pixel weights are one value (a flat prior) is
// evaluated with that value instead of a load per pixel (the array is still
// uploaded).
void set_uniform_weights(ProbDesc& d, const smili_imaging_args& a, int N) {
  const int has[5] = {d.has_l1, d.has_tv, d.has_tsv, d.has_kl, d.has_gs};
  const double* w[5] = {a.l1_wgt, a.tv_wgt, a.tsv_wgt, a.kl_wgt, a.gs_wgt};
  d.wuni = 0;
  for (int k = 0; k < 5; ++k) {
    d.wu[k] = 0.0;
    if (!has[k] || !w[k] || N < 1) continue;
    bool uni = true;
    for (int i = 1; uni && i < N; ++i) uni = w[k][i] == w[k][0];
    if (uni) {
      d.wuni |= 1 << k;
      d.wu[k] = w[k][0];
    }
  }
}

template <typename R>
int pack_problem(const smili_imaging_args& a, int kind, int niter, int nonneg, int m, double factr,
                 double pgtol, double eps, Arena& ar, HostProb& hp, const double* x_override,
                 const double* c_re, const double* c_im, double wtotal_override = 0.0, int bin = 8,
                 int transform = 0) {
  ProbDesc& d = hp.d;
  std::memset(&d, 0, sizeof(d));
  const int N = a.npix, nx = a.nx, ny = a.ny, nuv = a.nuv;
  const bool frame = kind == PK_FRAME;  // x / g / d live in the movie's vectors; data weights are global
  if (N < 1 || nx < 1 || ny < 1 || nuv < (frame ? 0 : 1) || (long)N > (long)nx * ny)
    return fail(SMILI_ERR_ARG, "invalid image or uv sizes");
  if (m < 1 || m > SMILI_MAXM_DEV) return fail(SMILI_ERR_UNSUPPORTED, "L-BFGS-B memory m must be 1..6");
  if (!a.iin || !a.xidx || !a.yidx || !a.u || !a.v) return fail(SMILI_ERR_ARG, "null array");
  std::vector<int> inv((size_t)nx * ny, -1);
  std::vector<int> xi(N), yi(N);
  for (int i = 0; i < N; ++i) {
    const int ix = a.xidx[i] - 1, iy = a.yidx[i] - 1;
    if (ix < 0 || ix >= nx || iy < 0 || iy >= ny) return fail(SMILI_ERR_ARG, "xidx/yidx out of range");
    if (inv[(size_t)iy * nx + ix] >= 0) return fail(SMILI_ERR_ARG, "duplicate pixel in xidx/yidx");
    inv[(size_t)iy * nx + ix] = i;
    xi[i] = ix;
    yi[i] = iy;
  }
  const double* x0 = x_override ? x_override : a.iin;
  if (!finite_all(x0, N) || !finite_all(a.u, nuv) || !finite_all(a.v, nuv))
    return fail(SMILI_ERR_DATA, "non-finite image or uv coordinates");
  // NUFFT parameters
  int w;
  double beta;
  es_params(eps, w, beta);
  d.w = w;
  d.beta = beta;
  d.nf1 = next235even(std::max(2 * nx, 2 * w));
  d.nf2 = next235even(std::max(2 * ny, 2 * w));
  if (d.nf1 > SMILI_SMEM_CPX || d.nf2 > SMILI_SMEM_CPX)
    return fail(SMILI_ERR_UNSUPPORTED, "fine grid larger than 2048 cells per axis");
  d.npix = N;
  d.nx = nx;
  d.ny = ny;
  d.nuv = nuv;
  d.m = m;
  d.niter = niter;
  d.nonneg = nonneg ? 1 : 0;
  d.factr = factr;
  d.pgtol = pgtol;
  d.ftarget = -INFINITY;
  d.prec64 = sizeof(R) == 8;
  d.nxref = a.nxref;
  d.nyref = a.nyref;
  d.windowed = N != nx * ny;
  d.ident = !d.windowed;
  for (int i = 0; d.ident && i < N; ++i) d.ident = xi[i] == i % nx && yi[i] == i / nx;
  // data terms
  const bool use_data = kind == PK_SOLVE || kind == PK_FG || kind == PK_MODEL || frame;
  const int nfcv = (use_data && a.isfcv) ? a.nfcv : 0;
  const int namp = (use_data && a.isamp) ? a.namp : 0;
  const int ncp = (use_data && a.iscp) ? a.ncp : 0;
  const int nca = (use_data && a.isca) ? a.nca : 0;
  if (use_data && nuv > 0 && nfcv + namp + ncp + nca == 0) return fail(SMILI_ERR_ARG, "no data terms");
  d.nfcv = nfcv;
  d.namp = namp;
  d.ncp = ncp;
  d.nca = nca;
  d.ndata = nfcv + namp + ncp + nca;
  const int nslot = (kind == PK_T1) ? nuv : nfcv + namp + 3 * ncp + 4 * nca;
  d.nslot = nslot;
  // normalised data weights (fftim2d.f90:178-213)
  double wtotal = 0;
  if (nfcv) wtotal += 2.0 * nfcv * a.wfcv;
  if (namp) wtotal += (double)namp * a.wamp;
  if (ncp) wtotal += (double)ncp * a.wcp;
  if (nca) wtotal += (double)nca * a.wca;
  if (wtotal_override > 0) wtotal = wtotal_override;  // a movie frame: the whole movie's data
  d.wfcv = nfcv ? a.wfcv / wtotal : 0;
  d.wamp = namp ? a.wamp / wtotal : 0;
  d.wcp = ncp ? a.wcp / wtotal : 0;
  d.wca = nca ? a.wca / wtotal : 0;
  // regularizers (active when lambda > 0, image.f90:112-175)
  const bool use_reg = kind == PK_SOLVE || kind == PK_FG || kind == PK_MODEL || frame;
  auto need_w = [&](double l, const double* wv, int nw, const char* nm) -> int {
    if (!(use_reg && l > 0)) return 0;
    if (!wv || nw != N) return fail(SMILI_ERR_ARG, std::string(nm) + " weights must have npix entries");
    if (!finite_all(wv, N)) return fail(SMILI_ERR_DATA, std::string(nm) + " weights not finite");
    return 1;
  };
  int rc;
  if ((rc = need_w(a.l1_l, a.l1_wgt, a.l1_nwgt, "l1")) < 0) return rc;
  d.has_l1 = rc;
  if ((rc = need_w(a.tv_l, a.tv_wgt, a.tv_nwgt, "tv")) < 0) return rc;
  d.has_tv = rc;
  if ((rc = need_w(a.tsv_l, a.tsv_wgt, a.tsv_nwgt, "tsv")) < 0) return rc;
  d.has_tsv = rc;
  if ((rc = need_w(a.kl_l, a.kl_wgt, a.kl_nwgt, "kl")) < 0) return rc;
  d.has_kl = rc;
  if ((rc = need_w(a.gs_l, a.gs_wgt, a.gs_nwgt, "gs")) < 0) return rc;
  d.has_gs = rc;
  d.has_tfd = use_reg && a.tfd_l > 0;
  d.has_cen = use_reg && a.cen_l > 0;
  d.has_sm = use_reg && a.sm_l > 0;
  d.l1_l = a.l1_l;
  d.tv_l = a.tv_l;
  d.tsv_l = a.tsv_l;
  d.kl_l = a.kl_l;
  d.gs_l = a.gs_l;
  d.tfd_l = a.tfd_l;
  d.tfd_tgtfd = a.tfd_tgtfd;
  d.cen_l = a.cen_l;
  d.cen_alpha = a.cen_alpha;
  d.sm_l = a.sm_l;
  d.sm_maj = a.sm_maj;
  d.sm_min = a.sm_min;
  d.sm_phi = a.sm_phi;
  if (frame && nuv == 0) {
    // a movie frame without data: pixel maps, regularizer weights and a
    // zero chi-square gradient (the arena is cleared at upload)
    d.o_xidx = ar.take(sizeof(int) * N);
    d.o_yidx = ar.take(sizeof(int) * N);
    d.o_inv = ar.take(sizeof(int) * (size_t)nx * ny);
    if (d.has_l1) d.o_l1w = ar.take(sizeof(double) * N);
    if (d.has_tv) d.o_tvw = ar.take(sizeof(double) * N);
    if (d.has_tsv) d.o_tsvw = ar.take(sizeof(double) * N);
    if (d.has_kl) d.o_klw = ar.take(sizeof(double) * N);
    if (d.has_gs) d.o_gsw = ar.take(sizeof(double) * N);
    d.o_gchi = ar.take(sizeof(double) * (size_t)nx * ny);
    hp.put(d.o_xidx, xi);
    hp.put(d.o_yidx, yi);
    hp.put(d.o_inv, inv);
    if (d.has_l1) hp.put(d.o_l1w, a.l1_wgt, (size_t)N);
    if (d.has_tv) hp.put(d.o_tvw, a.tv_wgt, (size_t)N);
    if (d.has_tsv) hp.put(d.o_tsvw, a.tsv_wgt, (size_t)N);
    if (d.has_kl) hp.put(d.o_klw, a.kl_wgt, (size_t)N);
    if (d.has_gs) hp.put(d.o_gsw, a.gs_wgt, (size_t)N);
    set_uniform_weights(d, a, N);
    return SMILI_OK;
  }

  // fine-grid coordinates in the kernel precision, band of touched cells
  std::vector<R> xu(nuv), xv(nuv);
  const R half = (R)0.5 * (R)w;
  long mn1 = 1L << 40, mx1 = -(1L << 40), mn2 = 1L << 40, mx2 = -(1L << 40);
  for (int j = 0; j < nuv; ++j) {
    xu[j] = (R)(a.u[j] * d.nf1 / (2.0 * M_PI));
    xv[j] = (R)(a.v[j] * d.nf2 / (2.0 * M_PI));
    const long l1 = (long)std::ceil(xu[j] - half), l2 = (long)std::ceil(xv[j] - half);
    mn1 = std::min(mn1, l1);
    mx1 = std::max(mx1, l1 + w - 1);
    mn2 = std::min(mn2, l2);
    mx2 = std::max(mx2, l2 + w - 1);
  }
  if (mx1 - mn1 + 1 >= d.nf1) {
    d.b1s = 0;
    d.b1n = d.nf1;
  } else {
    d.b1s = (int)mn1;
    d.b1n = (int)(mx1 - mn1 + 1);
  }
  if (mx2 - mn2 + 1 >= d.nf2) {
    d.b2s = 0;
    d.b2n = d.nf2;
  } else {
    d.b2s = (int)mn2;
    d.b2n = (int)(mx2 - mn2 + 1);
  }
  // spreading tile: 16 x 16 when its warp subgrids (one (16 + w - 1)^2
  // complex subgrid per warp) and the smallest weight table fit the dynamic
  // shared memory of the launch, else 8 x 8
  {
    const size_t dyn = (size_t)SMILI_DYN_CPX * sizeof(cpx<R>);
    const size_t sg = 16 + w - 1, nw = Shape<R>::warps;
    if (bin == 16 && nw * sg * sg * sizeof(cpx<R>) + nw * 8 * 2 * w * sizeof(R) + 16 > dyn) bin = 8;
    if (bin != 16) bin = 8;
  }
  d.bin = bin;
  // band passes: dense products with the twiddle matrices when the band is
  // narrow (at most 64 x 64 cells, 2048 in all) and their multiply-adds
  // (2 nx ny b1n + 4 b1n ny b2n per direction, real and complex halves) come
  // to less than twice the radix passes' flops; they run as register-tiled
  // loops, the FFTs as latency-bound shared-memory sweeps
  {
    const bool fits = d.b1n <= 64 && d.b2n <= 64 && d.b1n * d.b2n <= 2048;
    const double lg1 = std::log2((double)d.nf1), lg2 = std::log2((double)d.nf2);
    const double dft_fl = 2.0 * nx * ny * (d.b1n + d.b2n) + 8.0 * d.b1n * d.b2n * (nx + ny);
    const double fft_fl = 5.0 * ((double)(ny + d.b2n) * d.nf1 * lg1 + (double)(d.b1n + nx) * d.nf2 * lg2);
    d.dft = fits && (transform == 2 || (transform == 0 && dft_fl < 2.0 * fft_fl));
  }
  // sort the uv points by bin x bin tiles of the band (spreading subproblems
  // and locality); remap indices.  Band-relative cells are computed exactly as the
  // kernels do: imod(ceil(xi - w/2) - start, nf).
  auto imodh = [](long a, long n) {
    long r = a % n;
    return r < 0 ? r + n : r;
  };
  std::vector<long> bkey(nuv);
  std::vector<int> bidx(nuv);
  const int nb1 = (d.nf1 + bin - 1) / bin, nb2 = (d.nf2 + bin - 1) / bin;
  for (int j = 0; j < nuv; ++j) {
    const long c1 = imodh((long)std::ceil(xu[j] - half) - d.b1s, d.nf1);
    const long c2 = imodh((long)std::ceil(xv[j] - half) - d.b2s, d.nf2);
    bkey[j] = ((c2 / bin) << 32) + (c1 / bin);
    bidx[j] = (int)(c2 / bin) * nb1 + (int)(c1 / bin);  // the same order as bkey
  }
  const std::vector<int> perm = counting_order(nuv, nb1 * nb2, [&](int j) { return bidx[j]; });
  // spreading work items: <= 128 consecutive points of one bin
  std::vector<int> items;
  for (int j = 0; j < nuv;) {
    const long k = bkey[perm[j]];
    int e = j;
    while (e < nuv && bkey[perm[e]] == k && e - j < 128) ++e;
    items.push_back(j);
    items.push_back(e);
    items.push_back((int)((k >> 32) * bin));
    items.push_back((int)((k & 0xffffffffL) * bin));
    j = e;
  }
  d.nitems = (int)items.size() / 4;
  std::vector<int> newpos(nuv);
  for (int j = 0; j < nuv; ++j) newpos[perm[j]] = j;
  std::vector<R> su(nuv), sv(nuv);
  for (int j = 0; j < nuv; ++j) {
    su[j] = xu[perm[j]];
    sv[j] = xv[perm[j]];
  }
  // data: values, variances, slots
  std::vector<R> dre(std::max(d.ndata, 1)), dim(std::max(d.ndata, 1)), dvar(std::max(d.ndata, 1));
  std::vector<int> didx(std::max(nslot, 1));
  std::vector<signed char> dsgn(std::max(nslot, 1));
  auto slot = [&](int s, int uvidx) -> int {
    if (uvidx == 0 || std::abs(uvidx) > nuv) return fail(SMILI_ERR_ARG, "uv index out of range");
    didx[s] = newpos[std::abs(uvidx) - 1];
    dsgn[s] = uvidx > 0 ? 1 : -1;
    return 0;
  };
  auto check_var = [&](double v) { return std::isfinite(v) && v > 0.0; };
  int e = 0, s = 0;
  if (nfcv) {
    if (!a.uvidxfcv || !a.vfcvr || !a.vfcvi || !a.varfcv) return fail(SMILI_ERR_ARG, "null fcv array");
    const double dix = a.nxref - nx / 2.0 - 1, diy = a.nyref - ny / 2.0 - 1;
    for (int i = 0; i < nfcv; ++i, ++e, ++s) {
      if ((rc = slot(s, a.uvidxfcv[i])) < 0) return rc;
      const int k = std::abs(a.uvidxfcv[i]) - 1, sg = a.uvidxfcv[i] > 0 ? 1 : -1;
      if (!std::isfinite(a.vfcvr[i]) || !std::isfinite(a.vfcvi[i]) || !check_var(a.varfcv[i]))
        return fail(SMILI_ERR_DATA, "invalid complex visibility or variance");
      // phashift_r2c (fftlib.f90:223-244)
      const std::complex<double> z = std::complex<double>(a.vfcvr[i], a.vfcvi[i]) *
                                     std::exp(std::complex<double>(0.0, a.u[k] * sg * dix + a.v[k] * sg * diy));
      dre[e] = (R)z.real();
      dim[e] = (R)z.imag();
      dvar[e] = (R)a.varfcv[i];
    }
  }
  if (namp) {
    if (!a.uvidxamp || !a.vamp || !a.varamp) return fail(SMILI_ERR_ARG, "null amp array");
    for (int i = 0; i < namp; ++i, ++e, ++s) {
      if ((rc = slot(s, a.uvidxamp[i])) < 0) return rc;
      if (!std::isfinite(a.vamp[i]) || !check_var(a.varamp[i]))
        return fail(SMILI_ERR_DATA, "invalid amplitude or variance");
      dre[e] = (R)a.vamp[i];
      dim[e] = 0;
      dvar[e] = (R)a.varamp[i];
    }
  }
  if (ncp) {
    if (!a.uvidxcp || !a.cp || !a.varcp) return fail(SMILI_ERR_ARG, "null cp array");
    for (int i = 0; i < ncp; ++i, ++e) {
      for (int q = 0; q < 3; ++q, ++s)
        if ((rc = slot(s, a.uvidxcp[3 * i + q])) < 0) return rc;
      if (!std::isfinite(a.cp[i]) || !check_var(a.varcp[i]))
        return fail(SMILI_ERR_DATA, "invalid closure phase or variance");
      dre[e] = (R)a.cp[i];
      dim[e] = 0;
      dvar[e] = (R)a.varcp[i];
    }
  }
  if (nca) {
    if (!a.uvidxca || !a.ca || !a.varca) return fail(SMILI_ERR_ARG, "null ca array");
    for (int i = 0; i < nca; ++i, ++e) {
      for (int q = 0; q < 4; ++q, ++s)
        if ((rc = slot(s, a.uvidxca[4 * i + q])) < 0) return rc;
      if (!std::isfinite(a.ca[i]) || !check_var(a.varca[i]))
        return fail(SMILI_ERR_DATA, "invalid closure amplitude or variance");
      dre[e] = (R)a.ca[i];
      dim[e] = 0;
      dvar[e] = (R)a.varca[i];
    }
  }
  // Order the data of each type by the sorted position of their first uv
  // point (stable): neighbouring threads of the chi-square stage then gather
  // neighbouring model visibilities and add into neighbouring accumulators,
  // so an amplitude or visibility warp touches a few sectors instead of 32.
  // The sums only change order.  Per-datum models (PK_MODEL) keep the
  // callers' order.
  if (kind != PK_MODEL && d.ndata > 1) {
    auto reorder = [&](int e0, int ne, int s0, int nref) {
      if (ne < 2) return;
      const std::vector<int> ord = counting_order(ne, nuv, [&](int p) { return didx[s0 + nref * p]; });
      std::vector<R> r0(ne), r1(ne), r2(ne);
      std::vector<int> ix((size_t)ne * nref);
      std::vector<signed char> sg((size_t)ne * nref);
      for (int i = 0; i < ne; ++i) {
        const int o = ord[i];
        r0[i] = dre[e0 + o];
        r1[i] = dim[e0 + o];
        r2[i] = dvar[e0 + o];
        for (int q = 0; q < nref; ++q) {
          ix[(size_t)nref * i + q] = didx[s0 + nref * o + q];
          sg[(size_t)nref * i + q] = dsgn[s0 + nref * o + q];
        }
      }
      std::copy(r0.begin(), r0.end(), dre.begin() + e0);
      std::copy(r1.begin(), r1.end(), dim.begin() + e0);
      std::copy(r2.begin(), r2.end(), dvar.begin() + e0);
      std::copy(ix.begin(), ix.end(), didx.begin() + s0);
      std::copy(sg.begin(), sg.end(), dsgn.begin() + s0);
    };
    reorder(0, nfcv, 0, 1);
    reorder(nfcv, namp, nfcv, 1);
    reorder(nfcv + namp, ncp, nfcv + namp, 3);
    reorder(nfcv + namp + ncp, nca, nfcv + namp + 3 * ncp, 4);
  }
  // per-uv-point derivative accumulators: set here only for the bare type-1
  // mode (c = (Re c, -Im c) in sorted order); otherwise F3 zeroes them and F4
  // adds into them every evaluation
  std::vector<cpx<R>> contrib0;
  if (kind == PK_T1) {
    contrib0.resize(nuv);
    for (int j = 0; j < nuv; ++j) {
      const int o = perm[j];
      contrib0[j].x = (R)c_re[o];
      contrib0[j].y = (R)(-c_im[o]);
    }
  }
  // deconvolution factors and twiddles
  const std::vector<double> dc1 = deconv_factors(nx, d.nf1, w, beta), dc2 = deconv_factors(ny, d.nf2, w, beta);
  auto twiddles = [](int n) {
    std::vector<cpx<R>> t(n);
    for (int k = 0; k < n; ++k) {
      const long double ang = 2.0L * 3.14159265358979323846264338327950288L * k / n;
      t[k].x = (R)std::cos(ang);
      t[k].y = (R)std::sin(ang);
    }
    return t;
  };
  // ---- arena layout ----
  const size_t C = sizeof(cpx<R>);
  if (!frame) d.o_x0 = ar.take(sizeof(double) * N);
  d.o_xidx = ar.take(sizeof(int) * N);
  d.o_yidx = ar.take(sizeof(int) * N);
  d.o_inv = ar.take(sizeof(int) * (size_t)nx * ny);
  if (d.has_l1) d.o_l1w = ar.take(sizeof(double) * N);
  if (d.has_tv) d.o_tvw = ar.take(sizeof(double) * N);
  if (d.has_tsv) d.o_tsvw = ar.take(sizeof(double) * N);
  if (d.has_kl) d.o_klw = ar.take(sizeof(double) * N);
  if (d.has_gs) d.o_gsw = ar.take(sizeof(double) * N);
  d.o_dc1 = ar.take(sizeof(double) * nx);
  d.o_dc2 = ar.take(sizeof(double) * ny);
  d.o_tw1 = ar.take(C * d.nf1);
  d.o_tw2 = ar.take(C * d.nf2);
  if (d.dft) {
    d.o_ex = ar.take(C * (size_t)d.b1n * nx);
    d.o_ey = ar.take(C * (size_t)d.b2n * ny);
  }
  d.o_u = ar.take(sizeof(R) * nuv);
  d.o_v = ar.take(sizeof(R) * nuv);
  d.o_dre = ar.take(sizeof(R) * dre.size());
  d.o_dim = ar.take(sizeof(R) * dim.size());
  d.o_dvar = ar.take(sizeof(R) * dvar.size());
  d.o_didx = ar.take(sizeof(int) * didx.size());
  d.o_dsgn = ar.take(dsgn.size());
  d.o_items = ar.take(sizeof(int) * items.size());
  d.o_tmpA = ar.take(C * (size_t)ny * d.b1n);
  d.o_bandA = ar.take(C * (size_t)d.b2n * d.b1n);
  d.o_V = ar.take(C * nuv);
  d.o_contrib = ar.take(C * std::max(nuv, 1));
  d.o_bandC = ar.take(C * (size_t)d.b2n * d.b1n);
  d.o_tmpC = ar.take(C * (size_t)d.b2n * nx);
  d.o_gchi = ar.take(sizeof(double) * (size_t)nx * ny);
  d.o_xg = ar.take(sizeof(double) * (size_t)nx * ny);
  if (!frame) {
    d.o_x = ar.take(sizeof(double) * N);
    d.o_g = ar.take(sizeof(double) * N);
  }
  if (kind == PK_MODEL) d.o_model = ar.take(sizeof(double) * 4 * std::max(d.ndata, 1));
  if (kind == PK_SOLVE || kind == PK_FG || kind == PK_MODEL) {
    d.o_z = ar.take(sizeof(double) * N);
    d.o_r = ar.take(sizeof(double) * N);
    d.o_d = ar.take(sizeof(double) * N);
    d.o_t = ar.take(sizeof(double) * N);
    d.o_xp = ar.take(sizeof(double) * N);
    d.o_iwh = ar.take(N);
    d.o_free = ar.take(N);
    d.o_bkey = ar.take(sizeof(unsigned long long) * N);
    d.o_sbk = ar.take(sizeof(unsigned long long) * N);
    d.o_sbi = ar.take(sizeof(int) * N);
    d.o_hist = ar.take(sizeof(int) * 2 * 4096);
    d.o_lred = ar.take(sizeof(double) * 64);
    d.o_trace = ar.take(sizeof(double) * (niter + 2));
  }
  if (kind == PK_SOLVE) {  // S and Y: R per element (FP32 storage in the FP32 mode)
    d.o_ws = ar.take(sizeof(R) * (size_t)N * m);
    d.o_wy = ar.take(sizeof(R) * (size_t)N * m);
  }
  // ---- blobs ----
  if (!frame) hp.put(d.o_x0, x0, (size_t)N);
  hp.put(d.o_xidx, xi);
  hp.put(d.o_yidx, yi);
  hp.put(d.o_inv, inv);
  if (d.has_l1) hp.put(d.o_l1w, a.l1_wgt, (size_t)N);
  if (d.has_tv) hp.put(d.o_tvw, a.tv_wgt, (size_t)N);
  if (d.has_tsv) hp.put(d.o_tsvw, a.tsv_wgt, (size_t)N);
  if (d.has_kl) hp.put(d.o_klw, a.kl_wgt, (size_t)N);
  if (d.has_gs) hp.put(d.o_gsw, a.gs_wgt, (size_t)N);
  set_uniform_weights(d, a, N);
  hp.put(d.o_dc1, dc1);
  hp.put(d.o_dc2, dc2);
  hp.put(d.o_tw1, twiddles(d.nf1));
  hp.put(d.o_tw2, twiddles(d.nf2));
  if (d.dft) {
    // E[b][i] = tw[((i - n_img / 2) (bs + b)) mod nf]: the twiddle each FFT
    // pass applies between image index i and band index b
    auto emat = [&](int nb, int bs, int nimg, int nf) {
      const std::vector<cpx<R>> tw = twiddles(nf);
      std::vector<cpx<R>> e((size_t)nb * nimg);
      for (int b = 0; b < nb; ++b)
        for (int i = 0; i < nimg; ++i) {
          long k = ((long)(i - nimg / 2) * (long)(bs + b)) % nf;
          if (k < 0) k += nf;
          e[(size_t)b * nimg + i] = tw[k];
        }
      return e;
    };
    hp.put(d.o_ex, emat(d.b1n, d.b1s, nx, d.nf1));
    hp.put(d.o_ey, emat(d.b2n, d.b2s, ny, d.nf2));
  }
  hp.put(d.o_u, su);
  hp.put(d.o_v, sv);
  hp.put(d.o_dre, dre);
  hp.put(d.o_dim, dim);
  hp.put(d.o_dvar, dvar);
  hp.put(d.o_didx, didx);
  hp.put(d.o_dsgn, dsgn);
  hp.put(d.o_items, items);
  if (kind == PK_T1) hp.put(d.o_contrib, contrib0);
  // the original -> sorted uv permutation is needed to return visibilities
  if (!frame)
    hp.blobs.emplace_back(-1, std::vector<char>((const char*)perm.data(), (const char*)perm.data() + sizeof(int) * nuv));
  return SMILI_OK;
}

}  // namespace

struct smili_batch {
  int nprob = 0, prec64 = 1, G = 1, ngroups = 1, device = 0;
  int kind = PK_SOLVE;
  std::vector<ProbDesc> descs;
  std::vector<std::vector<int>> perms;
  char* d_arena = nullptr;
  size_t arena_bytes = 0;
  ProbDesc* d_descs = nullptr;
  char* d_aux = nullptr;  // queue, bars, reductions, results
  ProbResult* d_results = nullptr;
  int* d_queue = nullptr;
  unsigned* d_bars = nullptr;
  double* d_red_part = nullptr;
  double* d_red_out = nullptr;
  int* d_grp_prob = nullptr;
  int* d_abort = nullptr;
  unsigned long long* d_prof = nullptr;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  size_t dyn_bytes = 0;
  int profile = 0;
  std::vector<int> niter_cap;  // iteration caps at packing (trace buffers are sized for them)
  // start images as packed, saved before the first replacement (reset_starts)
  double* d_x0_saved = nullptr;
  std::vector<size_t> x0_saved_off;
  unsigned char* d_keep = nullptr;  // keep flags of set_starts_from_images
};

namespace {

template <typename R>
int launch_batch(smili_batch* b, int mode, float* ms) {
  const void* fn = (const void*)smili_batch_kernel<R>;
  const size_t aux_reset = 0;
  (void)aux_reset;
  CUDA_TRY(cudaMemsetAsync(b->d_queue, 0, sizeof(int), b->stream));
  CUDA_TRY(cudaMemsetAsync(b->d_bars, 0, sizeof(unsigned) * 2 * b->ngroups, b->stream));
  CUDA_TRY(cudaMemsetAsync(b->d_abort, 0, sizeof(int), b->stream));
  BatchArgs a;
  a.arena = b->d_arena;
  a.descs = b->d_descs;
  a.nprob = b->nprob;
  a.G = b->G;
  a.mode = mode;
  a.queue = b->d_queue;
  a.bars = b->d_bars;
  a.red_part = b->d_red_part;
  a.red_out = b->d_red_out;
  a.grp_prob = b->d_grp_prob;
  a.abort_flag = b->d_abort;
  a.results = b->d_results;
  a.prof = b->profile ? b->d_prof : nullptr;
  if (b->profile) CUDA_TRY(cudaMemsetAsync(b->d_prof, 0, sizeof(unsigned long long) * PR_NSTAGE, b->stream));
  void* args[] = {&a};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms) {
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, b->stream));
  }
  CUDA_TRY(cudaLaunchCooperativeKernel(fn, dim3(b->G * b->ngroups), dim3(Shape<R>::threads), args,
                                       b->dyn_bytes, b->stream));
  if (ms) {
    CUDA_TRY(cudaEventRecord(e1, b->stream));
    CUDA_TRY(cudaEventSynchronize(e1));
    CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  int abort_flag = 0;
  CUDA_TRY(cudaMemcpy(&abort_flag, b->d_abort, sizeof(int), cudaMemcpyDeviceToHost));
  if (abort_flag) return fail(SMILI_ERR_TIMEOUT, "a device-side group barrier timed out; solve aborted");
  return SMILI_OK;
}

template <typename R>
int finish_batch(smili_batch* b, std::vector<HostProb>& hps, int maxn, const smili_options* opt,
                 smili_batch** out);

template <typename R>
int create_batch(int nprob, const smili_imaging_args* const* probs, const int* niter, int nonneg,
                 int m, double factr, double pgtol, const smili_options* opt, int kind,
                 const double* const* x_over, const double* c_re, const double* c_im,
                 smili_batch** out) {
  const double eps = (opt && opt->nufft_eps > 0) ? opt->nufft_eps : 1e-6;
  const int device = opt ? opt->device : 0;
  if (!(eps < 1.0)) return fail(SMILI_ERR_ARG, "nufft_eps must be in (0, 1)");
  smili_batch* b = new smili_batch();
  b->nprob = nprob;
  b->prec64 = sizeof(R) == 8;
  b->device = device;
  b->kind = kind;
  // The problems are packed in parallel on the host cores, each into its own
  // arena region (starting with a 256-byte reserve, so no present field sits
  // at offset 0, the mark of an absent one); the regions are then laid end
  // to end and every offset moved by its region's start.
  std::vector<Arena> ars(nprob);
  std::vector<HostProb> hps(nprob);
  std::vector<int> rcs(nprob, SMILI_OK);
  std::vector<std::string> errs(nprob);
  std::atomic<int> next{0};
  auto work = [&]() {
    for (int p = next.fetch_add(1); p < nprob; p = next.fetch_add(1)) {
      try {  // an exception must not leave a worker thread (std::terminate)
        ars[p].take(256);
        rcs[p] = pack_problem<R>(*probs[p], kind, niter ? niter[p] : 0, nonneg, m, factr, pgtol, eps, ars[p],
                                 hps[p], x_over ? x_over[p] : nullptr, c_re, c_im, 0.0,
                                 opt && opt->spread_bin ? opt->spread_bin : 8, opt ? opt->transform : 0);
        if (rcs[p] != SMILI_OK) errs[p] = g_err;
      } catch (const std::exception& ex) {
        rcs[p] = SMILI_ERR_ARG;
        errs[p] = std::string("host packing of a problem failed: ") + ex.what();
      }
    }
  };
  const int nth = std::max(1, std::min(nprob, (int)std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (int t = 1; t < nth; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  for (int p = 0; p < nprob; ++p)
    if (rcs[p] != SMILI_OK) {
      delete b;
      return fail(rcs[p], errs[p]);
    }
  int maxn = 1;
  size_t base = 0;
  for (int p = 0; p < nprob; ++p) {
    ProbDesc& d = hps[p].d;
#define SMILI_MOVE(f) \
  if (d.f) d.f += (int64_t)base;
    SMILI_PROB_OFFSETS(SMILI_MOVE)
#undef SMILI_MOVE
    for (auto& bl : hps[p].blobs)
      if (bl.first >= 0) bl.first += (int64_t)base;
    base += ars[p].bytes;
    b->descs.push_back(d);
    maxn = std::max(maxn, d.npix);
  }
  b->arena_bytes = base;
  return finish_batch<R>(b, hps, maxn, opt, out);
}

// Device side of a batch whose problems are packed (descs, arena size, host
// blobs): launch geometry, buffers, upload.  Takes ownership of b.
template <typename R>
int finish_batch(smili_batch* b, std::vector<HostProb>& hps, int maxn, const smili_options* opt,
                 smili_batch** out) {
  const int device = b->device;
  const int nprob = b->nprob;
  b->niter_cap.clear();
  for (const ProbDesc& d : b->descs) b->niter_cap.push_back(d.niter);
  // inputs are valid: now the device
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) {
    delete b;
    return fail(SMILI_ERR_NODEV, "no CUDA device");
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    delete b;
    return fail(SMILI_ERR_NODEV, "cannot select the CUDA device");
  }
  // launch geometry: co-resident CTAs split into groups
  // FFT/spread staging (SMILI_DYN_CPX complex values) and the Cauchy scan's
  // batch buffers share the dynamic region: 96 KB in FP64 (two 256-thread
  // CTAs per SM), 54 KB in FP32 (two 512-thread CTAs per SM)
  b->dyn_bytes = dyn_smem_bytes<R>();
  const void* fn = (const void*)smili_batch_kernel<R>;
  auto cleanup = [&](int rc) {
    smili_batch_destroy(b);
    return rc;
  };
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->dyn_bytes) != cudaSuccess)
    return cleanup(fail(SMILI_ERR_CUDA, "cannot set dynamic shared memory size"));
  int occ = 0, nsm = 0, coop = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, Shape<R>::threads, b->dyn_bytes));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  if (!coop || occ < 1) return cleanup(fail(SMILI_ERR_CUDA, "cooperative launch unavailable"));
  const int maxres = occ * nsm;
  int G = opt && opt->ctas_per_problem > 0 ? opt->ctas_per_problem : 0;
  if (G <= 0) {
    const int per_cta = 4 * Shape<R>::threads;  // about four pixels per thread
    G = std::max(1, std::min(maxres, (maxn + per_cta - 1) / per_cta));
    if (nprob > 1) G = std::max(1, std::min(G, maxres / nprob));
  }
  G = std::min(G, maxres);
  b->G = G;
  b->ngroups = std::max(1, std::min(nprob, maxres / G));
  // device buffers
  if (cudaMalloc(&b->d_arena, std::max<size_t>(b->arena_bytes, 256)) != cudaSuccess)
    return cleanup(fail(SMILI_ERR_CUDA, "cudaMalloc of the problem arena failed"));
  size_t aux = 0;
  auto take = [&](size_t n) {
    const size_t o = aux;
    aux += (n + 255) / 256 * 256;
    return o;
  };
  const size_t o_desc = take(sizeof(ProbDesc) * nprob), o_res = take(sizeof(ProbResult) * nprob),
               o_q = take(sizeof(int)), o_bar = take(sizeof(unsigned) * 2 * b->ngroups),
               o_rp = take(sizeof(double) * (size_t)b->ngroups * G * SMILI_REDK),
               o_ro = take(sizeof(double) * (size_t)b->ngroups * SMILI_REDK),
               o_gp = take(sizeof(int) * b->ngroups), o_ab = take(sizeof(int)),
               o_pf = take(sizeof(unsigned long long) * PR_NSTAGE);
  if (cudaMalloc(&b->d_aux, aux) != cudaSuccess) return cleanup(fail(SMILI_ERR_CUDA, "cudaMalloc aux failed"));
  b->d_descs = reinterpret_cast<ProbDesc*>(b->d_aux + o_desc);
  b->d_results = reinterpret_cast<ProbResult*>(b->d_aux + o_res);
  b->d_queue = reinterpret_cast<int*>(b->d_aux + o_q);
  b->d_bars = reinterpret_cast<unsigned*>(b->d_aux + o_bar);
  b->d_red_part = reinterpret_cast<double*>(b->d_aux + o_rp);
  b->d_red_out = reinterpret_cast<double*>(b->d_aux + o_ro);
  b->d_grp_prob = reinterpret_cast<int*>(b->d_aux + o_gp);
  b->d_abort = reinterpret_cast<int*>(b->d_aux + o_ab);
  b->d_prof = reinterpret_cast<unsigned long long*>(b->d_aux + o_pf);
  if (opt && opt->stream) {
    b->stream = (cudaStream_t)opt->stream;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    b->own_stream = true;
  }
  // upload: zero the arena, then every blob
  CUDA_TRY(cudaMemsetAsync(b->d_arena, 0, b->arena_bytes, b->stream));
  for (int p = 0; p < nprob; ++p) {
    for (auto& bl : hps[p].blobs) {
      if (bl.first < 0) {
        b->perms.emplace_back((const int*)bl.second.data(), (const int*)(bl.second.data() + bl.second.size()));
        continue;
      }
      if (!bl.second.empty())
        CUDA_TRY(cudaMemcpyAsync(b->d_arena + bl.first, bl.second.data(), bl.second.size(),
                                 cudaMemcpyHostToDevice, b->stream));
    }
  }
  CUDA_TRY(cudaMemcpyAsync(b->d_descs, b->descs.data(), sizeof(ProbDesc) * nprob, cudaMemcpyHostToDevice,
                           b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  *out = b;
  return SMILI_OK;
}

// Pack one movie (fftim3d): the movie's descriptor carries the optimiser
// vectors over npix * nz values and the Rt / Ri / light-curve arrays; every
// frame is packed as a 2D problem (PK_FRAME) over its own slice of the uv
// list and its own data, with the whole movie's data weights, the static
// regularizers divided by nz (image3d.f90:219-257; per-frame weights scaled
// by the light curve when lc_nidx is 1 or 3, image3d.f90:188-200) and the
// centroid term off (image3d.f90:210); its x / g / d point into the
// movie's vectors.
template <typename R>
int pack_movie(const smili_imaging3d_args& a, int kind, int niter, int nonneg, int m, double factr,
               double pgtol, double eps, Arena& ar, HostProb& hp, const double* x_override, int spread_bin,
               int transform) {
  const int N = a.npix, Nz = a.nz, nuv = a.nuv;
  if (N < 1 || Nz < 1 || nuv < 0 || a.nx < 1 || a.ny < 1 || (long)N * Nz > 0x7fffffffL)
    return fail(SMILI_ERR_ARG, "invalid movie sizes");
  if (!a.iin || !a.xidx || !a.yidx || !a.nuvs || !a.lc_l || !a.lc_tgtfd || (nuv > 0 && (!a.u || !a.v)))
    return fail(SMILI_ERR_ARG, "null movie array");
  std::vector<int> off(Nz + 1, 0);
  for (int z = 0; z < Nz; ++z) {
    if (a.nuvs[z] < 0) return fail(SMILI_ERR_ARG, "negative nuvs");
    off[z + 1] = off[z] + a.nuvs[z];
  }
  if (off[Nz] != nuv) return fail(SMILI_ERR_ARG, "nuvs does not add up to nuv");
  for (int z = 0; z < Nz; ++z)
    if (!(a.lc_tgtfd[z] != 0.0) || !std::isfinite(a.lc_tgtfd[z]))
      return fail(SMILI_ERR_DATA, "lc_tgtfd must be finite and nonzero");
  const int nfcv = a.isfcv ? a.nfcv : 0, namp = a.isamp ? a.namp : 0, ncp = a.iscp ? a.ncp : 0,
            nca = a.isca ? a.nca : 0;
  double wtotal = 0;
  if (nfcv) wtotal += 2.0 * nfcv * a.wfcv;
  if (namp) wtotal += (double)namp * a.wamp;
  if (ncp) wtotal += (double)ncp * a.wcp;
  if (nca) wtotal += (double)nca * a.wca;
  if (!(wtotal > 0)) return fail(SMILI_ERR_ARG, "no data terms");
  auto frame_of = [&](int idx, int& z, int& local) -> int {
    const int k = std::abs(idx) - 1;
    if (idx == 0 || k >= nuv) return fail(SMILI_ERR_ARG, "uv index out of range");
    z = (int)(std::upper_bound(off.begin(), off.end(), k) - off.begin()) - 1;
    local = (idx > 0 ? 1 : -1) * (k - off[z] + 1);
    return SMILI_OK;
  };
  // split the data by frame (frame-local signed uv indices)
  struct FrameData {
    std::vector<int> ifcv, iamp, icp, ica;
    std::vector<double> fr, fi, fv, av, avar, cpv, cpvar, cav, cavar;
  };
  std::vector<FrameData> fd(Nz);
  int rc;
  for (int i = 0; i < nfcv; ++i) {
    int z, l;
    if ((rc = frame_of(a.uvidxfcv[i], z, l)) < 0) return rc;
    fd[z].ifcv.push_back(l);
    fd[z].fr.push_back(a.vfcvr[i]);
    fd[z].fi.push_back(a.vfcvi[i]);
    fd[z].fv.push_back(a.varfcv[i]);
  }
  for (int i = 0; i < namp; ++i) {
    int z, l;
    if ((rc = frame_of(a.uvidxamp[i], z, l)) < 0) return rc;
    fd[z].iamp.push_back(l);
    fd[z].av.push_back(a.vamp[i]);
    fd[z].avar.push_back(a.varamp[i]);
  }
  for (int i = 0; i < ncp; ++i) {
    int z0 = -1, ls[3];
    for (int q = 0; q < 3; ++q) {
      int z;
      if ((rc = frame_of(a.uvidxcp[3 * i + q], z, ls[q])) < 0) return rc;
      if (q && z != z0) return fail(SMILI_ERR_UNSUPPORTED, "a closure phase spans two frames");
      z0 = z;
    }
    for (int q = 0; q < 3; ++q) fd[z0].icp.push_back(ls[q]);
    fd[z0].cpv.push_back(a.cp[i]);
    fd[z0].cpvar.push_back(a.varcp[i]);
  }
  for (int i = 0; i < nca; ++i) {
    int z0 = -1, ls[4];
    for (int q = 0; q < 4; ++q) {
      int z;
      if ((rc = frame_of(a.uvidxca[4 * i + q], z, ls[q])) < 0) return rc;
      if (q && z != z0) return fail(SMILI_ERR_UNSUPPORTED, "a closure amplitude spans two frames");
      z0 = z;
    }
    for (int q = 0; q < 4; ++q) fd[z0].ica.push_back(ls[q]);
    fd[z0].cav.push_back(a.ca[i]);
    fd[z0].cavar.push_back(a.varca[i]);
  }
  for (int z = 0; z < Nz; ++z)
    if (a.nuvs[z] > 0 && fd[z].ifcv.empty() && fd[z].iamp.empty() && fd[z].icp.empty() && fd[z].ica.empty())
      return fail(SMILI_ERR_ARG, "a frame has uv points but no data");
  double lcsum = 0;
  for (int z = 0; z < Nz; ++z) lcsum += a.lc_l[z];
  const bool lc_on = lcsum > 0;
  const bool lc_scale = lc_on && (a.lc_nidx == 1 || a.lc_nidx == 3);
  const double* xsrc = x_override ? x_override : a.iin;
  if (!finite_all(xsrc, N * Nz)) return fail(SMILI_ERR_DATA, "non-finite initial movie");
  // movie descriptor and its vectors
  ProbDesc& d = hp.d;
  std::memset(&d, 0, sizeof(d));
  const int n = N * Nz;
  d.npix = n;
  d.nx = a.nx;
  d.ny = a.ny;
  d.m = m;
  d.niter = niter;
  d.nonneg = nonneg ? 1 : 0;
  d.factr = factr;
  d.pgtol = pgtol;
  d.ftarget = -INFINITY;
  d.prec64 = sizeof(R) == 8;
  d.nxref = a.nxref;
  d.nyref = a.nyref;
  d.nframes = Nz;
  d.frame_npix = N;
  d.nfcv = nfcv;
  d.namp = namp;
  d.ncp = ncp;
  d.nca = nca;
  d.wfcv = nfcv ? a.wfcv / wtotal : 0;
  d.wamp = namp ? a.wamp / wtotal : 0;
  d.wcp = ncp ? a.wcp / wtotal : 0;
  d.wca = nca ? a.wca / wtotal : 0;
  d.has_rt = a.rt_l > 0;
  d.has_ri = a.ri_l > 0;
  d.has_lc = lc_on;
  d.rt_l = a.rt_l;
  d.ri_l = a.ri_l;
  if (d.has_rt && (!a.rt_wgt || a.rt_nwgt != N)) return fail(SMILI_ERR_ARG, "rt weights must have npix entries");
  if (d.has_ri && (!a.ri_wgt || a.ri_nwgt != N)) return fail(SMILI_ERR_ARG, "ri weights must have npix entries");
  d.o_x0 = ar.take(sizeof(double) * n);
  d.o_x = ar.take(sizeof(double) * n);
  d.o_g = ar.take(sizeof(double) * n);
  d.o_z = ar.take(sizeof(double) * n);
  d.o_r = ar.take(sizeof(double) * n);
  d.o_d = ar.take(sizeof(double) * n);
  d.o_t = ar.take(sizeof(double) * n);
  d.o_xp = ar.take(sizeof(double) * n);
  d.o_iwh = ar.take(n);
  d.o_free = ar.take(n);
  d.o_bkey = ar.take(sizeof(unsigned long long) * n);
  d.o_sbk = ar.take(sizeof(unsigned long long) * n);
  d.o_sbi = ar.take(sizeof(int) * n);
  d.o_hist = ar.take(sizeof(int) * 2 * 4096);
  d.o_lred = ar.take(sizeof(double) * 64);
  d.o_trace = ar.take(sizeof(double) * (niter + 2));
  if (kind == PK_SOLVE) {  // S and Y: R per element (FP32 storage in the FP32 mode)
    d.o_ws = ar.take(sizeof(R) * (size_t)n * m);
    d.o_wy = ar.take(sizeof(R) * (size_t)n * m);
  }
  d.o_frames = ar.take(sizeof(ProbDesc) * Nz);
  d.o_lcf = ar.take(sizeof(double) * Nz);
  if (d.has_rt) d.o_rtw = ar.take(sizeof(double) * N);
  if (d.has_ri) {
    d.o_riw = ar.take(sizeof(double) * N);
    d.o_iavg = ar.take(sizeof(double) * N);
  }
  // frames
  std::vector<HostProb> fh(Nz);
  std::vector<double> w1, wtv, wtsv, wkl, wgs;
  for (int z = 0; z < Nz; ++z) {
    const FrameData& f = fd[z];
    smili_imaging_args fa;
    std::memset(&fa, 0, sizeof(fa));
    fa.npix = N;
    fa.nx = a.nx;
    fa.ny = a.ny;
    fa.iin = xsrc + (size_t)z * N;
    fa.xidx = a.xidx;
    fa.yidx = a.yidx;
    fa.nxref = a.nxref;
    fa.nyref = a.nyref;
    fa.nuv = a.nuvs[z];
    fa.u = nuv ? a.u + off[z] : nullptr;
    fa.v = nuv ? a.v + off[z] : nullptr;
    const double c = lc_scale ? a.tfd_tgtfd / a.lc_tgtfd[z] : 1.0;
    auto scaled = [&](const double* w, int nw, double fac, std::vector<double>& buf) -> const double* {
      if (!w || fac == 1.0) return w;
      buf.assign(w, w + nw);
      for (auto& v : buf) v *= fac;
      return buf.data();
    };
    fa.l1_l = a.l1_l > 0 ? a.l1_l / Nz : a.l1_l;
    fa.l1_wgt = scaled(a.l1_wgt, a.l1_nwgt, c, w1);
    fa.l1_nwgt = a.l1_nwgt;
    fa.tv_l = a.tv_l > 0 ? a.tv_l / Nz : a.tv_l;
    fa.tv_wgt = scaled(a.tv_wgt, a.tv_nwgt, c, wtv);
    fa.tv_nwgt = a.tv_nwgt;
    fa.tsv_l = a.tsv_l > 0 ? a.tsv_l / Nz : a.tsv_l;
    fa.tsv_wgt = scaled(a.tsv_wgt, a.tsv_nwgt, c * c, wtsv);
    fa.tsv_nwgt = a.tsv_nwgt;
    fa.kl_l = a.kl_l > 0 ? a.kl_l / Nz : a.kl_l;
    fa.kl_wgt = scaled(a.kl_wgt, a.kl_nwgt, c, wkl);
    fa.kl_nwgt = a.kl_nwgt;
    fa.gs_l = a.gs_l > 0 ? a.gs_l / Nz : a.gs_l;
    fa.gs_wgt = scaled(a.gs_wgt, a.gs_nwgt, c, wgs);
    fa.gs_nwgt = a.gs_nwgt;
    if (lc_on) {
      fa.tfd_l = a.lc_l[z] > 0 ? a.lc_l[z] / Nz : a.lc_l[z];
      fa.tfd_tgtfd = a.lc_tgtfd[z];
    } else {
      fa.tfd_l = a.tfd_l > 0 ? a.tfd_l / Nz : a.tfd_l;
      fa.tfd_tgtfd = a.tfd_tgtfd;
    }
    fa.cen_l = -1.0;
    fa.cen_alpha = 1.0;
    fa.sm_l = a.sm_l > 0 ? a.sm_l / Nz : a.sm_l;
    fa.sm_maj = a.sm_maj;
    fa.sm_min = a.sm_min;
    fa.sm_phi = a.sm_phi;
    fa.isfcv = !f.ifcv.empty();
    fa.nfcv = (int)f.ifcv.size();
    fa.uvidxfcv = f.ifcv.data();
    fa.vfcvr = f.fr.data();
    fa.vfcvi = f.fi.data();
    fa.varfcv = f.fv.data();
    fa.wfcv = a.wfcv;
    fa.isamp = !f.iamp.empty();
    fa.namp = (int)f.iamp.size();
    fa.uvidxamp = f.iamp.data();
    fa.vamp = f.av.data();
    fa.varamp = f.avar.data();
    fa.wamp = a.wamp;
    fa.iscp = !f.cpv.empty();
    fa.ncp = (int)f.cpv.size();
    fa.uvidxcp = f.icp.data();
    fa.cp = f.cpv.data();
    fa.varcp = f.cpvar.data();
    fa.wcp = a.wcp;
    fa.isca = !f.cav.empty();
    fa.nca = (int)f.cav.size();
    fa.uvidxca = f.ica.data();
    fa.ca = f.cav.data();
    fa.varca = f.cavar.data();
    fa.wca = a.wca;
    fa.inormfactr = a.inormfactr;
    if ((rc = pack_problem<R>(fa, PK_FRAME, 0, nonneg, m, factr, pgtol, eps, ar, fh[z], nullptr, nullptr, nullptr,
                              wtotal, spread_bin, transform)) != SMILI_OK)
      return rc;
    ProbDesc& F = fh[z].d;
    F.o_x = d.o_x + (int64_t)sizeof(double) * z * N;
    F.o_g = d.o_g + (int64_t)sizeof(double) * z * N;
    F.o_d = d.o_d + (int64_t)sizeof(double) * z * N;
    F.nonneg = d.nonneg;
  }
  // blobs: movie vectors, then every frame's arrays and the frame descriptors
  hp.put(d.o_x0, std::vector<double>(xsrc, xsrc + n));
  hp.put(d.o_lcf, std::vector<double>(a.lc_tgtfd, a.lc_tgtfd + Nz));
  if (d.has_rt) hp.put(d.o_rtw, a.rt_wgt, (size_t)N);
  if (d.has_ri) hp.put(d.o_riw, a.ri_wgt, (size_t)N);
  std::vector<ProbDesc> fdesc(Nz);
  for (int z = 0; z < Nz; ++z) {
    fdesc[z] = fh[z].d;
    for (auto& bl : fh[z].blobs)
      if (bl.first >= 0) hp.blobs.emplace_back(bl.first, std::move(bl.second));
  }
  hp.put(d.o_frames, fdesc);
  return SMILI_OK;
}

template <typename R>
int create_movie(const smili_imaging3d_args* a, int kind, int niter, int nonneg, int m, double factr,
                 double pgtol, const smili_options* opt, const double* x_over, smili_batch** out) {
  const double eps = (opt && opt->nufft_eps > 0) ? opt->nufft_eps : 1e-6;
  if (!(eps < 1.0)) return fail(SMILI_ERR_ARG, "nufft_eps must be in (0, 1)");
  if (m < 1 || m > SMILI_MAXM_DEV) return fail(SMILI_ERR_UNSUPPORTED, "L-BFGS-B memory m must be 1..6");
  smili_batch* b = new smili_batch();
  b->nprob = 1;
  b->prec64 = sizeof(R) == 8;
  b->device = opt ? opt->device : 0;
  b->kind = kind;
  Arena ar;
  std::vector<HostProb> hps(1);
  const int rc = pack_movie<R>(*a, kind, niter, nonneg, m, factr, pgtol, eps, ar, hps[0], x_over,
                               opt && opt->spread_bin ? opt->spread_bin : 8, opt ? opt->transform : 0);
  if (rc != SMILI_OK) {
    delete b;
    return rc;
  }
  b->descs.push_back(hps[0].d);
  b->arena_bytes = ar.bytes;
  return finish_batch<R>(b, hps, hps[0].d.npix, opt, out);
}

// One evaluation of a single data term with unit weight and no
// regularizer: the raw chi-square sum and gradient of model_fcv / amp / cp /
// ca (fftlib.f90:744-1254), with every datum's model and residual.
template <typename R>
int create_model(const smili_imaging_args& a, const double* x, const smili_options* opt, smili_batch** out) {
  const double eps = (opt && opt->nufft_eps > 0) ? opt->nufft_eps : 1e-6;
  if (!(eps < 1.0)) return fail(SMILI_ERR_ARG, "nufft_eps must be in (0, 1)");
  const int nterm = (a.isfcv != 0) + (a.isamp != 0) + (a.iscp != 0) + (a.isca != 0);
  if (nterm != 1) return fail(SMILI_ERR_ARG, "exactly one data term must be given");
  const double w = a.isfcv ? a.wfcv : a.isamp ? a.wamp : a.iscp ? a.wcp : a.wca;
  if (!(w > 0)) return fail(SMILI_ERR_ARG, "the data weight must be positive");
  smili_imaging_args b0 = a;
  b0.l1_l = b0.tv_l = b0.tsv_l = b0.kl_l = b0.gs_l = b0.tfd_l = b0.cen_l = b0.sm_l = -1.0;
  smili_batch* b = new smili_batch();
  b->nprob = 1;
  b->prec64 = sizeof(R) == 8;
  b->device = opt ? opt->device : 0;
  b->kind = PK_MODEL;
  Arena ar;
  std::vector<HostProb> hps(1);
  const int rc = pack_problem<R>(b0, PK_MODEL, 0, 0, 5, 1e1, 0.0, eps, ar, hps[0], x, nullptr, nullptr, w,
                                 opt && opt->spread_bin ? opt->spread_bin : 8, opt ? opt->transform : 0);
  if (rc != SMILI_OK) {
    delete b;
    return rc;
  }
  b->descs.push_back(hps[0].d);
  b->arena_bytes = ar.bytes;
  return finish_batch<R>(b, hps, hps[0].d.npix, opt, out);
}

int create_movie_any(const smili_imaging3d_args* a, int kind, int niter, int nonneg, int m, double factr,
                     double pgtol, const smili_options* opt, const double* x_over, smili_batch** out) {
  if (!a || !out) return fail(SMILI_ERR_ARG, "null argument");
  const int prec = opt && opt->precision ? opt->precision : 64;
  if (prec != 64 && prec != 32) return fail(SMILI_ERR_ARG, "precision must be 64 or 32");
  return prec == 64 ? create_movie<double>(a, kind, niter, nonneg, m, factr, pgtol, opt, x_over, out)
                    : create_movie<float>(a, kind, niter, nonneg, m, factr, pgtol, opt, x_over, out);
}

int run(smili_batch* b, int mode, float* ms) {
  CUDA_TRY(cudaSetDevice(b->device));
  return b->prec64 ? launch_batch<double>(b, mode, ms) : launch_batch<float>(b, mode, ms);
}

int create_any(int nprob, const smili_imaging_args* const* probs, const int* niter, int nonneg, int m,
               double factr, double pgtol, const smili_options* opt, int kind, const double* const* x_over,
               const double* c_re, const double* c_im, smili_batch** out) {
  if (nprob < 1 || !probs || !out) return fail(SMILI_ERR_ARG, "invalid batch arguments");
  const int prec = opt && opt->precision ? opt->precision : 64;
  if (prec != 64 && prec != 32) return fail(SMILI_ERR_ARG, "precision must be 64 or 32");
  if (prec == 64)
    return create_batch<double>(nprob, probs, niter, nonneg, m, factr, pgtol, opt, kind, x_over, c_re, c_im, out);
  return create_batch<float>(nprob, probs, niter, nonneg, m, factr, pgtol, opt, kind, x_over, c_re, c_im, out);
}

}  // namespace

// Every C-ABI entry point runs its body through guarded(): a C++ exception
// (host allocation failure, mostly) becomes SMILI_ERR_HOST with a message
// instead of unwinding into the C caller.
template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    return fail(SMILI_ERR_HOST, "out of host memory");
  } catch (const std::exception& e) {
    return fail(SMILI_ERR_HOST, std::string("host failure: ") + e.what());
  } catch (...) {
    return fail(SMILI_ERR_HOST, "host failure");
  }
}

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* smili_last_error(void) { return g_err.c_str(); }
int smili_version(void) { return SMILI_VERSION; }

int smili_batch_create(int nprob, const smili_imaging_args* const* probs, const int* niter, int nonneg,
                       int m, double factr, double pgtol, const smili_options* opt, smili_batch** out) {
  return guarded([&]() -> int {
    return create_any(nprob, probs, niter, nonneg, m, factr, pgtol, opt, PK_SOLVE, nullptr, nullptr, nullptr,
                      out);
  });
}

int smili_batch_run(smili_batch* b, int fg_only, float* kernel_ms) {
  return guarded([&]() -> int {
    if (!b) return fail(SMILI_ERR_ARG, "null batch");
    if (fg_only == 2) return run(b, MODE_BARRIER, kernel_ms);  // barrier timing (diagnostic)
    if (fg_only == 3) return run(b, MODE_WAIT_LIMIT, kernel_ms);  // bounded-wait check (diagnostic)
    return run(b, fg_only ? MODE_FG : MODE_SOLVE, kernel_ms);
  });
}

int smili_batch_fetch(smili_batch* b, int p, double* iout, double* terms, double* grad,
                      smili_solve_info* info) {
  return guarded([&]() -> int {
    if (!b || p < 0 || p >= b->nprob) return fail(SMILI_ERR_ARG, "invalid problem index");
    CUDA_TRY(cudaSetDevice(b->device));
    const ProbDesc& d = b->descs[p];
    if (iout) CUDA_TRY(cudaMemcpy(iout, b->d_arena + d.o_x, sizeof(double) * d.npix, cudaMemcpyDeviceToHost));
    if (grad) CUDA_TRY(cudaMemcpy(grad, b->d_arena + d.o_g, sizeof(double) * d.npix, cudaMemcpyDeviceToHost));
    ProbResult r;
    CUDA_TRY(cudaMemcpy(&r, b->d_results + p, sizeof(r), cudaMemcpyDeviceToHost));
    if (terms) std::memcpy(terms, r.terms, sizeof(double) * (d.nframes > 0 ? SMILI_NTERMS3D : SMILI_NTERMS));
    if (info) {
      info->task = r.task;
      info->niter = r.iter;
      info->nfg = r.nfg;
      info->error = r.error;
    }
    return SMILI_OK;
  });
}

int smili_batch_profile(smili_batch* b, int enable, double* stage_ns, int len) {
  return guarded([&]() -> int {
    if (!b) return fail(SMILI_ERR_ARG, "null batch");
    b->profile = enable ? 1 : 0;
    if (stage_ns && len > 0) {
      unsigned long long h[PR_NSTAGE];
      CUDA_TRY(cudaSetDevice(b->device));
      CUDA_TRY(cudaMemcpy(h, b->d_prof, sizeof(h), cudaMemcpyDeviceToHost));
      for (int i = 0; i < len; ++i) stage_ns[i] = i < PR_NSTAGE ? (double)h[i] : 0.0;
    }
    return SMILI_OK;
  });
}

int smili_batch_set_targets(smili_batch* b, const double* ftarget) {
  return guarded([&]() -> int {
    if (!b) return fail(SMILI_ERR_ARG, "null batch");
    for (int p = 0; p < b->nprob; ++p) b->descs[p].ftarget = ftarget ? ftarget[p] : -INFINITY;
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaMemcpyAsync(b->d_descs, b->descs.data(), sizeof(ProbDesc) * b->nprob, cudaMemcpyHostToDevice,
                             b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SMILI_OK;
  });
}

int smili_batch_set_niter(smili_batch* b, const int* niter) {
  return guarded([&]() -> int {
    if (!b) return fail(SMILI_ERR_ARG, "null batch");
    if ((int)b->niter_cap.size() != b->nprob) return fail(SMILI_ERR_ARG, "batch has no iteration caps");
    for (int p = 0; p < b->nprob; ++p) {
      const int v = niter ? niter[p] : b->niter_cap[p];
      if (v < 0 || v > b->niter_cap[p])
        return fail(SMILI_ERR_ARG, "niter must lie between 0 and the iteration cap the batch was created with");
    }
    for (int p = 0; p < b->nprob; ++p) b->descs[p].niter = niter ? niter[p] : b->niter_cap[p];
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaMemcpyAsync(b->d_descs, b->descs.data(), sizeof(ProbDesc) * b->nprob, cudaMemcpyHostToDevice,
                             b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SMILI_OK;
  });
}

namespace {

// Saves every problem's packed start image once, before the first call that
// replaces one (reset_starts puts them back).
int save_starts(smili_batch* b) {
  if (b->d_x0_saved) return SMILI_OK;
  size_t total = 0;
  b->x0_saved_off.assign(b->nprob, 0);
  for (int p = 0; p < b->nprob; ++p) {
    b->x0_saved_off[p] = total;
    if (b->descs[p].o_x0 && b->descs[p].nframes == 0) total += (size_t)b->descs[p].npix;
  }
  CUDA_TRY(cudaMalloc(&b->d_x0_saved, sizeof(double) * std::max<size_t>(total, 1)));
  for (int p = 0; p < b->nprob; ++p) {
    const ProbDesc& d = b->descs[p];
    if (!d.o_x0 || d.nframes > 0) continue;
    CUDA_TRY(cudaMemcpyAsync(b->d_x0_saved + b->x0_saved_off[p], b->d_arena + d.o_x0, sizeof(double) * d.npix,
                             cudaMemcpyDeviceToDevice, b->stream));
  }
  return SMILI_OK;
}

// checks shared by the device-side warm-start calls
int check_images(smili_batch* b, int nx, int ny) {
  if (nx <= 0 || ny <= 0) return fail(SMILI_ERR_ARG, "invalid grid size");
  for (const ProbDesc& d : b->descs)
    if (!d.o_x0 || d.nframes > 0 || d.nx != nx || d.ny != ny)
      return fail(SMILI_ERR_UNSUPPORTED, "every problem must be an nx x ny 2D image with a replaceable start");
  return SMILI_OK;
}

constexpr int kWarmThreads = 256;

__device__ double block_sum(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ double block_max(double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + st]);
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// one block per problem: its current image as a dense grid scaled to max 1
__global__ void __launch_bounds__(kWarmThreads) batch_images_kernel(const ProbDesc* descs, const char* arena,
                                                                    float* dst, int nx, int ny) {
  __shared__ double sh[kWarmThreads];
  const ProbDesc& d = descs[blockIdx.x];
  const double* x = reinterpret_cast<const double*>(arena + d.o_x);
  const int* xi = reinterpret_cast<const int*>(arena + d.o_xidx);
  const int* yi = reinterpret_cast<const int*>(arena + d.o_yidx);
  float* out = dst + (size_t)blockIdx.x * nx * ny;
  double m = -INFINITY;
  for (int i = threadIdx.x; i < d.npix; i += blockDim.x) m = fmax(m, x[i]);
  m = block_max(m, sh);
  for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) out[c] = 0.f;
  __syncthreads();
  if (m > 0.0)
    for (int i = threadIdx.x; i < d.npix; i += blockDim.x) out[(size_t)yi[i] * nx + xi[i]] = (float)(x[i] / m);
}

// one block per problem: start image from relu(img), scaled to the current
// image's total, or the current image itself
__global__ void __launch_bounds__(kWarmThreads) batch_starts_kernel(const ProbDesc* descs, char* arena,
                                                                    const float* img, int nx, int ny,
                                                                    const unsigned char* keep) {
  __shared__ double sh[kWarmThreads];
  const ProbDesc& d = descs[blockIdx.x];
  const double* x = reinterpret_cast<const double*>(arena + d.o_x);
  const int* xi = reinterpret_cast<const int*>(arena + d.o_xidx);
  const int* yi = reinterpret_cast<const int*>(arena + d.o_yidx);
  double* x0 = reinterpret_cast<double*>(arena + d.o_x0);
  const float* g = img + (size_t)blockIdx.x * nx * ny;
  double s = 0.0, bad = 0.0, f = 0.0;
  for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
    const float v = g[c];
    if (!isfinite(v)) bad = 1.0;
    else if (v > 0.f) s += (double)v;
  }
  for (int i = threadIdx.x; i < d.npix; i += blockDim.x) f += x[i];
  s = block_sum(s, sh);
  f = block_sum(f, sh);
  bad = block_max(bad, sh);
  const bool own = (keep && keep[blockIdx.x]) || bad > 0.0 || !(s > 0.0) || !(f > 0.0);
  const double sc = own ? 0.0 : f / s;
  for (int i = threadIdx.x; i < d.npix; i += blockDim.x)
    x0[i] = own ? x[i] : (double)fmaxf(g[(size_t)yi[i] * nx + xi[i]], 0.f) * sc;
}

}  // namespace

int smili_batch_set_start(smili_batch* b, int p, const double* x) {
  return guarded([&]() -> int {
    if (!b || p < 0 || p >= b->nprob || !x) return fail(SMILI_ERR_ARG, "invalid start-image request");
    const ProbDesc& d = b->descs[p];
    if (!d.o_x0 || d.nframes > 0) return fail(SMILI_ERR_UNSUPPORTED, "this problem has no replaceable start image");
    for (int i = 0; i < d.npix; ++i)
      if (!std::isfinite(x[i])) return fail(SMILI_ERR_DATA, "non-finite start image");
    CUDA_TRY(cudaSetDevice(b->device));
    const int rc = save_starts(b);
    if (rc != SMILI_OK) return rc;
    CUDA_TRY(cudaMemcpyAsync(b->d_arena + d.o_x0, x, sizeof(double) * d.npix, cudaMemcpyHostToDevice, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SMILI_OK;
  });
}

int smili_batch_images(smili_batch* b, float* dst, int nx, int ny) {
  return guarded([&]() -> int {
    if (!b || !dst) return fail(SMILI_ERR_ARG, "null argument");
    int rc = check_images(b, nx, ny);
    if (rc != SMILI_OK) return rc;
    CUDA_TRY(cudaSetDevice(b->device));
    batch_images_kernel<<<b->nprob, kWarmThreads, 0, b->stream>>>(b->d_descs, b->d_arena, dst, nx, ny);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SMILI_OK;
  });
}

int smili_batch_set_starts_from_images(smili_batch* b, const float* img, int nx, int ny,
                                       const unsigned char* keep) {
  return guarded([&]() -> int {
    if (!b || !img) return fail(SMILI_ERR_ARG, "null argument");
    int rc = check_images(b, nx, ny);
    if (rc != SMILI_OK) return rc;
    CUDA_TRY(cudaSetDevice(b->device));
    if ((rc = save_starts(b)) != SMILI_OK) return rc;
    if (keep) {
      if (!b->d_keep) CUDA_TRY(cudaMalloc(&b->d_keep, b->nprob));
      CUDA_TRY(cudaMemcpyAsync(b->d_keep, keep, b->nprob, cudaMemcpyHostToDevice, b->stream));
    }
    batch_starts_kernel<<<b->nprob, kWarmThreads, 0, b->stream>>>(b->d_descs, b->d_arena, img, nx, ny,
                                                                  keep ? b->d_keep : nullptr);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SMILI_OK;
  });
}

int smili_batch_reset_starts(smili_batch* b) {
  return guarded([&]() -> int {
    if (!b) return fail(SMILI_ERR_ARG, "null batch");
    if (!b->d_x0_saved) return SMILI_OK;  // nothing was replaced
    CUDA_TRY(cudaSetDevice(b->device));
    for (int p = 0; p < b->nprob; ++p) {
      const ProbDesc& d = b->descs[p];
      if (!d.o_x0 || d.nframes > 0) continue;
      CUDA_TRY(cudaMemcpyAsync(b->d_arena + d.o_x0, b->d_x0_saved + b->x0_saved_off[p], sizeof(double) * d.npix,
                               cudaMemcpyDeviceToDevice, b->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return SMILI_OK;
  });
}

int smili_batch_trace(smili_batch* b, int p, double* trace, int len) {
  return guarded([&]() -> int {
    if (!b || p < 0 || p >= b->nprob || !trace) return fail(SMILI_ERR_ARG, "invalid trace request");
    const ProbDesc& d = b->descs[p];
    if (!d.o_trace) return fail(SMILI_ERR_ARG, "no trace for this batch");
    const int n = std::min(len, d.niter + 2);
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaMemcpy(trace, b->d_arena + d.o_trace, sizeof(double) * n, cudaMemcpyDeviceToHost));
    for (int i = n; i < len; ++i) trace[i] = NAN;
    return SMILI_OK;
  });
}

void smili_batch_destroy(smili_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->d_arena) cudaFree(b->d_arena);
  if (b->d_aux) cudaFree(b->d_aux);
  if (b->d_x0_saved) cudaFree(b->d_x0_saved);
  if (b->d_keep) cudaFree(b->d_keep);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int smili_fftim2d_imaging(const smili_imaging_args* a, int niter, int nonneg, int nprint, int m, double factr,
                          double pgtol, const smili_options* opt, double* iout, double* terms,
                          smili_solve_info* info) {
  return guarded([&]() -> int {
    (void)nprint;  // progress prints re-evaluate the cost at the same image; no effect on the result
    if (!a || !iout) return fail(SMILI_ERR_ARG, "null argument");
    if (niter < 0) return fail(SMILI_ERR_ARG, "niter must be >= 0");
    smili_batch* b = nullptr;
    const smili_imaging_args* probs[1] = {a};
    int rc = create_any(1, probs, &niter, nonneg, m, factr, pgtol, opt, PK_SOLVE, nullptr, nullptr, nullptr, &b);
    if (rc != SMILI_OK) return rc;
    rc = run(b, MODE_SOLVE, nullptr);
    if (rc == SMILI_OK) rc = smili_batch_fetch(b, 0, iout, terms, nullptr, info);
    smili_batch_destroy(b);
    return rc;
  });
}

int smili_calc_cost(const smili_imaging_args* a, const double* x, const smili_options* opt, double* terms,
                    double* grad) {
  return guarded([&]() -> int {
    if (!a || !x) return fail(SMILI_ERR_ARG, "null argument");
    smili_batch* b = nullptr;
    const smili_imaging_args* probs[1] = {a};
    const double* xo[1] = {x};
    int rc = create_any(1, probs, nullptr, 0, 5, 1e1, 0.0, opt, PK_FG, xo, nullptr, nullptr, &b);
    if (rc != SMILI_OK) return rc;
    rc = run(b, MODE_FG, nullptr);
    if (rc == SMILI_OK) rc = smili_batch_fetch(b, 0, nullptr, terms, grad, nullptr);
    smili_batch_destroy(b);
    return rc;
  });
}

int smili_fftim3d_imaging(const smili_imaging3d_args* a, int niter, int nonneg, int nprint, int m, double factr,
                          double pgtol, const smili_options* opt, double* iout, double* terms3d,
                          smili_solve_info* info) {
  return guarded([&]() -> int {
    (void)nprint;  // progress prints re-evaluate the cost at the same movie; no effect on the result
    if (!a || !iout) return fail(SMILI_ERR_ARG, "null argument");
    if (niter < 0) return fail(SMILI_ERR_ARG, "niter must be >= 0");
    smili_batch* b = nullptr;
    int rc = create_movie_any(a, PK_SOLVE, niter, nonneg, m, factr, pgtol, opt, nullptr, &b);
    if (rc != SMILI_OK) return rc;
    rc = run(b, MODE_SOLVE, nullptr);
    if (rc == SMILI_OK) rc = smili_batch_fetch(b, 0, iout, terms3d, nullptr, info);
    smili_batch_destroy(b);
    if (rc == SMILI_OK) {
      const size_t n = (size_t)a->npix * a->nz;
      for (size_t i = 0; i < n; ++i)
        if (std::fabs(iout[i]) < 1e-10) iout[i] = 0.0;  // fftim3d.f90:466 (zeroeps)
    }
    return rc;
  });
}

int smili_calc_cost3d(const smili_imaging3d_args* a, const double* x, const smili_options* opt, double* terms3d,
                      double* grad) {
  return guarded([&]() -> int {
    if (!a || !x) return fail(SMILI_ERR_ARG, "null argument");
    smili_batch* b = nullptr;
    int rc = create_movie_any(a, PK_FG, 0, 0, 5, 1e1, 0.0, opt, x, &b);
    if (rc != SMILI_OK) return rc;
    rc = run(b, MODE_FG, nullptr);
    if (rc == SMILI_OK) rc = smili_batch_fetch(b, 0, nullptr, terms3d, grad, nullptr);
    smili_batch_destroy(b);
    return rc;
  });
}

int smili_model_terms(const smili_imaging_args* a, const double* x, const smili_options* opt, double* chisq,
                      double* grad, double* model_re, double* model_im, double* resid_re, double* resid_im) {
  return guarded([&]() -> int {
    if (!a || !x) return fail(SMILI_ERR_ARG, "null argument");
    const int prec = opt && opt->precision ? opt->precision : 64;
    if (prec != 64 && prec != 32) return fail(SMILI_ERR_ARG, "precision must be 64 or 32");
    smili_batch* b = nullptr;
    int rc = prec == 64 ? create_model<double>(*a, x, opt, &b) : create_model<float>(*a, x, opt, &b);
    if (rc != SMILI_OK) return rc;
    rc = run(b, MODE_FG, nullptr);
    double terms[SMILI_NTERMS];
    if (rc == SMILI_OK) rc = smili_batch_fetch(b, 0, nullptr, terms, grad, nullptr);
    if (rc == SMILI_OK) {
      const ProbDesc& d = b->descs[0];
      std::vector<double> mr(4 * (size_t)d.ndata);
      cudaError_t e = cudaMemcpy(mr.data(), b->d_arena + d.o_model, sizeof(double) * mr.size(), cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        rc = fail(SMILI_ERR_CUDA, cudaGetErrorString(e));
      } else {
        if (chisq) *chisq = terms[0];
        const double dix = a->nx / 2.0 + 1 - a->nxref, diy = a->ny / 2.0 + 1 - a->nyref;
        for (int i = 0; i < d.ndata; ++i) {
          std::complex<double> mo(mr[4 * i], mr[4 * i + 1]), re(mr[4 * i + 2], mr[4 * i + 3]);
          if (a->isfcv) {  // phashift_c2r (fftlib.f90:200-220) of model and residual
            const int k = std::abs(a->uvidxfcv[i]) - 1, sg = a->uvidxfcv[i] > 0 ? 1 : -1;
            const std::complex<double> ph = std::exp(std::complex<double>(0.0, a->u[k] * sg * dix + a->v[k] * sg * diy));
            mo *= ph;
            re *= ph;
          } else if (a->iscp) {  // model_cp wraps both into (-pi, pi] (fftlib.f90:1227-1228)
            mo = std::atan2(std::sin(mo.real()), std::cos(mo.real()));
            re = std::atan2(std::sin(re.real()), std::cos(re.real()));
          }
          if (model_re) model_re[i] = mo.real();
          if (model_im) model_im[i] = mo.imag();
          if (resid_re) resid_re[i] = re.real();
          if (resid_im) resid_im[i] = re.imag();
        }
      }
    }
    smili_batch_destroy(b);
    return rc;
  });
}

static smili_imaging_args bare_args(int nuv, const double* u, const double* v, int nx, int ny,
                                    std::vector<double>& img, std::vector<int>& xi, std::vector<int>& yi) {
  smili_imaging_args a;
  std::memset(&a, 0, sizeof(a));
  a.npix = nx * ny;
  a.nx = nx;
  a.ny = ny;
  xi.resize(a.npix);
  yi.resize(a.npix);
  for (int i = 0; i < a.npix; ++i) {
    xi[i] = i % nx + 1;
    yi[i] = i / nx + 1;
  }
  if ((int)img.size() < a.npix) img.resize(a.npix, 0.0);
  a.iin = img.data();
  a.xidx = xi.data();
  a.yidx = yi.data();
  a.nxref = nx / 2 + 1;
  a.nyref = ny / 2 + 1;
  a.nuv = nuv;
  a.u = u;
  a.v = v;
  return a;
}

int smili_nufft_fwd_real(int nuv, const double* u, const double* v, int nx, int ny, const double* img,
                         const smili_options* opt, double* vreal, double* vimag) {
  return guarded([&]() -> int {
    if (!u || !v || !img || !vreal || !vimag || nx < 1 || ny < 1 || nuv < 1)
      return fail(SMILI_ERR_ARG, "invalid nufft arguments");
    std::vector<double> im(img, img + (size_t)nx * ny);
    std::vector<int> xi, yi;
    smili_imaging_args a = bare_args(nuv, u, v, nx, ny, im, xi, yi);
    smili_batch* b = nullptr;
    const smili_imaging_args* probs[1] = {&a};
    int rc = create_any(1, probs, nullptr, 0, 5, 1e1, 0.0, opt, PK_T2, nullptr, nullptr, nullptr, &b);
    if (rc != SMILI_OK) return rc;
    // x = image in evaluation mode
    rc = run(b, MODE_T2, nullptr);
    if (rc == SMILI_OK) {
      const ProbDesc& d = b->descs[0];
      const size_t C = b->prec64 ? 16 : 8;
      std::vector<char> buf(C * nuv);
      cudaError_t e = cudaMemcpy(buf.data(), b->d_arena + d.o_V, C * nuv, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = fail(SMILI_ERR_CUDA, cudaGetErrorString(e));
      const std::vector<int>& perm = b->perms[0];
      for (int j = 0; j < nuv && rc == SMILI_OK; ++j) {
        double re, im_;
        if (b->prec64) {
          re = reinterpret_cast<double*>(buf.data())[2 * j];
          im_ = reinterpret_cast<double*>(buf.data())[2 * j + 1];
        } else {
          re = reinterpret_cast<float*>(buf.data())[2 * j];
          im_ = reinterpret_cast<float*>(buf.data())[2 * j + 1];
        }
        vreal[perm[j]] = re;
        vimag[perm[j]] = im_;
      }
    }
    smili_batch_destroy(b);
    return rc;
  });
}

int smili_nufft_adj_real1d(int nuv, const double* u, const double* v, const double* vreal, const double* vimag,
                           int nx, int ny, const smili_options* opt, double* img) {
  return guarded([&]() -> int {
    if (!u || !v || !vreal || !vimag || !img || nx < 1 || ny < 1 || nuv < 1)
      return fail(SMILI_ERR_ARG, "invalid nufft arguments");
    std::vector<double> im;
    std::vector<int> xi, yi;
    smili_imaging_args a = bare_args(nuv, u, v, nx, ny, im, xi, yi);
    smili_batch* b = nullptr;
    const smili_imaging_args* probs[1] = {&a};
    int rc = create_any(1, probs, nullptr, 0, 5, 1e1, 0.0, opt, PK_T1, nullptr, vreal, vimag, &b);
    if (rc != SMILI_OK) return rc;
    rc = run(b, MODE_T1, nullptr);
    if (rc == SMILI_OK) {
      const ProbDesc& d = b->descs[0];
      cudaError_t e = cudaMemcpy(img, b->d_arena + d.o_gchi, sizeof(double) * nx * ny, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) rc = fail(SMILI_ERR_CUDA, cudaGetErrorString(e));
    }
    smili_batch_destroy(b);
    return rc;
  });
}

}  // extern "C"

#include "uvlist.cuh"

extern "C" int smili_get_uvlist(int n, const double* u, const double* v, const smili_options* opt, int* nuv,
                                double* u_out, double* v_out, int* uvidx) {
  return guarded([&]() -> int {
    return uvlist_run(n, u, v, opt ? opt->device : 0, opt ? static_cast<cudaStream_t>(opt->stream) : nullptr, nuv,
                      u_out, v_out, uvidx);
  });
}

// ===========================================================================
// Allocation-free calc_cost (no reference counterpart)
//
// The same evaluation as smili_calc_cost, with the problem arena and the
// launch's bookkeeping placed in one file-scope device array instead of
// cudaMalloc'd buffers.  It calls no CUDA allocator and no allocating
// library: its device scratch is g_noalloc_scratch, whose address is taken
// once per device with cudaGetSymbolAddress.  Problems whose arena does not
// fit are rejected with SMILI_ERR_ARG.  The one scratch array is shared by
// all calls on a device, so calls that overlap in time (other threads or
// streams) race; the first call on a device performs the set-up and should
// come before any stream capture.  The call is synchronous (it waits for its
// stream and copies the results back with blocking copies), so it must not
// be made while any stream of the process is capturing.  The set-up is kept
// for the life of the process: a cudaDeviceReset after the first call on a
// device is not supported.
// ===========================================================================
#include <mutex>

namespace {

constexpr size_t kNoAllocBytes = (size_t)SMILI_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDev = 64;
std::mutex g_noalloc_mu;
char* g_noalloc_ptr[kNoAllocMaxDev] = {};

// device address of the scratch array on `device` (which must be current)
int noalloc_scratch(int device, char** out) {
  if (device < 0 || device >= kNoAllocMaxDev) return fail(SMILI_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p || (reinterpret_cast<uintptr_t>(p) & 255u))
      return fail(SMILI_ERR_CUDA, "scratch symbol address is null or not 256-byte aligned");
    const size_t dyn64 = dyn_smem_bytes<double>();
    const size_t dyn32 = dyn_smem_bytes<float>();
    CUDA_TRY(cudaFuncSetAttribute((const void*)smili_batch_kernel<double>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn64));
    CUDA_TRY(cudaFuncSetAttribute((const void*)smili_batch_kernel<float>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn32));
    g_noalloc_ptr[device] = static_cast<char*>(p);
  }
  *out = g_noalloc_ptr[device];
  return SMILI_OK;
}

size_t round256(size_t n) { return (n + 255) / 256 * 256; }

template <typename R>
int calc_cost_noalloc(const smili_imaging_args* a, const double* x, const smili_options* opt, double* terms,
                      double* grad) {
  const double eps = (opt && opt->nufft_eps > 0) ? opt->nufft_eps : 1e-6;
  const int device = opt ? opt->device : 0;
  if (!(eps < 1.0)) return fail(SMILI_ERR_ARG, "nufft_eps must be in (0, 1)");
  Arena ar;
  HostProb hp;
  ar.take(256);  // as create_batch: no present field at offset 0, the mark of an absent one
  int rc = pack_problem<R>(*a, PK_FG, 0, 0, 5, 1e1, 0.0, eps, ar, hp, x, nullptr, nullptr, 0.0,
                           opt && opt->spread_bin ? opt->spread_bin : 8, opt ? opt->transform : 0);
  if (rc != SMILI_OK) return rc;
  const size_t arena_al = round256(std::max<size_t>(ar.bytes, 256));
  if (arena_al > kNoAllocBytes)
    return fail(SMILI_ERR_ARG, "smili_calc_cost_noalloc: the problem needs " + std::to_string(arena_al) +
                                   " bytes of device scratch, more than the " + std::to_string(kNoAllocBytes) +
                                   " of the static scratch; use smili_calc_cost");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) return fail(SMILI_ERR_NODEV, "no CUDA device");
  if (cudaSetDevice(device) != cudaSuccess) return fail(SMILI_ERR_NODEV, "cannot select the CUDA device");
  char* scratch = nullptr;
  rc = noalloc_scratch(device, &scratch);
  if (rc != SMILI_OK) return rc;
  // launch geometry for one problem (as in create_batch)
  smili_batch b;  // host bookkeeping only: every device pointer points into the scratch
  b.nprob = 1;
  b.prec64 = sizeof(R) == 8;
  b.device = device;
  b.kind = PK_FG;
  b.descs.push_back(hp.d);
  b.dyn_bytes = dyn_smem_bytes<R>();
  const void* fn = (const void*)smili_batch_kernel<R>;
  int occ = 0, nsm = 0, coop = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, Shape<R>::threads, b.dyn_bytes));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  if (!coop || occ < 1) return fail(SMILI_ERR_CUDA, "cooperative launch unavailable");
  const int maxres = occ * nsm;
  int G = opt && opt->ctas_per_problem > 0 ? opt->ctas_per_problem : 0;
  if (G <= 0) {  // finish_batch's rule for one problem: about four pixels per thread
    const int per_cta = 4 * Shape<R>::threads;
    G = std::max(1, std::min(maxres, (hp.d.npix + per_cta - 1) / per_cta));
  }
  G = std::min(G, maxres);
  b.G = G;
  b.ngroups = 1;
  // bookkeeping after the arena, laid out as in create_batch
  size_t off = arena_al;
  auto take = [&](size_t n) {
    const size_t o = off;
    off += round256(n);
    return o;
  };
  const size_t o_desc = take(sizeof(ProbDesc)), o_res = take(sizeof(ProbResult)), o_q = take(sizeof(int)),
               o_bar = take(sizeof(unsigned) * 2), o_rp = take(sizeof(double) * (size_t)G * SMILI_REDK),
               o_ro = take(sizeof(double) * SMILI_REDK), o_gp = take(sizeof(int)), o_ab = take(sizeof(int)),
               o_pf = take(sizeof(unsigned long long) * PR_NSTAGE);
  if (off > kNoAllocBytes)
    return fail(SMILI_ERR_ARG, "smili_calc_cost_noalloc: the problem needs " + std::to_string(off) +
                                   " bytes of device scratch, more than the " + std::to_string(kNoAllocBytes) +
                                   " of the static scratch; use smili_calc_cost");
  b.d_arena = scratch;
  b.arena_bytes = ar.bytes;
  b.d_aux = scratch + arena_al;
  b.d_descs = reinterpret_cast<ProbDesc*>(scratch + o_desc);
  b.d_results = reinterpret_cast<ProbResult*>(scratch + o_res);
  b.d_queue = reinterpret_cast<int*>(scratch + o_q);
  b.d_bars = reinterpret_cast<unsigned*>(scratch + o_bar);
  b.d_red_part = reinterpret_cast<double*>(scratch + o_rp);
  b.d_red_out = reinterpret_cast<double*>(scratch + o_ro);
  b.d_grp_prob = reinterpret_cast<int*>(scratch + o_gp);
  b.d_abort = reinterpret_cast<int*>(scratch + o_ab);
  b.d_prof = reinterpret_cast<unsigned long long*>(scratch + o_pf);
  b.stream = (opt && opt->stream) ? (cudaStream_t)opt->stream : cudaStreamPerThread;
  b.own_stream = false;
  // what must start at zero: the arena (as the allocating path clears it);
  // the queue, barrier counters and abort flag are cleared by launch_batch
  CUDA_TRY(cudaMemsetAsync(b.d_arena, 0, arena_al, b.stream));
  for (auto& bl : hp.blobs) {
    if (bl.first < 0 || bl.second.empty()) continue;  // host-side permutation; not needed for calc_cost
    CUDA_TRY(cudaMemcpyAsync(b.d_arena + bl.first, bl.second.data(), bl.second.size(), cudaMemcpyHostToDevice,
                             b.stream));
  }
  CUDA_TRY(cudaMemcpyAsync(b.d_descs, b.descs.data(), sizeof(ProbDesc), cudaMemcpyHostToDevice, b.stream));
  rc = launch_batch<R>(&b, MODE_FG, nullptr);
  if (rc != SMILI_OK) return rc;
  return smili_batch_fetch(&b, 0, nullptr, terms, grad, nullptr);
}

}  // namespace

extern "C" int smili_calc_cost_noalloc(const smili_imaging_args* a, const double* x, const smili_options* opt,
                                       double* terms, double* grad) {
  return guarded([&]() -> int {
    if (!a || !x) return fail(SMILI_ERR_ARG, "null argument");
    const int prec = opt && opt->precision ? opt->precision : 64;
    if (prec != 64 && prec != 32) return fail(SMILI_ERR_ARG, "precision must be 64 or 32");
    return prec == 64 ? calc_cost_noalloc<double>(a, x, opt, terms, grad)
                      : calc_cost_noalloc<float>(a, x, opt, terms, grad);
  });
}
