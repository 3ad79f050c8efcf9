// Device-resident L-BFGS-B (version 3.0), restating src/lbfgsb/lbfgsb.f.
//
// The CTAs of a group run the algorithm SPMD: vector work (length n) is split
// into one contiguous chunk per CTA; every reduction goes through
// group_reduce, whose result is bit-identical in every CTA, so each CTA keeps
// its own copy of the scalar state (LbState in shared memory, updated by
// thread 0) and all CTAs take the same branches without a broadcast.
//
// Differences from the sequential Fortran that only change rounding:
//  * dot products and norms are parallel reductions;
//  * formk builds the 2m x 2m matrix from Gram sums over the current free /
//    active sets instead of updating it with entering / leaving variables
//    (same matrix in exact arithmetic, lbfgsb.f:1848-2172);
//  * the generalized Cauchy point (cauchy, lbfgsb.f:1222-1719) visits the
//    breakpoints in increasing (t, index) order, taken in batches by radix
//    selection, and evaluates the piecewise quadratic in closed form from
//    prefix sums (D_k = sum d^2 over moving variables, P_k = W'd_k,
//    Q_k = sum t_i d_i w_i), instead of popping a heap and updating f1, f2
//    incrementally.  The f2 safeguard max(eps*f2_org, f2) is applied per
//    segment.  Ties between equal breakpoints are visited in index order.
// Only the bounds SMILI uses are supported: all variables unbounded
// (nbd = 0) or all bounded below by zero (nbd = 1, l = 0).
#pragma once
#include <cfloat>

#include "common.cuh"

#define SMILI_MAXM_DEV 6  // largest L-BFGS-B memory the device solver accepts
#define SMILI_KC 1024     // breakpoints per selection round of the Cauchy search

typedef unsigned __int128 u128;

// SY: the storage type of the limited-memory matrices S and Y (double in the
// FP64 mode, float in the FP32 mode); every dot product over them
// accumulates in FP64.
template <typename SY>
struct LbCtxT {
  const ProbDesc* P;
  char* base;
  GroupCtx* g;
  LbState* S;  // shared
  int n, m, lo, hi;
  double *x, *gv, *z, *r, *d, *t, *xp;
  SY *ws, *wy;
  signed char* iwh;
  unsigned char* freef;
  unsigned long long* bkey;
  double* lred;   // global scratch for results of the group-leader scan
  double* trace;
  double* red;    // shared [SMILI_REDK]
  unsigned char* ops;
  double* scratch;
  char* dyn;      // shared scratch (the FFT buffers)
  Prof* prof;
};

// S and Y element i (column-major, n per column), widened to FP64
template <typename SY>
__device__ __forceinline__ double ld_ws(const LbCtxT<SY>& c, size_t i) { return (double)c.ws[i]; }
template <typename SY>
__device__ __forceinline__ double ld_wy(const LbCtxT<SY>& c, size_t i) { return (double)c.wy[i]; }
template <typename SY>
__device__ __forceinline__ void st_sy(const LbCtxT<SY>& c, size_t i, double s, double y) {
  c.ws[i] = (SY)s;
  c.wy[i] = (SY)y;
}

// ---------------------------------------------------------------------------
// small dense algebra (thread 0)
// ---------------------------------------------------------------------------
__device__ int d_chol_upper(double* a, int lda, int nn) {  // linpack dpofa
  for (int j = 0; j < nn; ++j) {
    double s = 0.0;
    for (int k = 0; k < j; ++k) {
      double t = a[k + j * lda];
      for (int i = 0; i < k; ++i) t -= a[i + k * lda] * a[i + j * lda];
      t /= a[k + k * lda];
      a[k + j * lda] = t;
      s += t * t;
    }
    s = a[j + j * lda] - s;
    if (s <= 0.0) return j + 1;
    a[j + j * lda] = sqrt(s);
  }
  return 0;
}

__device__ int d_tri_solve(const double* t, int ldt, int nn, double* b, bool trans) {  // dtrsl 11/01
  for (int i = 0; i < nn; ++i)
    if (t[i + i * ldt] == 0.0) return i + 1;
  if (trans) {
    for (int j = 0; j < nn; ++j) {
      double s = b[j];
      for (int i = 0; i < j; ++i) s -= t[i + j * ldt] * b[i];
      b[j] = s / t[j + j * ldt];
    }
  } else {
    for (int j = nn - 1; j >= 0; --j) {
      b[j] /= t[j + j * ldt];
      const double bj = b[j];
      for (int i = 0; i < j; ++i) b[i] -= bj * t[i + j * ldt];
    }
  }
  return 0;
}

// product with the 2col x 2col middle matrix (bmv, lbfgsb.f:1106-1220)
__device__ int d_bmv(const LbState& S, int m, int col, const double* v, double* p) {
  if (col == 0) return 0;
#define SY(i, j) S.sy[((i)-1) + m * ((j)-1)]
  p[col] = v[col];
  for (int i = 2; i <= col; ++i) {
    double s = 0.0;
    for (int k = 1; k <= i - 1; ++k) s += SY(i, k) * v[k - 1] / SY(k, k);
    p[col + i - 1] = v[col + i - 1] + s;
  }
  if (d_tri_solve(S.wt, m, col, p + col, true)) return -1;
  for (int i = 1; i <= col; ++i) p[i - 1] = v[i - 1] / sqrt(SY(i, i));
  if (d_tri_solve(S.wt, m, col, p + col, false)) return -1;
  for (int i = 1; i <= col; ++i) p[i - 1] = -p[i - 1] / sqrt(SY(i, i));
  for (int i = 1; i <= col; ++i) {
    double s = 0.0;
    for (int k = i + 1; k <= col; ++k) s += SY(k, i) * p[col + k - 1] / SY(i, i);
    p[i - 1] += s;
  }
#undef SY
  return 0;
}

__device__ int d_formt(LbState& S, int m) {  // lbfgsb.f:2173-2240
  const int col = S.col;
#define SY(i, j) S.sy[((i)-1) + m * ((j)-1)]
#define SS(i, j) S.ss[((i)-1) + m * ((j)-1)]
#define WT(i, j) S.wt[((i)-1) + m * ((j)-1)]
  for (int j = 1; j <= col; ++j) WT(1, j) = S.theta * SS(1, j);
  for (int i = 2; i <= col; ++i)
    for (int j = i; j <= col; ++j) {
      const int k1 = min(i, j) - 1;
      double dd = 0.0;
      for (int k = 1; k <= k1; ++k) dd += SY(i, k) * SY(j, k) / SY(k, k);
      WT(i, j) = dd + S.theta * SS(i, j);
    }
#undef SY
#undef SS
#undef WT
  return d_chol_upper(S.wt, m, col) ? -3 : 0;
}

__device__ void d_dcstep(double& stx, double& fx, double& dx, double& sty, double& fy, double& dy,
                         double& stp, double fp, double dp, int& brackt, double stpmin,
                         double stpmax) {  // lbfgsb.f:3694-3949
  const double sgnd = dp * (dx / fabs(dx));
  double stpf, stpc, stpq;
  if (fp > fx) {
    const double th = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    const double s = fmax(fabs(th), fmax(fabs(dx), fabs(dp)));
    double gam = s * sqrt((th / s) * (th / s) - (dx / s) * (dp / s));
    if (stp < stx) gam = -gam;
    const double p = (gam - dx) + th, q = ((gam - dx) + gam) + dp, rr = p / q;
    stpc = stx + rr * (stp - stx);
    stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx);
    stpf = (fabs(stpc - stx) < fabs(stpq - stx)) ? stpc : stpc + (stpq - stpc) / 2.0;
    brackt = 1;
  } else if (sgnd < 0.0) {
    const double th = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    const double s = fmax(fabs(th), fmax(fabs(dx), fabs(dp)));
    double gam = s * sqrt((th / s) * (th / s) - (dx / s) * (dp / s));
    if (stp > stx) gam = -gam;
    const double p = (gam - dp) + th, q = ((gam - dp) + gam) + dx, rr = p / q;
    stpc = stp + rr * (stx - stp);
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    stpf = (fabs(stpc - stp) > fabs(stpq - stp)) ? stpc : stpq;
    brackt = 1;
  } else if (fabs(dp) < fabs(dx)) {
    const double th = 3.0 * (fx - fp) / (stp - stx) + dx + dp;
    const double s = fmax(fabs(th), fmax(fabs(dx), fabs(dp)));
    double gam = s * sqrt(fmax(0.0, (th / s) * (th / s) - (dx / s) * (dp / s)));
    if (stp > stx) gam = -gam;
    const double p = (gam - dp) + th, q = (gam + (dx - dp)) + gam, rr = p / q;
    if (rr < 0.0 && gam != 0.0) stpc = stp + rr * (stx - stp);
    else if (stp > stx) stpc = stpmax;
    else stpc = stpmin;
    stpq = stp + (dp / (dp - dx)) * (stx - stp);
    if (brackt) {
      stpf = (fabs(stpc - stp) < fabs(stpq - stp)) ? stpc : stpq;
      stpf = (stp > stx) ? fmin(stp + 0.66 * (sty - stp), stpf) : fmax(stp + 0.66 * (sty - stp), stpf);
    } else {
      stpf = (fabs(stpc - stp) > fabs(stpq - stp)) ? stpc : stpq;
      stpf = fmin(stpmax, stpf);
      stpf = fmax(stpmin, stpf);
    }
  } else {
    if (brackt) {
      const double th = 3.0 * (fp - fy) / (sty - stp) + dy + dp;
      const double s = fmax(fabs(th), fmax(fabs(dy), fabs(dp)));
      double gam = s * sqrt((th / s) * (th / s) - (dy / s) * (dp / s));
      if (stp > sty) gam = -gam;
      const double p = (gam - dp) + th, q = ((gam - dp) + gam) + dy, rr = p / q;
      stpc = stp + rr * (sty - stp);
      stpf = stpc;
    } else {
      stpf = (stp > stx) ? stpmax : stpmin;
    }
  }
  if (fp > fx) {
    sty = stp;
    fy = fp;
    dy = dp;
  } else {
    if (sgnd < 0.0) {
      sty = stx;
      fy = fx;
      dy = dx;
    }
    stx = stp;
    fx = fp;
    dx = dp;
  }
  stp = stpf;
}

enum { CS_START = 0, CS_FG = 1, CS_CONV = 2, CS_WARN = 3, CS_ERROR = 4 };

__device__ void d_dcsrch(LbState& S, double f, double g, double stpmin, double stpmax) {
  const double ftol = 1e-3, gtol = 0.9, xtol = 0.1;  // lnsrlb parameters (lbfgsb.f:2497)
  if (S.csave == CS_START) {
    if (S.stp < stpmin || S.stp > stpmax || g >= 0.0 || stpmax < stpmin) {
      S.csave = CS_ERROR;
      return;
    }
    S.brackt = 0;
    S.stage = 1;
    S.finit = f;
    S.ginit = g;
    S.gtest = ftol * S.ginit;
    S.width = stpmax - stpmin;
    S.width1 = S.width / 0.5;
    S.stx = 0.0;
    S.fx = S.finit;
    S.gx = S.ginit;
    S.sty = 0.0;
    S.fy = S.finit;
    S.gy = S.ginit;
    S.stmin = 0.0;
    S.stmax = S.stp + 4.0 * S.stp;
    S.csave = CS_FG;
    return;
  }
  const double ftest = S.finit + S.stp * S.gtest;
  if (S.stage == 1 && f <= ftest && g >= 0.0) S.stage = 2;
  int task = CS_FG;
  if (S.brackt && (S.stp <= S.stmin || S.stp >= S.stmax)) task = CS_WARN;
  if (S.brackt && S.stmax - S.stmin <= xtol * S.stmax) task = CS_WARN;
  if (S.stp == stpmax && f <= ftest && g <= S.gtest) task = CS_WARN;
  if (S.stp == stpmin && (f > ftest || g >= S.gtest)) task = CS_WARN;
  if (f <= ftest && fabs(g) <= gtol * (-S.ginit)) task = CS_CONV;
  if (task == CS_WARN || task == CS_CONV) {
    S.csave = task;
    return;
  }
  if (S.stage == 1 && f <= S.fx && f > ftest) {
    double fm = f - S.stp * S.gtest, fxm = S.fx - S.stx * S.gtest, fym = S.fy - S.sty * S.gtest;
    double gm = g - S.gtest, gxm = S.gx - S.gtest, gym = S.gy - S.gtest;
    d_dcstep(S.stx, fxm, gxm, S.sty, fym, gym, S.stp, fm, gm, S.brackt, S.stmin, S.stmax);
    S.fx = fxm + S.stx * S.gtest;
    S.fy = fym + S.sty * S.gtest;
    S.gx = gxm + S.gtest;
    S.gy = gym + S.gtest;
  } else {
    d_dcstep(S.stx, S.fx, S.gx, S.sty, S.fy, S.gy, S.stp, f, g, S.brackt, S.stmin, S.stmax);
  }
  if (S.brackt) {
    if (fabs(S.sty - S.stx) >= 0.66 * S.width1) S.stp = S.stx + 0.5 * (S.sty - S.stx);
    S.width1 = S.width;
    S.width = fabs(S.sty - S.stx);
  }
  if (S.brackt) {
    S.stmin = fmin(S.stx, S.sty);
    S.stmax = fmax(S.stx, S.sty);
  } else {
    S.stmin = S.stp + 1.1 * (S.stp - S.stx);
    S.stmax = S.stp + 4.0 * (S.stp - S.stx);
  }
  S.stp = fmax(S.stp, stpmin);
  S.stp = fmin(S.stp, stpmax);
  if ((S.brackt && (S.stp <= S.stmin || S.stp >= S.stmax)) ||
      (S.brackt && S.stmax - S.stmin <= xtol * S.stmax))
    S.stp = S.stx;
  S.csave = CS_FG;
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lptr(const LbState& S, int m, int j) {  // logical j (0-based) -> column
  return (S.head - 1 + j) % m;
}

__device__ __forceinline__ void reset_memory(LbState& S) {
  S.info = 0;
  S.col = 0;
  S.head = 1;
  S.theta = 1.0;
  S.iupdat = 0;
  S.updatd = 0;
}

// reduce acc[0..K) over the group with the ops in c.ops; result in c.red
template <typename SY>
__device__ bool lb_reduce(LbCtxT<SY>& c, const double* acc, int K) {
  block_reduce_arr(acc, c.ops, K, c.red, c.scratch);
  return group_reduce(*c.g, c.red, c.ops, K);
}

template <typename SY>
__device__ void set_ops(LbCtxT<SY>& c, int K, int op_default) {
  for (int k = threadIdx.x; k < K; k += blockDim.x) c.ops[k] = (unsigned char)op_default;
  __syncthreads();
}

// ---------------------------------------------------------------------------
// init: active() projection and state (lbfgsb.f:1004-1104, mainlb START)
// ---------------------------------------------------------------------------
template <typename SY>
__device__ void lb_init(LbCtxT<SY>& c, const double* x0) {
  LbState& S = *c.S;
  const ProbDesc& P = *c.P;
  if (threadIdx.x == 0) {
    S.task = LB_TASK_FG_START;
    S.done = 0;
    S.error = 0;
    S.col = 0;
    S.head = 1;
    S.itail = 0;
    S.iupdat = 0;
    S.iter = 0;
    S.nfgv = 0;
    S.ifun = 0;
    S.iback = 0;
    S.nseg = 0;
    S.nskip = 0;
    S.nintol = 0;
    S.info = 0;
    S.iword = 0;
    S.nfree = c.n;
    S.nact = 0;
    S.ileave = 0;
    S.nenter = 0;
    S.updatd = 0;
    S.wrk = 0;
    S.cnstnd = P.nonneg ? 1 : 0;
    S.boxed = 0;
    S.prjctd = 0;
    S.stage = 1;
    S.brackt = 0;
    S.csave = CS_START;
    S.nfg_total = 0;
    S.f = 0;
    S.theta = 1.0;
    S.fold = 0;
    S.epsmch = DBL_EPSILON;
    S.tol = P.factr * S.epsmch;
    S.dnorm = S.gd = S.stpmx = S.sbgnrm = S.stp = S.gdold = S.dtd = S.xstep = 0;
  }
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    double v = x0[i];
    if (P.nonneg && v < 0.0) v = 0.0;
    c.x[i] = v;
    c.iwh[i] = P.nonneg ? 0 : -1;
    c.freef[i] = 1;
    c.d[i] = 0.0;
    for (int j = 0; j < c.m; ++j) st_sy(c, (size_t)j * c.n + i, 0.0, 0.0);
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Cauchy point
// ---------------------------------------------------------------------------
// results written by the group leader to c.lred (global) for all CTAs
enum {
  CR_INFO = 0, CR_MODE, CR_TSUM, CR_NSEG, CR_BHI, CR_BLO, CR_C  // CR_C.. 2m values of c
};
enum { CM_NONE_FIXED = 0, CM_BOUNDARY = 1, CM_XCP_IS_X = 2 };

__device__ __forceinline__ u128 comp_key(unsigned long long key, int idx) {
  return ((u128)key << 32) | (u128)(unsigned)idx;
}

// Block-wide inclusive scan of V values per thread (vals in/out), V <= 32.
__device__ void block_scan_incl(double* vals, int V, double* wtot /* shared [WARPS][32] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = 0; v < V; ++v) {
    double a = vals[v];
    for (int s = 1; s < 32; s <<= 1) {
      const double o = __shfl_up_sync(0xffffffffu, a, s);
      if (lane >= s) a += o;
    }
    vals[v] = a;
    if (lane == 31) wtot[wid * 32 + v] = a;
  }
  __syncthreads();
  for (int v = 0; v < V; ++v) {
    double pre = 0.0;
    for (int w = 0; w < wid; ++w) pre += wtot[w * 32 + v];
    vals[v] += pre;
  }
  __syncthreads();
}

// Breakpoint bucketing (all CTAs of the group).  Keys are the IEEE bits of
// the breakpoint times t > 0, which order like the times; bucket =
// (key - kmin) >> shift, with the shift chosen so that the keys span at most
// SMILI_NBUCKET buckets.  sbk/sbi receive the breakpoints grouped by bucket in
// increasing bucket order (unordered inside a bucket); hist the bucket counts.
#define SMILI_NBUCKET 2048

__device__ __forceinline__ int bucket_of(unsigned long long k, unsigned long long kmin, int shift) {
  const unsigned long long q = (k - kmin) >> shift;
  return q < (unsigned long long)SMILI_NBUCKET ? (int)q : SMILI_NBUCKET - 1;
}

// Select the next batch (<= SMILI_KC elements, the smallest composites above
// lo_key) from the unordered range [r0, r1) of the bucketed arrays into cand,
// by radix selection on 12-bit digits of the 96-bit composite (key, index).
// Used for a bucket that holds more than SMILI_KC breakpoints.
template <typename SY>
__device__ int select_from_range(LbCtxT<SY>& c, const unsigned long long* sbk, const int* sbi, int r0,
                                 int r1, u128 lo_key, u128* cand, unsigned* hist) {
  __shared__ int cnt_s, vstar_s, cum_s;
  u128 prefix = 0;
  int level = 0, budget = SMILI_KC;
  u128 sel_hi = ~(u128)0;
  bool have_hi = false;
  while (true) {
    const int shift = 96 - 12 * (level + 1);
    for (int i = threadIdx.x; i < 4096; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const u128 ck = comp_key(sbk[i], sbi[i]);
      if (ck <= lo_key) continue;
      if (level > 0 && (ck >> (96 - 12 * level)) != prefix) continue;
      atomicAdd(&hist[(unsigned)((ck >> shift) & 0xfffu)], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int cum = 0, vstar = -1;
      for (int b = 0; b < 4096; ++b) {
        if (cum + (int)hist[b] > budget) {
          vstar = b;
          break;
        }
        cum += hist[b];
      }
      vstar_s = vstar;
      cum_s = cum;
    }
    __syncthreads();
    const int vstar = vstar_s, cum = cum_s;
    if (vstar < 0) {
      if (level > 0) {
        sel_hi = (prefix + 1) << (96 - 12 * level);
        have_hi = true;
      }
      break;
    }
    const u128 np = (prefix << 12) | (u128)vstar;
    if (cum == budget || (cum > 0 && (4 * cum >= budget || level == 7))) {
      sel_hi = np << shift;
      have_hi = true;
      break;
    }
    budget -= cum;
    prefix = np;
    ++level;
  }
  if (threadIdx.x == 0) cnt_s = 0;
  __syncthreads();
  for (int i0 = r0; i0 < r1; i0 += blockDim.x) {
    const int i = i0 + threadIdx.x;
    bool take = false;
    u128 ck = 0;
    if (i < r1) {
      ck = comp_key(sbk[i], sbi[i]);
      take = ck > lo_key && !(have_hi && ck >= sel_hi);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, take);
    if (bal) {
      const int lane = threadIdx.x & 31;
      int base = 0;
      if (lane == __ffs(bal) - 1) base = atomicAdd(&cnt_s, __popc(bal));
      base = __shfl_sync(0xffffffffu, base, __ffs(bal) - 1);
      const int pos = base + __popc(bal & ((1u << lane) - 1));
      if (take && pos < SMILI_KC) cand[pos] = ck;
    }
  }
  __syncthreads();
  const int cnt = min(cnt_s, SMILI_KC);
  __syncthreads();
  return cnt;
}

// Sequential-order scan of the bucketed breakpoints by one CTA (the group
// leader): batches of whole buckets (<= SMILI_KC elements) are sorted by
// (t, index) and swept with the closed-form piecewise quadratic.  Writes the
// CR_* results.
// Bytes of dynamic shared memory the scan lays out (cand, hist, hist2, wtot,
// dtm_s, t_s, Mm, st); the launch gives every CTA at least this much.
constexpr size_t SMILI_CAUCHY_SMEM =
    16 * SMILI_KC + 4 * SMILI_NBUCKET + 4 * 4096 +
    8 * (SMILI_MAX_WARPS * 32 + 2 * SMILI_MAX_THREADS + 4 * SMILI_MAXM_DEV * SMILI_MAXM_DEV + 5 + 4 * SMILI_MAXM_DEV);
template <typename SY>
__device__ void cauchy_scan(LbCtxT<SY>& c, double f1_0, const double* p0, int nbreak, int bnded,
                            const unsigned long long* sbk, const int* sbi, const int* ghist) {
  LbState& S = *c.S;
  const int m = c.m, col = S.col, col2 = 2 * col, n = c.n;
  const double theta = S.theta;
  // shared layout inside dyn
  u128* cand = reinterpret_cast<u128*>(c.dyn);                        // SMILI_KC
  unsigned* hist = reinterpret_cast<unsigned*>(cand + SMILI_KC);      // NBUCKET (bucket counts)
  unsigned* hist2 = hist + SMILI_NBUCKET;                             // 4096 (fallback)
  double* wtot = reinterpret_cast<double*>(hist2 + 4096);             // MAX_WARPS*32
  double* dtm_s = wtot + SMILI_MAX_WARPS * 32;                        // MAX_THREADS
  double* t_s = dtm_s + SMILI_MAX_THREADS;                            // MAX_THREADS
  double* Mm = t_s + SMILI_MAX_THREADS;                               // dense M (2col)^2
  double* st = Mm + 4 * SMILI_MAXM_DEV * SMILI_MAXM_DEV;              // carried state
  // st: [0]=D [1]=tprev [2]=dtm_cur [3..] unused [5..5+2m)=P [..+2m)=Q
  __shared__ unsigned long long bnd_hi_s, bnd_lo_s;
  __shared__ int e_star_s, info_s;
  __shared__ double f2org_s;
  double* Pst = st + 5;
  double* Qst = Pst + 2 * SMILI_MAXM_DEV;
  Prof& pf = *c.prof;
  double* lr = c.lred;

  // dense middle matrix: column j = M e_j
  if (threadIdx.x == 0) info_s = 0;
  __syncthreads();
  if (threadIdx.x < col2) {
    double e[2 * SMILI_MAXM_DEV], mc[2 * SMILI_MAXM_DEV];
    for (int k = 0; k < col2; ++k) e[k] = (k == (int)threadIdx.x) ? 1.0 : 0.0;
    if (d_bmv(S, m, col, e, mc)) info_s = -1;
    for (int k = 0; k < col2; ++k) Mm[k * col2 + threadIdx.x] = mc[k];
  }
  for (int i = threadIdx.x; i < SMILI_NBUCKET; i += blockDim.x) hist[i] = (unsigned)ghist[i];
  __syncthreads();
  if (info_s) {  // singular middle matrix (bmv failure)
    if (threadIdx.x == 0) lr[CR_INFO] = -1;
    __syncthreads();
    return;
  }
  if (threadIdx.x == 0) {
    double f2 = -theta * f1_0;
    const double f2_org = f2;
    if (col > 0) {
      double s = 0;
      for (int i = 0; i < col2; ++i)
        for (int j = 0; j < col2; ++j) s += p0[i] * Mm[i * col2 + j] * p0[j];
      f2 -= s;
    }
    st[0] = -f1_0;
    st[1] = 0.0;
    st[2] = -f1_0 / f2;
    for (int j = 0; j < col2; ++j) {
      Pst[j] = p0[j];
      Qst[j] = 0.0;
    }
    f2org_s = f2_org;
    bnd_hi_s = 0;
    bnd_lo_s = 0;
  }
  __syncthreads();
  const double f2_org = f2org_s;
  if (nbreak == 0) {  // GCP in the first segment (lbfgsb.f:1433, label 888)
    if (threadIdx.x == 0) {
      double dtm = st[2];
      if (dtm <= 0.0) dtm = 0.0;
      lr[CR_INFO] = 0;
      lr[CR_MODE] = CM_NONE_FIXED;
      lr[CR_TSUM] = dtm;
      lr[CR_NSEG] = 1;
      lr[CR_BHI] = 0.0;
      lr[CR_BLO] = 0.0;
      for (int j = 0; j < col2; ++j) lr[CR_C + j] = dtm * Pst[j];
    }
    __syncthreads();
    return;
  }
  int pj[SMILI_MAXM_DEV];
  for (int j = 0; j < col; ++j) pj[j] = lptr(S, m, j);
  const int V = 1 + 2 * col2;
  int kdone = 0, pos = 0, bucket = 0;
  // state of an oversized bucket being consumed by radix selection
  int big_r0 = -1, big_r1 = -1;
  while (true) {
    // ---------------- next batch ----------------
    int cnt = 0;
    const u128 lo_key = ((u128)bnd_hi_s << 64) | (u128)bnd_lo_s;
    if (big_r0 < 0) {
      while (bucket < SMILI_NBUCKET && hist[bucket] == 0) ++bucket;
      if (bucket < SMILI_NBUCKET && (int)hist[bucket] > SMILI_KC) {
        big_r0 = pos;
        big_r1 = pos + (int)hist[bucket];
      }
    }
    if (big_r0 >= 0) {
      cnt = select_from_range(c, sbk, sbi, big_r0, big_r1, lo_key, cand, hist2);
    } else {
      int b2 = bucket, tot = 0;
      while (b2 < SMILI_NBUCKET && tot + (int)hist[b2] <= SMILI_KC) tot += hist[b2++];
      for (int i = threadIdx.x; i < tot; i += blockDim.x) cand[i] = comp_key(sbk[pos + i], sbi[pos + i]);
      cnt = tot;
      pos += tot;
      bucket = b2;
    }
    __syncthreads();
    pf.mark(PR_C_SEL);
    pf.count(PR_C_ROUNDS);
    int np2 = 1;
    while (np2 < cnt) np2 <<= 1;
    for (int i = cnt + threadIdx.x; i < np2; i += blockDim.x) cand[i] = ~(u128)0;
    __syncthreads();
    // ---------------- bitonic sort ----------------
    for (int k2 = 2; k2 <= np2; k2 <<= 1) {
      for (int j2 = k2 >> 1; j2 > 0; j2 >>= 1) {
        for (int i = threadIdx.x; i < np2; i += blockDim.x) {
          const int ixj = i ^ j2;
          if (ixj > i) {
            const u128 a = cand[i], b = cand[ixj];
            const bool up = (i & k2) == 0;
            if ((a > b) == up) {
              cand[i] = b;
              cand[ixj] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    pf.mark(PR_C_SORT);
    // ---------------- scan in chunks of THREADS ----------------
    bool finished = false;
    const int T = blockDim.x;
    for (int base = 0; base < cnt; base += T) {
      const int e = threadIdx.x;
      const int ge = base + e;
      const bool valid = ge < cnt;
      double vals[1 + 4 * SMILI_MAXM_DEV];
      double te = 0.0;
      int idx = 0;
      for (int v = 0; v < V; ++v) vals[v] = 0.0;
      if (valid) {
        const u128 ck = cand[ge];
        idx = (int)(unsigned)(ck & 0xffffffffu);
        const unsigned long long kb = (unsigned long long)(ck >> 32);
        te = __longlong_as_double((long long)kb);
        const double dibp = c.d[idx];
        vals[0] = dibp * dibp;
        for (int j = 0; j < col; ++j) {
          const double wy_ = ld_wy(c, (size_t)pj[j] * n + idx);
          const double ws_ = theta * ld_ws(c, (size_t)pj[j] * n + idx);
          vals[1 + j] = dibp * wy_;
          vals[1 + col + j] = dibp * ws_;
          vals[1 + col2 + j] = te * dibp * wy_;
          vals[1 + col2 + col + j] = te * dibp * ws_;
        }
      }
      block_scan_incl(vals, V, wtot);
      double dtm_e = 0.0;
      double Pk[2 * SMILI_MAXM_DEV], ck_[2 * SMILI_MAXM_DEV];
      double Dk = 0.0;
      if (valid) {
        Dk = st[0] - vals[0];
        for (int j = 0; j < col2; ++j) {
          Pk[j] = Pst[j] - vals[1 + j];
          ck_[j] = te * Pk[j] + (Qst[j] + vals[1 + col2 + j]);
        }
        double cMp = 0.0, pMp = 0.0;
        for (int i = 0; i < col2; ++i) {
          double mp = 0.0;
          for (int j = 0; j < col2; ++j) mp += Mm[i * col2 + j] * Pk[j];
          cMp += ck_[i] * mp;
          pMp += Pk[i] * mp;
        }
        const double f1 = -Dk + theta * te * Dk - cMp;
        double f2 = theta * Dk - pMp;
        f2 = fmax(S.epsmch * f2_org, f2);
        dtm_e = -f1 / f2;
        dtm_s[e] = dtm_e;
        t_s[e] = te;
      }
      __syncthreads();
      // stop test for the segment ending at this element
      int stop = 0;
      if (valid) {
        const double pd = (e == 0) ? st[2] : dtm_s[e - 1];
        const double pt = (e == 0) ? st[1] : t_s[e - 1];
        stop = pd < (te - pt);
      }
      if (threadIdx.x == 0) e_star_s = T;
      __syncthreads();
      if (stop) atomicMin(&e_star_s, e);
      __syncthreads();
      const int es = e_star_s;
      const int nvalid = min(T, cnt - base);
      if (es < T) {
        // GCP inside the segment before element es: breakpoints up to es-1 fixed
        if ((es == 0 && threadIdx.x == 0) || (es > 0 && e == es - 1)) {
          double Pf[2 * SMILI_MAXM_DEV], Cf[2 * SMILI_MAXM_DEV];
          double tsum, dtm;
          if (es == 0) {
            tsum = st[1];
            dtm = st[2];
            for (int j = 0; j < col2; ++j) {
              Pf[j] = Pst[j];
              Cf[j] = tsum * Pst[j] + Qst[j];
            }
          } else {
            tsum = te;
            dtm = dtm_e;
            for (int j = 0; j < col2; ++j) {
              Pf[j] = Pk[j];
              Cf[j] = ck_[j];
            }
            const u128 ckk = comp_key(__double_as_longlong(te), idx);
            bnd_hi_s = (unsigned long long)(ckk >> 64);
            bnd_lo_s = (unsigned long long)ckk;
          }
          if (dtm <= 0.0) dtm = 0.0;
          lr[CR_INFO] = 0;
          lr[CR_MODE] = (kdone + es == 0) ? CM_NONE_FIXED : CM_BOUNDARY;
          lr[CR_TSUM] = tsum + dtm;
          lr[CR_NSEG] = kdone + es + 1;
          for (int j = 0; j < col2; ++j) lr[CR_C + j] = Cf[j] + dtm * Pf[j];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
          lr[CR_BHI] = __longlong_as_double((long long)bnd_hi_s);
          lr[CR_BLO] = __longlong_as_double((long long)bnd_lo_s);
        }
        finished = true;
        __syncthreads();
        break;
      }
      // no stop in this chunk: carry the state of its last element
      if (e == nvalid - 1) {
        st[0] = Dk;
        st[1] = te;
        st[2] = dtm_e;
        for (int j = 0; j < col2; ++j) {
          Pst[j] = Pk[j];
          Qst[j] = ck_[j] - te * Pk[j];
        }
        const u128 ckk = comp_key(__double_as_longlong(te), idx);
        bnd_hi_s = (unsigned long long)(ckk >> 64);
        bnd_lo_s = (unsigned long long)ckk;
      }
      __syncthreads();
      kdone += nvalid;
      if (kdone == nbreak) {
        // every breakpoint passed without a stop (lbfgsb.f:1640-1660)
        if (threadIdx.x == 0) {
          lr[CR_INFO] = 0;
          lr[CR_MODE] = CM_BOUNDARY;
          lr[CR_NSEG] = kdone;
          lr[CR_BHI] = __longlong_as_double((long long)bnd_hi_s);
          lr[CR_BLO] = __longlong_as_double((long long)bnd_lo_s);
          if (nbreak == n) {
            // all variables at their bounds; c = W'(xcp - x) = t_n P_n + Q_n
            lr[CR_TSUM] = st[1];
            for (int j = 0; j < col2; ++j) lr[CR_C + j] = st[1] * Pst[j] + Qst[j];
          } else {
            double dtm = bnded ? 0.0 : st[2];
            if (dtm <= 0.0) dtm = 0.0;
            lr[CR_TSUM] = st[1] + dtm;
            for (int j = 0; j < col2; ++j) lr[CR_C + j] = st[1] * Pst[j] + Qst[j] + dtm * Pst[j];
          }
        }
        finished = true;
        __syncthreads();
        break;
      }
    }
    pf.mark(PR_C_SCAN);
    if (finished) break;
    if (big_r0 >= 0 && kdone >= big_r1) {  // the oversized bucket is consumed
      pos = big_r1;
      ++bucket;
      big_r0 = big_r1 = -1;
    }
  }
  __syncthreads();
}

// Returns 0 on success, -1 when bmv failed (info != 0).
template <typename SY>
__device__ int lb_cauchy(LbCtxT<SY>& c) {
  LbState& S = *c.S;
  const ProbDesc& P = *c.P;
  const int m = c.m, n = c.n, col = S.col, col2 = 2 * col;
  const bool nonneg = P.nonneg;
  unsigned long long* sbk = at<unsigned long long>(c.base, P.o_sbk);
  int* sbi = at<int>(c.base, P.o_sbi);
  int* ghist = at<int>(c.base, P.o_hist);  // [NBUCKET] counts, [NBUCKET] cursors
  if (S.sbgnrm <= 0.0) {
    // GCP = X (lbfgsb.f:1318-1322): z = x, iwhere untouched
    for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) c.z[i] = c.x[i];
    if (threadIdx.x == 0) c.lred[CR_MODE] = CM_XCP_IS_X;
  } else {
    int pj[SMILI_MAXM_DEV];
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) pj[j] = j < col ? lptr(S, m, j) : 0;
    // acc: [0]=f1 [1..2col]=p [2col+1]=nbreak [2col+2]=nfree_nb [2col+3]=notbnded
    //      [2col+4]=tmin [2col+5]=tmax; accumulated in scalars and the
    //      guarded, unrolled column arrays py/ps, packed after the loop
    const int K = col2 + 6;
    double f1a = 0.0, nbr = 0.0, nfr = 0.0, notb = 0.0, tmn = 1.0e308, tmx = 0.0;
    double py[SMILI_MAXM_DEV], ps[SMILI_MAXM_DEV];
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) py[j] = ps[j] = 0.0;
    for (int i = c.g->rank * blockDim.x + threadIdx.x; i < 2 * SMILI_NBUCKET; i += c.g->G * blockDim.x)
      ghist[i] = 0;
    for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
      const double neggi = -c.gv[i];
      int iw = c.iwh[i];
      double tl = 0.0;
      if (iw != 3 && iw != -1) {
        tl = c.x[i];  // x - l with l = 0 (nbd = 1)
        const bool xlower = tl <= 0.0;
        iw = 0;
        if (xlower) {
          if (neggi <= 0.0) iw = 1;
        } else {
          if (fabs(neggi) <= 0.0) iw = -3;
        }
        c.iwh[i] = (signed char)iw;
      }
      unsigned long long key = ~0ULL;
      if (iw != 0 && iw != -1) {
        c.d[i] = 0.0;
      } else {
        c.d[i] = neggi;
        f1a -= neggi * neggi;
#pragma unroll
        for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
          if (j < col) {
            py[j] += ld_wy(c, (size_t)pj[j] * n + i) * neggi;
            ps[j] += ld_ws(c, (size_t)pj[j] * n + i) * neggi;
          }
        }
        if (nonneg && neggi < 0.0) {
          const double tb = tl / (-neggi);
          nbr += 1.0;
          tmn = fmin(tmn, tb);
          tmx = fmax(tmx, tb);
          key = (unsigned long long)__double_as_longlong(tb);
        } else {
          nfr += 1.0;
          if (fabs(neggi) > 0.0) notb = 1.0;
        }
      }
      c.bkey[i] = key;
    }
    double acc[2 * SMILI_MAXM_DEV + 6];
    acc[0] = f1a;
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
      if (j < col) {
        acc[1 + j] = py[j];
        acc[1 + col + j] = ps[j];
      }
    }
    acc[col2 + 1] = nbr;
    acc[col2 + 2] = nfr;
    acc[col2 + 3] = notb;
    acc[col2 + 4] = tmn;
    acc[col2 + 5] = tmx;
    for (int k = threadIdx.x; k < K; k += blockDim.x)
      c.ops[k] = (k == col2 + 3 || k == col2 + 5) ? RED_MAX : (k == col2 + 4 ? RED_MIN : RED_SUM);
    __syncthreads();
    if (!lb_reduce(c, acc, K)) return -2;
    const double f1 = c.red[0];
    double p[2 * SMILI_MAXM_DEV];
    for (int j = 0; j < col2; ++j) p[j] = c.red[1 + j];
    const int nbreak = (int)c.red[col2 + 1];
    const int nfree_nb = (int)c.red[col2 + 2];
    const int bnded = c.red[col2 + 3] > 0.5 ? 0 : 1;
    const unsigned long long kmin = (unsigned long long)__double_as_longlong(c.red[col2 + 4]);
    const unsigned long long kmax = (unsigned long long)__double_as_longlong(c.red[col2 + 5]);
    if (S.theta != 1.0)
      for (int j = 0; j < col; ++j) p[col + j] *= S.theta;
    __syncthreads();
    if (nbreak == 0 && nfree_nb == 0) {
      for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) c.z[i] = c.x[i];
      if (threadIdx.x == 0 && c.g->rank == 0) c.lred[CR_MODE] = CM_XCP_IS_X;
    } else {
      if (nbreak > 0) {
        // bucket the breakpoints: histogram, then scatter in bucket order
        int shift = 0;
        while (shift < 63 && ((kmax - kmin) >> shift) >= (unsigned long long)SMILI_NBUCKET) ++shift;
        unsigned* lh = reinterpret_cast<unsigned*>(c.dyn);
        for (int i = threadIdx.x; i < SMILI_NBUCKET; i += blockDim.x) lh[i] = 0;
        __syncthreads();
        for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
          const unsigned long long k = c.bkey[i];
          if (k != ~0ULL) atomicAdd(&lh[bucket_of(k, kmin, shift)], 1u);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < SMILI_NBUCKET; i += blockDim.x)
          if (lh[i]) atomicAdd(&ghist[i], (int)lh[i]);
        if (!group_sync(*c.g)) return -2;
        // exclusive prefix of the bucket counts -> start offsets (in lh)
        for (int i = threadIdx.x; i < SMILI_NBUCKET; i += blockDim.x) lh[i] = (unsigned)((volatile int*)ghist)[i];
        __syncthreads();
        if (threadIdx.x < 32) {
          // warp 0: sequential chunks of 128 buckets per lane, then a warp scan
          const int per = SMILI_NBUCKET / 32;
          unsigned run = 0;
          for (int q = 0; q < per; ++q) run += lh[threadIdx.x * per + q];
          unsigned incl = run;
          for (int s2 = 1; s2 < 32; s2 <<= 1) {
            const unsigned o = __shfl_up_sync(0xffffffffu, incl, s2);
            if (threadIdx.x >= s2) incl += o;
          }
          unsigned acc2 = incl - run;
          for (int q = 0; q < per; ++q) {
            const unsigned v = lh[threadIdx.x * per + q];
            lh[threadIdx.x * per + q] = acc2;
            acc2 += v;
          }
        }
        __syncthreads();
        for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
          const unsigned long long k = c.bkey[i];
          if (k != ~0ULL) {
            const int b = bucket_of(k, kmin, shift);
            const int q = (int)lh[b] + atomicAdd(&ghist[SMILI_NBUCKET + b], 1);
            sbk[q] = k;
            sbi[q] = i;
          }
        }
        if (!group_sync(*c.g)) return -2;
      }
      if (c.g->rank == 0) cauchy_scan(c, f1, p, nbreak, bnded, sbk, sbi, ghist);
    }
  }
  if (!group_sync(*c.g)) return -2;
  // every CTA reads the leader's results
  const double* lr = c.lred;
  __shared__ double cr_s[CR_C + 2 * SMILI_MAXM_DEV];
  for (int k = threadIdx.x; k < CR_C + col2; k += blockDim.x) cr_s[k] = ((const volatile double*)lr)[k];
  __syncthreads();
  const int mode = (int)cr_s[CR_MODE];
  if (mode != CM_XCP_IS_X && cr_s[CR_INFO] != 0) return -1;
  // apply the GCP and run freev (lbfgsb.f:2241-2340)
  double acc[3] = {0, 0, 0};  // nfree, nenter, nleave
  const u128 bnd = ((u128)(unsigned long long)__double_as_longlong(cr_s[CR_BHI]) << 64) |
                   (u128)(unsigned long long)__double_as_longlong(cr_s[CR_BLO]);
  const double tsum = cr_s[CR_TSUM];
  const bool count_moves = S.iter > 0 && S.cnstnd;
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    if (mode == CM_BOUNDARY || mode == CM_NONE_FIXED) {
      const unsigned long long k = c.bkey[i];
      if (mode == CM_BOUNDARY && k != ~0ULL && comp_key(k, i) <= bnd) {
        c.z[i] = 0.0;  // lower bound (d < 0 at every breakpoint)
        c.iwh[i] = 1;
        c.d[i] = 0.0;
      } else {
        c.z[i] = c.x[i] + tsum * c.d[i];
      }
    }
    const int fnew = c.iwh[i] <= 0;
    const int fold_ = c.freef[i];
    if (count_moves) {
      if (fold_ && !fnew) acc[2] += 1;
      if (!fold_ && fnew) acc[1] += 1;
    }
    c.freef[i] = (unsigned char)fnew;
    acc[0] += fnew;
  }
  set_ops(c, 3, RED_SUM);
  if (!lb_reduce(c, acc, 3)) return -2;
  if (threadIdx.x == 0) {
    if (mode != CM_XCP_IS_X) {
      S.nseg = (int)cr_s[CR_NSEG];
      for (int j = 0; j < col2; ++j) S.wa[2 * m + j] = cr_s[CR_C + j];  // c
    }
    S.nfree = (int)c.red[0];
    S.nenter = (int)c.red[1];
    S.ileave = n + 1 - (int)c.red[2];
    S.wrk = (c.red[2] > 0) || (c.red[1] > 0) || S.updatd;
    S.nact = n - S.nfree;
  }
  __syncthreads();
  return 0;
}

// ---------------------------------------------------------------------------
// formk (lbfgsb.f:1848-2172) from Gram sums over the free/active sets
// ---------------------------------------------------------------------------
// One FP64 tensor-core product D = A B + D of an 8x4 by 4x8 tile
// (mma.sync m8n8k4 f64).  Lane l holds A[l/4][l%4], B[l%4][l/4] and
// D[l/4][2(l%4) + {0,1}].
__device__ __forceinline__ void dmma_884(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

template <typename SY>
__device__ int lb_formk(LbCtxT<SY>& c) {
  LbState& S = *c.S;
  const int m = c.m, n = c.n, col = S.col;
  // entries: Fyy (a<=b), Ass (a<=b), Fsy (a,b), Asy (a,b) over physical columns
  const int nsym = m * (m + 1) / 2;
  const int E = 2 * nsym + 2 * m * m;
  // The four masked Gram blocks W' diag(mask) W over this CTA's pixels on
  // the FP64 tensor cores: per 4 pixels, A = (masked column a at pixel k),
  // B = (column b at pixel k); lane (a = l/4, k = l%4) holds the same
  // element of both operands, so one load per matrix feeds both.
  //   Fyy = Y'FY, Fsy = S'FY (free pixels), Ass = S'AS, Asy = S'AY (active)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int ca = lane >> 2, pk = lane & 3;
  const bool cval = ca < m;  // m <= 6 < 8: one 8x8 tile per block
  const size_t colo = (size_t)(cval ? ca : 0) * n;
  double fyy[2] = {0.0, 0.0}, fsy[2] = {0.0, 0.0}, ass[2] = {0.0, 0.0}, asy[2] = {0.0, 0.0};
  const int nchunk = (c.hi - c.lo + 3) >> 2;
  constexpr int U = 4;  // chunks in flight per warp
  for (int q0 = warp; q0 < nchunk; q0 += U * nw) {
    double y[U], sv[U];
    bool fr[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = c.lo + 4 * (q0 + u * nw) + pk;
      const bool ok = i < c.hi;  // q0 + u*nw < nchunk whenever i < hi
      y[u] = (ok && cval) ? ld_wy(c, colo + i) : 0.0;
      sv[u] = (ok && cval) ? ld_ws(c, colo + i) : 0.0;
      fr[u] = ok && c.freef[i] != 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const double yf = fr[u] ? y[u] : 0.0, sf = fr[u] ? sv[u] : 0.0, sa = fr[u] ? 0.0 : sv[u];
      dmma_884(fyy, yf, y[u]);
      dmma_884(fsy, sf, y[u]);
      dmma_884(ass, sa, sv[u]);
      dmma_884(asy, sa, y[u]);
    }
  }
  // combine the warps' tiles in fixed order: part[warp][tile][8x8]
  double* part = reinterpret_cast<double*>(c.dyn);
  {
    double* pw = part + (size_t)warp * 4 * 64 + ca * 8 + 2 * pk;
    pw[0] = fyy[0];
    pw[1] = fyy[1];
    pw[64] = fsy[0];
    pw[65] = fsy[1];
    pw[128] = ass[0];
    pw[129] = ass[1];
    pw[192] = asy[0];
    pw[193] = asy[1];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < E; e += blockDim.x) {
    int t, a, b;
    if (e < 2 * nsym) {  // triangular index -> (a, b), a <= b
      t = e < nsym ? 0 : 2;
      int r = e < nsym ? e : e - nsym;
      a = 0;
      while (r >= m - a) {
        r -= m - a;
        ++a;
      }
      b = a + r;
    } else {
      const int r = e - 2 * nsym;
      t = r < m * m ? 1 : 3;
      const int q = r < m * m ? r : r - m * m;
      a = q / m;
      b = q % m;
    }
    double sum = 0.0;
    for (int w = 0; w < nw; ++w) sum += part[(size_t)w * 256 + t * 64 + a * 8 + b];
    c.red[e] = sum;
  }
  for (int k = threadIdx.x; k < E; k += blockDim.x) c.ops[k] = RED_SUM;
  __syncthreads();
  if (!group_reduce(*c.g, c.red, c.ops, E)) return -9;
  int info = 0;
  if (threadIdx.x == 0) {
    auto sym = [&](int base, int a, int b) {  // symmetric block entry
      if (a > b) {
        const int t = a;
        a = b;
        b = t;
      }
      int e = 0;
      for (int q = 0; q < a; ++q) e += m - q;
      return c.red[base + e + (b - a)];
    };
    auto fyy = [&](int a, int b) { return sym(0, a, b); };
    auto ass = [&](int a, int b) { return sym(nsym, a, b); };
    auto fsy = [&](int a, int b) { return c.red[2 * nsym + a * m + b]; };
    auto asy = [&](int a, int b) { return c.red[2 * nsym + m * m + a * m + b]; };
    const int m2 = 2 * m;
#define WN(i, j) S.wn[((i)-1) + m2 * ((j)-1)]
#define SY(i, j) S.sy[((i)-1) + m * ((j)-1)]
    for (int iy = 1; iy <= col; ++iy) {
      const int is = col + iy;
      const int pi = lptr(S, m, iy - 1);
      for (int jy = 1; jy <= iy; ++jy) {
        const int js = col + jy;
        const int pjj = lptr(S, m, jy - 1);
        WN(jy, iy) = fyy(pi, pjj) / S.theta;
        WN(js, is) = ass(pi, pjj) * S.theta;
      }
      // wn1(m+iy, jy): active sum for iy > jy, free sum for iy <= jy
      for (int jy = 1; jy <= iy - 1; ++jy) WN(jy, is) = -asy(pi, lptr(S, m, jy - 1));
      for (int jy = iy; jy <= col; ++jy) WN(jy, is) = fsy(pi, lptr(S, m, jy - 1));
      WN(iy, iy) = WN(iy, iy) + SY(iy, iy);
    }
    if (d_chol_upper(S.wn, m2, col)) {
      info = -1;
    } else {
      const int col2 = 2 * col;
      for (int js = col + 1; js <= col2; ++js) d_tri_solve(S.wn, m2, col, &WN(1, js), true);
      for (int is = col + 1; is <= col2; ++is)
        for (int js = is; js <= col2; ++js) {
          double s = 0;
          for (int k = 1; k <= col; ++k) s += WN(k, is) * WN(k, js);
          WN(is, js) = WN(is, js) + s;
        }
      if (d_chol_upper(&WN(col + 1, col + 1), m2, col)) info = -2;
    }
#undef WN
#undef SY
    c.red[0] = info;
  }
  __syncthreads();
  info = (int)c.red[0];
  __syncthreads();
  return info;
}

// ---------------------------------------------------------------------------
// cmprlb + subsm (lbfgsb.f:1720-1786, 2991-3346).  Returns 0 or an error.
// ---------------------------------------------------------------------------
template <typename SY>
__device__ int lb_cmprlb_subsm(LbCtxT<SY>& c) {
  LbState& S = *c.S;
  const ProbDesc& P = *c.P;
  const int m = c.m, n = c.n, col = S.col, col2 = 2 * col;
  int pj[SMILI_MAXM_DEV];
#pragma unroll
  for (int j = 0; j < SMILI_MAXM_DEV; ++j) pj[j] = j < col ? lptr(S, m, j) : 0;
  __shared__ double a_s[2 * SMILI_MAXM_DEV], wv_s[2 * SMILI_MAXM_DEV];
  __shared__ int err_s;
  const bool unc = !S.cnstnd && col > 0;
  if (threadIdx.x == 0) {
    err_s = 0;
    if (!unc) {
      double a[2 * SMILI_MAXM_DEV];
      if (d_bmv(S, m, col, S.wa + 2 * m, a)) err_s = -8;
      for (int j = 0; j < col2; ++j) a_s[j] = a[j];
    }
  }
  __syncthreads();
  if (err_s) return err_s;
  const double theta = S.theta;
  double ay[SMILI_MAXM_DEV], as[SMILI_MAXM_DEV];
#pragma unroll
  for (int j = 0; j < SMILI_MAXM_DEV; ++j) ay[j] = as[j] = 0.0;
  // the free flag of the next element is fetched one iteration ahead, so
  // the loads of an element wait for nothing but themselves
  const int bd = blockDim.x;
  int i = c.lo + threadIdx.x;
  bool f_next = i < c.hi && (unc || c.freef[i]);
  for (; i < c.hi; i += bd) {
    const bool fr = f_next;
    f_next = i + bd < c.hi && (unc || c.freef[i + bd]);
    if (!fr) continue;
    // the row of W at pixel i, loaded once for r_i and for W'Z r
    double wyv[SMILI_MAXM_DEV], wsv[SMILI_MAXM_DEV];
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
      wyv[j] = j < col ? ld_wy(c, (size_t)pj[j] * n + i) : 0.0;
      wsv[j] = j < col ? ld_ws(c, (size_t)pj[j] * n + i) : 0.0;
    }
    double ri;
    if (unc) {
      ri = -c.gv[i];
    } else {
      ri = -theta * (c.z[i] - c.x[i]) - c.gv[i];
#pragma unroll
      for (int j = 0; j < SMILI_MAXM_DEV; ++j)
        if (j < col) ri += wyv[j] * a_s[j] + wsv[j] * (theta * a_s[col + j]);
    }
    c.r[i] = ri;
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
      if (j < col) {
        ay[j] += wyv[j] * ri;
        as[j] += wsv[j] * ri;
      }
    }
  }
  double acc[2 * SMILI_MAXM_DEV];
#pragma unroll
  for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
    if (j < col) {
      acc[j] = ay[j];
      acc[col + j] = as[j];
    }
  }
  set_ops(c, col2, RED_SUM);
  if (!lb_reduce(c, acc, col2)) return -9;
  if (threadIdx.x == 0) {
    double wv[2 * SMILI_MAXM_DEV];
    for (int j = 0; j < col; ++j) {
      wv[j] = c.red[j];
      wv[col + j] = theta * c.red[col + j];
    }
    const int m2 = 2 * m;
    if (d_tri_solve(S.wn, m2, col2, wv, true)) {
      err_s = -1;
    } else {
      for (int j = 0; j < col; ++j) wv[j] = -wv[j];
      if (d_tri_solve(S.wn, m2, col2, wv, false)) err_s = -1;
    }
    for (int j = 0; j < col2; ++j) wv_s[j] = wv[j];
  }
  __syncthreads();
  if (err_s) return err_s;
  // d := (d + W wv) / theta on the free set, then project z + d
  double acc2[2] = {0.0, 0.0};  // iword (max), dd_p (sum)
  double wq[SMILI_MAXM_DEV], wr[SMILI_MAXM_DEV];
#pragma unroll
  for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
    wq[j] = j < col ? wv_s[j] : 0.0;
    wr[j] = j < col ? wv_s[col + j] : 0.0;
  }
  const double rtheta = 1.0 / theta;
  // one pass: d, the projected z and the directional derivative (z - x).g;
  // all loads of an element before its stores (which may alias them for the
  // compiler), the free flag one element ahead
  i = c.lo + threadIdx.x;
  f_next = i < c.hi && (unc || c.freef[i]);
  for (; i < c.hi; i += bd) {
    const bool fr = f_next;
    f_next = i + bd < c.hi && (unc || c.freef[i + bd]);
    const double zi = c.z[i], xv = c.x[i], gvi = c.gv[i];
    double ri = fr ? c.r[i] : 0.0;
    SY wyr[SMILI_MAXM_DEV], wsr[SMILI_MAXM_DEV];
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
      wyr[j] = (fr && j < col) ? c.wy[(size_t)pj[j] * n + i] : (SY)0;
      wsr[j] = (fr && j < col) ? c.ws[(size_t)pj[j] * n + i] : (SY)0;
    }
    c.xp[i] = zi;
    double zn = zi;
    if (fr) {
#pragma unroll
      for (int j = 0; j < SMILI_MAXM_DEV; ++j)
        if (j < col) ri += (double)wyr[j] * wq[j] / theta + (double)wsr[j] * wr[j];
      ri *= rtheta;
      c.r[i] = ri;
      if (P.nonneg) {
        zn = fmax(0.0, zi + ri);
        if (zn == 0.0) acc2[0] = 1.0;
      } else {
        zn = zi + ri;
      }
      c.z[i] = zn;
    }
    acc2[1] += (zn - xv) * gvi;
  }
  if (threadIdx.x == 0) {
    c.ops[0] = RED_MAX;
    c.ops[1] = RED_SUM;
  }
  __syncthreads();
  if (!lb_reduce(c, acc2, 2)) return -9;
  const int iword = c.red[0] > 0.5;
  const double dd_p = c.red[1];
  if (threadIdx.x == 0) S.iword = iword;
  __syncthreads();
  if (!iword || dd_p <= 0.0) return 0;
  // backtrack: z = xp, alpha = largest feasible step along d (lbfgsb.f:3270-3330)
  double acc3[1] = {1.0};
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    c.z[i] = c.xp[i];
    if ((c.freef[i] || unc) && P.nonneg) {
      const double dk = c.r[i];
      if (dk < 0.0) {
        const double t2 = -c.z[i];
        acc3[0] = fmin(acc3[0], t2 >= 0.0 ? 0.0 : t2 / dk);
      }
    }
  }
  set_ops(c, 1, RED_MIN);
  if (!lb_reduce(c, acc3, 1)) return -9;
  const double alpha = c.red[0];
  __syncthreads();
  double acc4[1] = {(double)n};
  if (alpha < 1.0) {
    for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
      if ((c.freef[i] || unc) && P.nonneg && c.r[i] < 0.0) {
        const double t2 = -c.z[i];
        const double v = t2 >= 0.0 ? 0.0 : t2 / c.r[i];
        if (v == alpha) acc4[0] = fmin(acc4[0], (double)i);
      }
    }
    set_ops(c, 1, RED_MIN);
    if (!lb_reduce(c, acc4, 1)) return -9;
  }
  const int ibd = alpha < 1.0 ? (int)c.red[0] : -1;
  __syncthreads();
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    if (c.freef[i] || unc) {
      if (i == ibd) {
        c.z[i] = 0.0;
        c.r[i] = 0.0;
      }
      c.z[i] += alpha * c.r[i];
    }
  }
  __syncthreads();
  return 0;
}

// ---------------------------------------------------------------------------
// mainlb control flow (lbfgsb.f:287-1003) between function evaluations
// ---------------------------------------------------------------------------
enum { LB_RET_DONE = 0, LB_RET_FG = 1, LB_RET_RESTART = 2, LB_RET_ABORT = -9 };

template <typename SY>
__device__ int lb_abort(LbCtxT<SY>& c) {
  if (threadIdx.x == 0) {
    c.S->error = 1;
    c.S->task = LB_TASK_ERROR;
    c.S->done = 1;
  }
  __syncthreads();
  return LB_RET_DONE;
}

// x = t + stp d, or z when stp == 1 (lnsrlb, lbfgsb.f:2562-2570)
template <typename SY>
__device__ void lb_set_trial_x(LbCtxT<SY>& c) {
  const double stp = c.S->stp;
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x)
    c.x[i] = (stp == 1.0) ? c.z[i] : stp * c.d[i] + c.t[i];
  __syncthreads();
}

// "info /= 0 or iback >= 20" branch of mainlb (lbfgsb.f:888-920)
template <typename SY>
__device__ int lb_ls_fail(LbCtxT<SY>& c) {
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    c.x[i] = c.t[i];
    c.gv[i] = c.r[i];
  }
  __shared__ int res_s;
  if (threadIdx.x == 0) {
    LbState& S = *c.S;
    S.f = S.fold;
    if (S.col == 0) {
      if (S.info == 0) {
        S.info = -9;
        S.nfgv--;
        S.ifun--;
        S.iback--;
      }
      S.task = LB_TASK_ABNORMAL;
      S.iter++;
      S.done = 1;
      res_s = LB_RET_DONE;
    } else {
      if (S.info == 0) S.nfgv--;
      reset_memory(S);
      res_s = LB_RET_RESTART;
    }
  }
  __syncthreads();
  const int r = res_s;
  __syncthreads();
  return r;
}

// label 555 + the first part of lnsrlb (lbfgsb.f:2480-2575)
template <typename SY>
__device__ int lb_lnsrch_start(LbCtxT<SY>& c) {
  LbState& S = *c.S;
  const bool bounded_steps = S.cnstnd && S.iter > 0;
  double acc[3] = {0.0, 1.0e10, 0.0};  // dtd, stpmx (min), gd
  for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
    const double di = c.z[i] - c.x[i];
    const double xi = c.x[i], gi = c.gv[i];
    c.d[i] = di;
    c.t[i] = xi;
    c.r[i] = gi;
    acc[0] += di * di;
    acc[2] += gi * di;
    if (bounded_steps && c.P->nonneg && di < 0.0) {
      const double a2 = -xi;  // l - x with l = 0
      acc[1] = fmin(acc[1], a2 >= 0.0 ? 0.0 : a2 / di);
    }
  }
  if (threadIdx.x == 0) {
    c.ops[0] = RED_SUM;
    c.ops[1] = RED_MIN;
    c.ops[2] = RED_SUM;
  }
  __syncthreads();
  if (!lb_reduce(c, acc, 3)) return LB_RET_ABORT;
  __shared__ int act_s;
  if (threadIdx.x == 0) {
    S.dtd = c.red[0];
    S.dnorm = sqrt(S.dtd);
    S.stpmx = 1.0e10;
    if (S.cnstnd) S.stpmx = (S.iter == 0) ? 1.0 : c.red[1];
    S.stp = (S.iter == 0 && !S.boxed) ? fmin(1.0 / S.dnorm, S.stpmx) : 1.0;
    S.fold = S.f;
    S.ifun = 0;
    S.iback = 0;
    S.csave = CS_START;
    S.gd = c.red[2];
    S.gdold = S.gd;
    if (S.gd >= 0.0) {
      S.info = -4;  // ascent direction in projection
      act_s = 0;
    } else {
      d_dcsrch(S, S.f, S.gd, 0.0, S.stpmx);
      S.xstep = S.stp * S.dnorm;
      S.ifun++;
      S.nfgv++;
      S.iback = S.ifun - 1;
      act_s = 1;
    }
  }
  __syncthreads();
  const int act = act_s;
  __syncthreads();
  if (!act) {
    const int r = lb_ls_fail(c);
    return r == LB_RET_RESTART ? LB_RET_RESTART : LB_RET_DONE;
  }
  lb_set_trial_x(c);
  if (threadIdx.x == 0) S.task = LB_TASK_FG_LN;
  __syncthreads();
  return LB_RET_FG;
}

// label 222 onwards: Cauchy point, subspace minimisation, line-search start
template <typename SY>
__device__ int lb_iter(LbCtxT<SY>& c) {
  LbState& S = *c.S;
  for (int guard = 0; guard < 4; ++guard) {
    if (threadIdx.x == 0) S.iword = -1;
    __syncthreads();
    if (!S.cnstnd && S.col > 0) {
      for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) c.z[i] = c.x[i];
      if (threadIdx.x == 0) {
        S.wrk = S.updatd;
        S.nseg = 0;
      }
      __syncthreads();
    } else {
      c.prof->mark(PR_LB_POST);
      const int rc = lb_cauchy(c);
      c.prof->mark(PR_CAUCHY);
      if (rc == -2) return lb_abort(c);
      if (rc != 0) {
        if (threadIdx.x == 0) reset_memory(S);
        __syncthreads();
        continue;
      }
      if (threadIdx.x == 0) S.nintol += S.nseg;
      __syncthreads();
    }
    if (S.nfree != 0 && S.col != 0) {
      if (S.wrk) {
        c.prof->mark(PR_LB_POST);
        const int rc = lb_formk(c);
        c.prof->mark(PR_FORMK);
        if (rc == -9) return lb_abort(c);
        if (rc != 0) {
          if (threadIdx.x == 0) reset_memory(S);
          __syncthreads();
          continue;
        }
      }
      c.prof->mark(PR_LB_POST);
      const int rc = lb_cmprlb_subsm(c);
      c.prof->mark(PR_SUBSM);
      if (rc == -9) return lb_abort(c);
      if (rc != 0) {
        if (threadIdx.x == 0) reset_memory(S);
        __syncthreads();
        continue;
      }
    }
    c.prof->mark(PR_LB_POST);
    const int r = lb_lnsrch_start(c);
    c.prof->mark(PR_LNSRCH);
    if (r == LB_RET_ABORT) return lb_abort(c);
    if (r == LB_RET_RESTART) continue;
    return r;
  }
  return lb_abort(c);  // repeated restarts: not reachable with an empty memory
}

// Called after every function/gradient evaluation with the group-reduced
// f, g.d and projected-gradient norm.  Returns LB_RET_FG when x holds the next
// point to evaluate, LB_RET_DONE when the solve is over.
template <typename SY>
__device__ int lb_after_fg(LbCtxT<SY>& c, double f, double gd_fg, double sbg) {
  LbState& S = *c.S;
  const ProbDesc& P = *c.P;
  const int m = c.m;
  __shared__ int act_s;
  if (threadIdx.x == 0) {
    S.f = f;
    S.nfg_total++;
  }
  __syncthreads();
  if (S.task == LB_TASK_FG_START) {
    if (threadIdx.x == 0) {
      S.nfgv = 1;
      S.sbgnrm = sbg;
      if (S.sbgnrm <= P.pgtol) {
        S.task = LB_TASK_CONV;
        S.done = 1;
      }
    }
    __syncthreads();
    if (S.done) return LB_RET_DONE;
    return lb_iter(c);
  }
  // FG_LN: lnsrlb from label 556
  if (threadIdx.x == 0) {
    S.gd = gd_fg;
    d_dcsrch(S, S.f, S.gd, 0.0, S.stpmx);
    S.xstep = S.stp * S.dnorm;
    if (S.csave != CS_CONV && S.csave != CS_WARN) {
      S.ifun++;
      S.nfgv++;
      S.iback = S.ifun - 1;
      act_s = (S.iback >= 20) ? 2 : 1;
    } else {
      act_s = 0;
    }
  }
  __syncthreads();
  const int act = act_s;
  __syncthreads();
  if (act == 1) {
    lb_set_trial_x(c);
    return LB_RET_FG;
  }
  if (act == 2) {
    const int r = lb_ls_fail(c);
    return r == LB_RET_RESTART ? lb_iter(c) : LB_RET_DONE;
  }
  // NEW_X: iteration finished (lbfgsb.f:931-944), driver test, label 777
  if (threadIdx.x == 0) {
    S.iter++;
    S.sbgnrm = sbg;
    if (c.g->rank == 0 && S.iter - 1 < P.niter + 2) c.trace[S.iter - 1] = S.f;
    if (S.f <= P.ftarget) {
      S.task = LB_TASK_TARGET;  // requested objective reached (no reference counterpart)
      S.done = 1;
    } else if (S.iter > P.niter) {
      S.task = LB_TASK_STOP;  // fftim2d.f90:324-325
      S.done = 1;
    } else if (S.sbgnrm <= P.pgtol) {
      S.task = LB_TASK_CONV;
      S.done = 1;
    } else {
      const double ddum = fmax(fabs(S.fold), fmax(fabs(S.f), 1.0));
      if ((S.fold - S.f) <= S.tol * ddum) {
        S.task = LB_TASK_CONV;
        S.done = 1;
      }
    }
    if (!S.done) {
      double dr, dd;
      if (S.stp == 1.0) {
        dr = S.gd - S.gdold;
        dd = -S.gdold;
      } else {
        dr = (S.gd - S.gdold) * S.stp;
        dd = -S.gdold * S.stp;
      }
      S.wa[0] = dr;  // keep dr for matupd below
      if (dr <= S.epsmch * dd) {
        S.nskip++;
        S.updatd = 0;
        act_s = 0;
      } else {
        S.updatd = 1;
        S.iupdat++;
        if (S.iupdat <= m) {
          S.col = S.iupdat;
          S.itail = (S.head + S.iupdat - 2) % m + 1;
        } else {
          S.itail = S.itail % m + 1;
          S.head = S.head % m + 1;
        }
        act_s = 1;
      }
    }
  }
  __syncthreads();
  if (S.done) return LB_RET_DONE;
  if (act_s) {
    // matupd (lbfgsb.f:2584-2670) fused with r = g - r, d = stp d and rr
    const int n = c.n, itail = S.itail - 1;
    const double sc = (S.stp == 1.0) ? 1.0 : S.stp;
    const int K = 1 + 2 * m;
    // per-column partial sums in registers: the column loops are unrolled
    // to the largest memory with a guard, so no array is indexed at run time
    double rr_acc = 0.0, ay[SMILI_MAXM_DEV], as[SMILI_MAXM_DEV];
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) ay[j] = as[j] = 0.0;
    for (int i = c.lo + threadIdx.x; i < c.hi; i += blockDim.x) {
      const double ri = c.gv[i] - c.r[i];
      const double di = c.d[i] * sc;
      rr_acc += ri * ri;
#pragma unroll
      for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
        if (j < m) {
          ay[j] += di * ld_wy(c, (size_t)j * n + i);
          as[j] += ld_ws(c, (size_t)j * n + i) * di;
        }
      }
      st_sy(c, (size_t)itail * n + i, di, ri);
      c.r[i] = ri;
      c.d[i] = di;
    }
    double acc[1 + 2 * SMILI_MAXM_DEV];
    acc[0] = rr_acc;
#pragma unroll
    for (int j = 0; j < SMILI_MAXM_DEV; ++j) {
      if (j < m) {
        acc[1 + j] = ay[j];
        acc[1 + m + j] = as[j];
      }
    }
    set_ops(c, K, RED_SUM);
    if (!lb_reduce(c, acc, K)) return lb_abort(c);
    if (threadIdx.x == 0) {
      const double rr = c.red[0], dr = S.wa[0];
      const int col = S.col;
#define SY(i, j) S.sy[((i)-1) + m * ((j)-1)]
#define SS(i, j) S.ss[((i)-1) + m * ((j)-1)]
      S.theta = rr / dr;
      if (S.iupdat > m) {
        for (int j = 1; j <= col - 1; ++j) {
          for (int k = 0; k < j; ++k) SS(1 + k, j) = SS(2 + k, j + 1);
          for (int k = 0; k < col - j; ++k) SY(j + k, j) = SY(j + 1 + k, j + 1);
        }
      }
      int pointr = S.head;
      for (int j = 1; j <= col - 1; ++j) {
        SY(col, j) = c.red[1 + (pointr - 1)];
        SS(j, col) = c.red[1 + m + (pointr - 1)];
        pointr = pointr % m + 1;
      }
      SS(col, col) = (S.stp == 1.0) ? S.dtd : S.stp * S.stp * S.dtd;
      SY(col, col) = dr;
#undef SY
#undef SS
      if (d_formt(S, m) != 0) reset_memory(S);
    }
    __syncthreads();
  }
  return lb_iter(c);
}
