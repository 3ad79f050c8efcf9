// Device-side layout of one imaging problem and of its L-BFGS-B state.
//
// Shared by the host packer (host.cu) and the kernels.  Every problem of a
// batch lives in one device arena; ProbDesc holds the byte offsets of its
// arrays inside that arena plus the scalars the kernels need.  All offsets
// are multiples of 256 bytes.
#pragma once
#include <stdint.h>

#define SMILI_MAXM 8          // largest L-BFGS-B memory supported on the device
#define SMILI_MAXW 16         // largest ES kernel width
#define SMILI_NTERMS 15       // chisq, chisqfcv, chisqamp, chisqcp, chisqca, reg, l1..sm, cost
#define SMILI_NTERMS3D 20     // a movie: ..., reg, l1, sm, tv, tsv, kl, gs, tfd, lc, cen, rt, ri, rs, rf, cost
#define SMILI_NPART 16        // partial sums produced by one FG evaluation

// data-term kinds in the flattened datum index space
enum { KIND_FCV = 0, KIND_AMP = 1, KIND_CP = 2, KIND_CA = 3 };

// L-BFGS-B driver states (what the last advance asked for)
enum {
  LB_TASK_FG_START = 1,   // evaluate f, g at the projected initial x
  LB_TASK_FG_LN = 2,      // evaluate f, g at a line-search trial point
  LB_TASK_CONV = 3,       // converged (pgtol or factr test)
  LB_TASK_ABNORMAL = 4,   // line search failed with an empty memory
  LB_TASK_STOP = 5,       // iteration limit reached (iter > niter)
  LB_TASK_ERROR = 6,      // invalid input or a device-side wait timed out
  LB_TASK_FG_ONLY = 7,    // single evaluation, no optimisation
  LB_TASK_TARGET = 8      // reached the requested objective value
};

struct ProbDesc {
  // sizes
  int npix, nx, ny, nuv;
  int nf1, nf2;            // fine grid
  int w;                   // ES kernel width
  int b1s, b1n, b2s, b2n;  // band of fine-grid cells touched by the uv points
  int nfcv, namp, ncp, nca;
  int nslot;               // uv references of the data (slots): nfcv + namp + 3 ncp + 4 nca
  int ndata;               // nfcv + namp + ncp + nca
  int nonneg, m, niter, prec64;
  int has_l1, has_tv, has_tsv, has_kl, has_gs, has_tfd, has_cen, has_sm;
  int windowed;            // 1 when the pixel set is not the full nx*ny grid
  int ident;               // 1 when pixel p is grid cell (p % nx, p / nx): the full grid in
                           // row-major order, so x is its own dense image grid
  int nitems;              // spreading work items (<= 128 points of one bin x bin tile)
  int bin;                 // spreading bin side in fine-grid cells (8 or 16)
  int dft;                 // 1: the four band passes as dense products with the
                           // twiddle matrices o_ex / o_ey instead of FFTs
  // movies (dynamic imaging): nframes >= 1 on a movie's descriptor (0 for a
  // 2D problem), whose vectors hold npix = frame_npix * nframes values; each
  // frame is a 2D descriptor (o_frames) whose x / g / d point into them
  int nframes, frame_npix;
  int has_rt, has_ri, has_lc;
  // scalars
  double beta;
  double wfcv, wamp, wcp, wca;       // normalised data weights (w / wtotal)
  double l1_l, tv_l, tsv_l, kl_l, gs_l, tfd_l, tfd_tgtfd, cen_l, cen_alpha;
  // per-pixel regularizer weights that are one value over the whole image
  // (flat priors): bit 0..4 of wuni for l1, tv, tsv, kl, gs, value in wu[]
  int wuni;
  double wu[5];
  double sm_l, sm_maj, sm_min, sm_phi;
  double nxref, nyref;
  double factr, pgtol;
  double rt_l, ri_l;
  double ftarget;          // stop once f <= ftarget at a completed iteration (-inf: off)
  // byte offsets in the arena (0 = absent)
  int64_t o_x0, o_xidx, o_yidx, o_inv;
  int64_t o_xg;                         // dense image grid [ny][nx] (double), written by F1
  int64_t o_ex, o_ey;                   // twiddle matrices [b1n][nx], [b2n][ny] (cpx<R>) when dft
  int64_t o_l1w, o_tvw, o_tsvw, o_klw, o_gsw;
  int64_t o_dc1, o_dc2, o_tw1, o_tw2;   // deconvolution factors, twiddle tables
  int64_t o_u, o_v;                     // fine-grid coordinates xi = u n / 2pi (R)
  int64_t o_dre, o_dim, o_dvar;         // per datum: value(s) and variance (R)
  int64_t o_didx;                       // per slot: 0-based uv index (sorted order)
  int64_t o_dsgn;                       // per slot: sign (+1 / -1) as int8
  int64_t o_items;                      // int4 work items: start, end, row0, col0
  int64_t o_tmpA, o_bandA, o_V, o_contrib, o_bandC, o_tmpC, o_gchi;  // o_contrib: per uv point, the
                                                                      // sum of the chi-square derivatives
  int64_t o_part;                       // FG partial sums [npart_ctas][SMILI_NPART] (double)
  // optimiser (double precision)
  int64_t o_x, o_g, o_z, o_r, o_d, o_t, o_xp, o_ws, o_wy, o_iwh, o_free, o_bkey;
  int64_t o_sbk, o_sbi, o_hist;         // bucketed breakpoints, bucket counts/cursors
  int64_t o_cand, o_lred, o_state;
  int64_t o_trace;                      // cost at each NEW_X (double[niter+2])
  int64_t o_model;                      // per datum: model re, im, residual re, im (double), or 0
  int64_t o_frames;                     // movie: ProbDesc[nframes]
  int64_t o_rtw, o_riw, o_lcf, o_iavg;  // movie: Rt / Ri weights, light curve, pixel average
  int64_t o_out;                        // results: terms[15], counters
};

// every arena offset of ProbDesc, for code that moves a problem's region
#define SMILI_PROB_OFFSETS(X)                                                                          \
  X(o_x0) X(o_xidx) X(o_yidx) X(o_inv) X(o_xg) X(o_ex) X(o_ey) X(o_l1w) X(o_tvw) X(o_tsvw) X(o_klw)  \
  X(o_gsw) X(o_dc1) X(o_dc2) X(o_tw1) X(o_tw2) X(o_u) X(o_v) X(o_dre) X(o_dim) X(o_dvar) X(o_didx)   \
  X(o_dsgn) X(o_items) X(o_tmpA) X(o_bandA) X(o_V) X(o_contrib) X(o_bandC) \
  X(o_tmpC) X(o_gchi) X(o_part) X(o_x) X(o_g) X(o_z) X(o_r) X(o_d) X(o_t) X(o_xp) X(o_ws) X(o_wy)     \
  X(o_iwh) X(o_free) X(o_bkey) X(o_sbk) X(o_sbi) X(o_hist) X(o_cand) X(o_lred) X(o_state) X(o_trace) \
  X(o_model) X(o_frames) X(o_rtw) X(o_riw) X(o_lcf) X(o_iavg) X(o_out)

// Scalar L-BFGS-B state (setulb's isave/dsave/lsave plus the small matrices).
struct LbState {
  int task, done, error;
  int col, head, itail, iupdat, iter, nfgv, ifun, iback, nseg, nskip, nintol, info, iword;
  int nfree, nact, ileave, nenter;
  int updatd, wrk, cnstnd, boxed, prjctd;
  int stage, brackt, csave;
  int nfg_total;
  double f, theta, fold, tol, dnorm, gd, gdold, stp, stpmx, sbgnrm, dtd, xstep, epsmch;
  double ginit, gtest, gx, gy, finit, fx, fy, stx, sty, stmin, stmax, width, width1;
  double terms[SMILI_NTERMS3D];
  double sy[SMILI_MAXM * SMILI_MAXM], ss[SMILI_MAXM * SMILI_MAXM], wt[SMILI_MAXM * SMILI_MAXM];
  double wn[4 * SMILI_MAXM * SMILI_MAXM], wn1[4 * SMILI_MAXM * SMILI_MAXM];
  double wa[8 * SMILI_MAXM];
};

// per-problem results copied back to the host
struct ProbResult {
  double terms[SMILI_NTERMS3D];
  int task, iter, nfg, error;
};
