/* smili_b200: C ABI of the B200 static-imaging solver (libsmili_b200.so).
 *
 * Replaces the native core that SMILI reaches through its f2py module
 * `fortlib` (built from src/fortlib/*.f90 by src/fortlib/makefile.in:135-136):
 * the objective/gradient evaluation calc_cost (src/fortlib/fftim2d.f90:387)
 * and the L-BFGS-B driver fftim2d.imaging (src/fortlib/fftim2d.f90:11-382),
 * including the FINUFFT transforms it calls (src/wrapfinufft/wrapfinufft.f90).
 *
 * All entry points return SMILI_OK (0) or a negative error code; the text of
 * the last error of the calling thread is available from smili_last_error().
 * Device memory is allocated and owned by the library; callers pass host
 * pointers only.  Arrays use the Fortran layouts of the reference: image
 * vectors of Npix pixels with 1-based xidx/yidx, uvidxcp as (3,Ncp) and
 * uvidxca as (4,Nca) column-major (the indices of one datum contiguous).
 */
#ifndef SMILI_B200_H
#define SMILI_B200_H
#ifdef __cplusplus
extern "C" {
#endif

#define SMILI_OK 0
#define SMILI_ERR_ARG (-1)         /* invalid size, index or option */
#define SMILI_ERR_DATA (-2)        /* non-finite value or non-positive variance */
#define SMILI_ERR_CUDA (-3)        /* CUDA runtime failure */
#define SMILI_ERR_NODEV (-4)       /* no usable CUDA device */
#define SMILI_ERR_TIMEOUT (-5)     /* a device-side wait gave up (solve aborted) */
#define SMILI_ERR_UNSUPPORTED (-6) /* e.g. L-BFGS-B memory m > 6 */
#define SMILI_ERR_HOST (-7)        /* host-side failure, e.g. out of host memory */

/* Solver task codes reported in smili_solve_info.task */
#define SMILI_TASK_CONV 3      /* CONVERGENCE: pgtol or factr test */
#define SMILI_TASK_ABNORMAL 4  /* ABNORMAL_TERMINATION_IN_LNSRCH */
#define SMILI_TASK_STOP 5      /* STOP: TOTAL ITERATION NUMBER EXCEEDS LIMIT */
#define SMILI_TASK_ERROR 6
#define SMILI_TASK_TARGET 8    /* reached the target set by smili_batch_set_targets */

/* The arguments of fortlib.fftim2d.imaging / calc_cost
 * (src/fortlib/fftim2d.f90:11-34, smili/imaging/lbfgs.py:492-564). */
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
} smili_imaging_args;

/* Options that have no counterpart in the reference's signature. */
typedef struct {
  int precision;        /* 64 (default, FP64 throughout) or 32 (FP32 transforms,
                           compensated FP32 chi-square sums, FP64 optimiser) */
  double nufft_eps;     /* NUFFT tolerance; 0 -> 1e-6 (the reference's ffteps) */
  int ctas_per_problem; /* 0 -> automatic */
  int device;           /* CUDA device ordinal */
  void* stream;         /* cudaStream_t, NULL -> the library's own stream */
  int spread_bin;       /* spreading tile side in fine-grid cells: 8 or 16; 0 -> 8.  A
                           16-cell tile whose subgrids do not fit in shared memory
                           falls back to 8 */
  int transform;        /* fine-grid passes of the NUFFT: 0 -> automatic, 1 -> FFTs,
                           2 -> dense products with the twiddle matrices (used only
                           where the data's band is at most 64 x 64 fine-grid cells;
                           otherwise FFTs) */
} smili_options;

typedef struct {
  int task;   /* SMILI_TASK_* */
  int niter;  /* L-BFGS-B iterations completed (isave(30)) */
  int nfg;    /* function/gradient evaluations, including the final summary */
  int error;  /* nonzero when the solve was aborted */
} smili_solve_info;

/* terms[15] = chisq, chisqfcv, chisqamp, chisqcp, chisqca, reg, l1_cost,
 * tv_cost, tsv_cost, kl_cost, gs_cost, tfd_cost, cen_cost, sm_cost, cost
 * (the intent(out) scalars of fftim2d.imaging, fftim2d.f90:29-32). */

/* fortlib.fftim2d.imaging (fftim2d.f90:11-382): L-BFGS-B with m, factr,
 * pgtol from smili/imaging/lbfgs.py:34-38, stopped after niter+1 iterations
 * like fftim2d.f90:324.  Writes Iout[npix] and the final cost terms. */
int smili_fftim2d_imaging(const smili_imaging_args* a, int niter, int nonneg, int nprint, int m,
                          double factr, double pgtol, const smili_options* opt, double* iout,
                          double* terms, smili_solve_info* info);

/* calc_cost (fftim2d.f90:387-607): cost terms and gradient at image x. */
int smili_calc_cost(const smili_imaging_args* a, const double* x, const smili_options* opt,
                    double* terms, double* grad);

/* Batched solves: many independent problems (different image sizes, data and
 * weights) in one persistent launch.  No reference counterpart: the reference
 * solves one problem per call of fftim2d.imaging. */
typedef struct smili_batch smili_batch;
int smili_batch_create(int nprob, const smili_imaging_args* const* probs, const int* niter,
                       int nonneg, int m, double factr, double pgtol, const smili_options* opt,
                       smili_batch** out);
/* Solve (fg_only = 0) or evaluate calc_cost once (fg_only = 1) for every
 * problem on the device; fg_only = 2 only times 1000 group barriers (a
 * diagnostic); fg_only = 3 checks the bounded waits: one CTA of every group
 * skips a group barrier, the others give up after about 10 ms and the call
 * returns SMILI_ERR_TIMEOUT (with one CTA per problem there is no group
 * barrier to miss and it returns SMILI_OK).  The batch stays usable.
 * kernel_ms (optional) receives the device time of the launch. */
int smili_batch_run(smili_batch* b, int fg_only, float* kernel_ms);
int smili_batch_fetch(smili_batch* b, int p, double* iout, double* terms, double* grad,
                      smili_solve_info* info);
/* Per-problem objective targets (no reference counterpart): a solve stops
 * with SMILI_TASK_TARGET at the first completed iteration whose cost is
 * <= ftarget[p]; niter stays the iteration cap.  NULL clears the targets. */
int smili_batch_set_targets(smili_batch* b, const double* ftarget);

/* Replace problem p's start image (no reference counterpart): the npix
 * pixel values x (in the kwargs' scaled units) become the initial image of
 * the next smili_batch_run, as `iin` at packing did.  Lets a caller restart
 * a device-resident batch from new images (a warm start) without packing
 * and uploading its data again.  Movies are not supported. */
int smili_batch_set_start(smili_batch* b, int p, const double* x);

/* Change the iteration caps of the next runs (no reference counterpart):
 * niter[p] between 0 and the cap problem p was created with; NULL restores
 * those caps.  With smili_batch_set_start this lets one device-resident
 * batch run a few iterations, restart from new images and run the rest. */
int smili_batch_set_niter(smili_batch* b, const int* niter);

/* Device-side warm start (no reference counterpart), for a batch whose
 * problems are all nx x ny 2D images.  The three calls run on the batch's
 * stream and return once their work is done.
 *
 * smili_batch_images: every problem's current image (its pixel vector after
 * the last run) as a dense grid scaled to max 1: dst[p][iy][ix] =
 * x_p(ix, iy) / max x_p, zero at cells outside the problem's pixels (all
 * zero where max x_p <= 0).  dst: device memory on the batch's device,
 * nprob * ny * nx floats.
 *
 * smili_batch_set_starts_from_images: replaces every problem's start image.
 * For problem p the start is relu(img[p]) at its pixels, scaled so that it
 * sums to the total of its current image x_p; it is x_p itself where
 * keep[p] != 0, where relu(img[p]) has a non-finite cell or no positive one,
 * or where x_p sums to <= 0.  img: device memory, nprob * ny * nx floats,
 * complete before the call; keep: host array of nprob bytes, or NULL.
 *
 * smili_batch_reset_starts: puts back the start images the problems were
 * created with. */
int smili_batch_images(smili_batch* b, float* dst, int nx, int ny);
int smili_batch_set_starts_from_images(smili_batch* b, const float* img, int nx, int ny,
                                       const unsigned char* keep);
int smili_batch_reset_starts(smili_batch* b);
/* Cost recorded at each completed iteration of problem p (NaN where absent). */
int smili_batch_trace(smili_batch* b, int p, double* trace, int len);
void smili_batch_destroy(smili_batch* b);
/* Stage profiler (no reference counterpart): with enable != 0 the next runs
 * accumulate the device time of each solver stage of the first CTA group;
 * stage_ns (optional, len entries) receives the last accumulated values in
 * the order F1..F8 (transform and data stages), L-BFGS-B bookkeeping,
 * Cauchy point, formk, subspace minimisation, line-search start, set-up,
 * other, evaluation count. */
int smili_batch_profile(smili_batch* b, int enable, double* stage_ns, int len);

/* The arguments of fortlib.fftim3d.imaging / calc_cost (dynamic imaging,
 * src/fortlib/fftim3d.f90:11-44, smili/imaging/lbfgs3d.py:732-784): a movie
 * of nz frames of npix pixels each (iin frame-major), u/v the frames' uv
 * lists concatenated with nuvs[nz] points per frame (get_uvlist_loop), data
 * indices into that list.  Every closure quantity must lie within one frame.
 * Weights of the static regularizers have npix entries; lc_l / lc_tgtfd
 * have nz; rs / rf are accepted but, as in the reference, not evaluated. */
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
  double l1_l;  const double* l1_wgt;  int l1_nwgt;
  double sm_l, sm_maj, sm_min, sm_phi;
  double tv_l;  const double* tv_wgt;  int tv_nwgt;
  double tsv_l; const double* tsv_wgt; int tsv_nwgt;
  double kl_l;  const double* kl_wgt;  int kl_nwgt;
  double gs_l;  const double* gs_wgt;  int gs_nwgt;
  double tfd_l, tfd_tgtfd;
  const double* lc_l;
  const double* lc_tgtfd;
  int lc_nidx;
  double cen_l, cen_alpha;
  double rt_l; const double* rt_wgt; int rt_nwgt;
  double ri_l; const double* ri_wgt; int ri_nwgt;
  double rs_l; const double* rs_wgt; int rs_nwgt;
  double rf_l; const double* rf_wgt; int rf_nwgt;
  int isfcv, nfcv; const int* uvidxfcv; const double* vfcvr; const double* vfcvi; const double* varfcv; double wfcv;
  int isamp, namp; const int* uvidxamp; const double* vamp; const double* varamp; double wamp;
  int iscp, ncp;   const int* uvidxcp;  const double* cp;   const double* varcp;  double wcp;
  int isca, nca;   const int* uvidxca;  const double* ca;   const double* varca;  double wca;
  double inormfactr;
} smili_imaging3d_args;

/* terms3d[20] = chisq, chisqfcv, chisqamp, chisqcp, chisqca, reg, l1_cost,
 * sm_cost, tv_cost, tsv_cost, kl_cost, gs_cost, tfd_cost, lc_cost,
 * cen_cost, rt_cost, ri_cost, rs_cost, rf_cost, cost (fftim3d.f90:41-44). */

/* fortlib.fftim3d.imaging (fftim3d.f90:11-467): one L-BFGS-B solve over all
 * npix * nz values; Iout is thresholded at 1e-10 like fftim3d.f90:466. */
int smili_fftim3d_imaging(const smili_imaging3d_args* a, int niter, int nonneg, int nprint, int m,
                          double factr, double pgtol, const smili_options* opt, double* iout,
                          double* terms3d, smili_solve_info* info);

/* calc_cost of fftim3d (fftim3d.f90:473-614) at the movie vector x. */
int smili_calc_cost3d(const smili_imaging3d_args* a, const double* x, const smili_options* opt,
                      double* terms3d, double* grad);

/* model_fcv / model_amp / model_cp / model_ca (src/fortlib/fftlib.f90:744-1254):
 * exactly one data term of `a` is given (is* flags); regularizers are
 * ignored.  chisq = sum over that term of resid^2 / var (2 (1 - cos resid)
 * / var for closure phases), grad its gradient, and per datum the model and
 * residual: complex for fcv (shifted back to the reference pixel as
 * phashift_c2r does), real for amp / cp / ca (model_im, resid_im zero; cp
 * wrapped into (-pi, pi]).  The output arrays may be NULL. */
int smili_model_terms(const smili_imaging_args* a, const double* x, const smili_options* opt, double* chisq,
                      double* grad, double* model_re, double* model_im, double* resid_re, double* resid_im);

/* The non-redundant uv list of get_uvlist (smili/uvdata/uvtable/tools.py:
 * 12-132), computed on the GPU.  u, v: the n uv points of all data terms
 * stacked in the reference's order (fcv, amp, closure phases uv12 | uv23 |
 * uv31, closure amplitudes uv1 | uv2 | uv3 | uv4, each block contiguous).
 * A point with v < 0 counts as (-u, -v) with sign -1.  Out: *nuv distinct
 * folded points in u_out, v_out (capacity n) in the order np.unique gives
 * complex values (u, then v; -0 equals +0), each as first stacked; uvidx[n]
 * = sign * (1 + position of the point in that list), in stack order.
 * The library keeps a device work space per device between calls (about
 * 100 bytes per point, grown for larger lists); calls are serialised. */
int smili_get_uvlist(int n, const double* u, const double* v, const smili_options* opt, int* nuv,
                     double* u_out, double* v_out, int* uvidx);

/* NUFFTs of the imaging path with the reference's conventions (sign "+",
 * modes -N/2..(N-1)/2 at pixels 1..N): fortlib.fftlib.nufft_fwd_real
 * (type 2, fftlib.f90:86-100) and nufft_adj_real1d (type 1, real part,
 * fftlib.f90:118-133).  u, v already multiplied by 2*pi*dx, 2*pi*dy. */
int smili_nufft_fwd_real(int nuv, const double* u, const double* v, int nx, int ny,
                         const double* img, const smili_options* opt, double* vreal,
                         double* vimag);
int smili_nufft_adj_real1d(int nuv, const double* u, const double* v, const double* vreal,
                           const double* vimag, int nx, int ny, const smili_options* opt,
                           double* img);

/* Allocation-free calc_cost (no reference counterpart).  Same inputs,
 * outputs and results as smili_calc_cost (the same options: precision,
 * NUFFT tolerance, CTAs per problem, spreading tile, transform), for
 * callers that must not allocate device memory, e.g. a host whose device
 * memory is owned by another allocator or pool that leaves no room for
 * cudaMalloc.  Its device scratch is one static array of
 * SMILI_NOALLOC_SCRATCH_BYTES per device: problems that need more are
 * rejected with SMILI_ERR_ARG (use smili_calc_cost for those).  It calls no
 * CUDA allocator; host-side packing uses ordinary host memory.  Calls on
 * the same device share the scratch, so calls that overlap in time race.
 * The first call on a device does the set-up (cudaGetSymbolAddress and
 * kernel attributes), kept for the life of the process: a cudaDeviceReset
 * after it is not supported.  The call is synchronous (it waits for its
 * stream and reads the results back with blocking copies): do not make it
 * while any stream of the process is capturing.  Runs on opt->stream, or
 * the per-thread default stream when that is NULL. */
#define SMILI_NOALLOC_SCRATCH_BYTES (16u << 20)
int smili_calc_cost_noalloc(const smili_imaging_args* a, const double* x, const smili_options* opt,
                            double* terms, double* grad);

const char* smili_last_error(void);
int smili_version(void);

#ifdef __cplusplus
}
#endif
#endif
