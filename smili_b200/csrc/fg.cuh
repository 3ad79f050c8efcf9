// One function/gradient evaluation of the static-imaging objective, split into
// stages that the CTAs of a group share (a group barrier separates stages).
//
// Replaces calc_cost (src/fortlib/fftim2d.f90:387-607) =
//   calc_chisq (src/fortlib/fftlib.f90:250-382):
//     I1d_I2d_fwd + FINUFFT type 2 (wrapfinufft.f90:94-128)   -> stages F1-F3
//     calc_chisq_fcv/amp/ca/cp (fftlib.f90:384-655)           -> stage F4
//     NUFFT_adj_resid: 2 x FINUFFT type 1 (fftlib.f90:152-174) -> stages F5-F7
//       (one type-1 of c = Vresre - i Vresim: Re T1(c) = Re T1(Vresre) + Im T1(Vresim))
//   + calc_cost_reg (src/fortlib/image.f90:12-200)             -> stage F8
//
// NUFFT (exponential-of-semicircle kernel, upsampling 2) restricted to the
// "band" of fine-grid cells that the uv points touch: the type-2 row pass
// keeps only band columns and the column pass only runs on band columns; the
// type-1 passes run only on band rows.  Fine-grid coordinates xi = u n / 2pi
// are precomputed at set-up.
#pragma once
#include "common.cuh"
#include "fft.cuh"

template <typename R>
__device__ __forceinline__ R es_kernel(R z, R beta) {
  const R s = (R)1 - z * z;
  return s > (R)0 ? exp(beta * (sqrt(s) - (R)1)) : (R)0;
}

// FP32: the hardware exponential; its error (a few ulps over the kernel's
// argument range [-beta, 0]) is far below the 1e-6 tolerance of the transform
template <>
__device__ __forceinline__ float es_kernel<float>(float z, float beta) {
  const float s = 1.f - z * z;
  return s > 0.f ? __expf(beta * (sqrtf(s) - 1.f)) : 0.f;
}

__device__ __forceinline__ int imod(int a, int n) {
  if ((unsigned)a < (unsigned)n) return a;  // the common case
  int r = a % n;
  return r < 0 ? r + n : r;
}
// a in (-n, 2n): one conditional add or subtract
__device__ __forceinline__ int wrapn(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__device__ __forceinline__ double smabs(double x) { return sqrt(x * x + 1e-10); }
__device__ __forceinline__ float smabs(float x) { return sqrtf(x * x + 1e-10f); }

// rows (sequences) per CTA pass for an FFT of length n
__device__ __forceinline__ int fft_batch(int n) {
  int s = (int)(blockDim.x * 8) / n;
  return s < 1 ? 1 : s;
}

// Working context of one problem inside a kernel
template <typename R>
struct FgCtx {
  const ProbDesc* P;
  char* base;
  cpx<R>* sbuf;   // shared: 2 * SMEM_CPX complex values
  cpx<R>* swork;
  int smem_cpx;   // capacity of each of the two FFT buffers (complex elements)
  int dyn_cpx;    // capacity of the whole dynamic shared region (complex elements)
};

// Running compensated sum (TwoSum) used for the chi-square terms
struct KSum {
  double s, c;
  __device__ void add(double v) {
    const double t = s + v;
    const double bp = t - s;
    c += (s - (t - bp)) + (v - bp);
    s = t;
  }
  __device__ double value() const { return s + c; }
};
struct KSumF {
  float s, c;
  __device__ void add(float v) {
    const float t = s + v;
    const float bp = t - s;
    c += (s - (t - bp)) + (v - bp);
    s = t;
  }
  __device__ double value() const { return (double)s + (double)c; }
};

// ---------------------------------------------------------------------------
// Band passes as dense products (P.dft): with the twiddle matrices
//   Ex[b][ix] = exp(+2 pi i (ix - nx/2)(b1s + b) / nf1)   [b1n][nx]
//   Ey[r][iy] = exp(+2 pi i (iy - ny/2)(b2s + r) / nf2)   [b2n][ny]
// the four FFT passes of the band-pruned NUFFT are
//   F1  tmpA[iy][b]  = sum_ix U[iy][ix] Ex[b][ix],  U = x dc1[ix] dc2[iy]
//   F2  bandA[r][b]  = sum_iy Ey[r][iy] tmpA[iy][b]
//   F6  tmpC[r][ix]  = sum_b  bandC[r][b] Ex[b][ix]
//   F7  gchi[iy][ix] = Re sum_r Ey[r][iy] tmpC[r][ix]  * dc1[ix] dc2[iy]
// (the same twiddles the radix passes apply, exp periodic in nf).  Used
// for bands of at most 64 x 64 cells, where each pass is a few million
// multiply-adds that run as register-tiled loops.
// ---------------------------------------------------------------------------
constexpr int DFT_NB = 64;  // largest band side on this path
constexpr int DFT_KC = 32;  // image columns per staged chunk in F1

// F1 on the DFT path; also writes the dense image grid and the moments.
// Threads: 16 column lanes x (T/16) row lanes; each thread accumulates 2 rows
// x 4 band columns (b = lane, lane + 16, ...).  Row blocks of 2 T/16 rows go
// to the group's CTAs in turn; per block the image and Ex are staged in
// chunks of DFT_KC columns (rows padded by one element against bank
// conflicts).
template <typename R>
__device__ void dft_t2_rows(FgCtx<R>& c, const GroupCtx& g, double (&mom)[10]) {
  const ProbDesc& P = *c.P;
  const double* x = at<double>(c.base, P.o_x);
  const int* inv = at<int>(c.base, P.o_inv);
  double* xg = at<double>(c.base, P.o_xg);
  const double* dc1 = at<double>(c.base, P.o_dc1);
  const double* dc2 = at<double>(c.base, P.o_dc2);
  const cpx<R>* Ex = at<cpx<R>>(c.base, P.o_ex);
  cpx<R>* tmpA = at<cpx<R>>(c.base, P.o_tmpA);
  cpx<R>* bandC = at<cpx<R>>(c.base, P.o_bandC);
  const int nx = P.nx, ny = P.ny, nb = P.b1n;
  const int T = blockDim.x, tc = threadIdx.x & 15, tr = threadIdx.x >> 4;
  const int RB = 2 * (T >> 4);  // rows per block
  const int KP = DFT_KC + 1;
  R* Us = reinterpret_cast<R*>(c.sbuf);                                             // [RB][KP]
  cpx<R>* Es = reinterpret_cast<cpx<R>*>(c.sbuf) + ((size_t)RB * KP * sizeof(R) + sizeof(cpx<R>) - 1) / sizeof(cpx<R>);  // [64][KP]
  for (int i = g.rank * T + threadIdx.x; i < P.b2n * P.b1n; i += g.G * T) bandC[i] = cmk<R>(0, 0);
  const bool need_mom = P.has_tfd || P.has_cen || P.has_sm;
  for (int y0 = g.rank * RB; y0 < ny; y0 += g.G * RB) {
    cpx<R> acc[2][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[a][q] = cmk<R>(0, 0);
    for (int k0 = 0; k0 < nx; k0 += DFT_KC) {
      for (int i = threadIdx.x; i < RB * DFT_KC; i += T) {
        const int rr = i / DFT_KC, kk = i - rr * DFT_KC, iy = y0 + rr, ix = k0 + kk;
        R u = 0;
        if (iy < ny && ix < nx) {
          const int pv = P.ident ? iy * nx + ix : inv[iy * nx + ix];
          const double val = pv >= 0 ? x[pv] : 0.0;
          if (!P.ident) xg[(size_t)iy * nx + ix] = val;
          u = (R)(val * dc1[ix] * dc2[iy]);
          if (need_mom && pv >= 0) {
            const double fx = ix + 1, fy = iy + 1;  // 1-based pixel numbers as the reference
            mom[0] += val;
            mom[1] += fabs(val);
            mom[2] += val * fx;
            mom[3] += val * fy;
            mom[4] += val * fx * fx;
            mom[5] += val * fy * fy;
            mom[6] += val * fx * fy;
            if (P.has_cen) {
              const double Ip = fabs(P.cen_alpha - 1) < 1e-10 ? smabs(val) : pow(smabs(val), P.cen_alpha);
              mom[7] += Ip * (fx - P.nxref);
              mom[8] += Ip * (fy - P.nyref);
              mom[9] += Ip;
            }
          }
        }
        Us[rr * KP + kk] = u;
      }
      for (int i = threadIdx.x; i < DFT_NB * DFT_KC; i += T) {
        const int b = i / DFT_KC, kk = i - b * DFT_KC, ix = k0 + kk;
        Es[b * KP + kk] = (b < nb && ix < nx) ? Ex[(size_t)b * nx + ix] : cmk<R>(0, 0);
      }
      __syncthreads();
      const R* u0 = Us + (2 * tr) * KP;
#pragma unroll 4
      for (int kk = 0; kk < DFT_KC; ++kk) {
        const R ua = u0[kk], ub = u0[KP + kk];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const cpx<R> e = Es[(tc + 16 * q) * KP + kk];
          acc[0][q].x += ua * e.x;
          acc[0][q].y += ua * e.y;
          acc[1][q].x += ub * e.x;
          acc[1][q].y += ub * e.y;
        }
      }
      __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const int iy = y0 + 2 * tr + a;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int b = tc + 16 * q;
        if (iy < ny && b < nb) tmpA[(size_t)iy * nb + b] = acc[a][q];
      }
    }
  }
}

// F2 on the DFT path: one band cell per thread and pass; tmpA and Ey staged
// in chunks of DFT_KC rows.
template <typename R>
__device__ void dft_t2_cols(FgCtx<R>& c, const GroupCtx& g) {
  const ProbDesc& P = *c.P;
  const cpx<R>* Ey = at<cpx<R>>(c.base, P.o_ey);
  const cpx<R>* tmpA = at<cpx<R>>(c.base, P.o_tmpA);
  cpx<R>* bandA = at<cpx<R>>(c.base, P.o_bandA);
  const int ny = P.ny, nb = P.b1n, nr = P.b2n, ncell = nb * nr;
  const int T = blockDim.x, KP = DFT_KC + 1;
  cpx<R>* As = c.sbuf;                   // [DFT_KC][nb]
  cpx<R>* Ys = c.sbuf + DFT_KC * DFT_NB;  // [nr][KP]
  for (int o0 = g.rank * T; o0 < ncell; o0 += g.G * T) {
    const int o = o0 + threadIdx.x, r = o / nb, b = o - r * nb;
    cpx<R> acc = cmk<R>(0, 0);
    for (int k0 = 0; k0 < ny; k0 += DFT_KC) {
      for (int i = threadIdx.x; i < DFT_KC * nb; i += T) {
        const int kk = i / nb, bb = i - kk * nb;
        As[i] = k0 + kk < ny ? tmpA[(size_t)(k0 + kk) * nb + bb] : cmk<R>(0, 0);
      }
      for (int i = threadIdx.x; i < nr * DFT_KC; i += T) {
        const int rr = i / DFT_KC, kk = i - rr * DFT_KC;
        Ys[rr * KP + kk] = k0 + kk < ny ? Ey[(size_t)rr * ny + k0 + kk] : cmk<R>(0, 0);
      }
      __syncthreads();
      if (o < ncell) {
#pragma unroll 4
        for (int kk = 0; kk < DFT_KC; ++kk) {
          const cpx<R> e = Ys[r * KP + kk], t = As[kk * nb + b];
          acc.x += e.x * t.x - e.y * t.y;
          acc.y += e.x * t.y + e.y * t.x;
        }
      }
      __syncthreads();
    }
    if (o < ncell) bandA[o] = acc;
  }
}

// F6 on the DFT path: bandC staged whole; a thread takes one image column
// and up to 8 band rows, streaming its column of Ex.
template <typename R>
__device__ void dft_t1_rows(FgCtx<R>& c, const GroupCtx& g) {
  const ProbDesc& P = *c.P;
  const cpx<R>* Ex = at<cpx<R>>(c.base, P.o_ex);
  const cpx<R>* bandC = at<cpx<R>>(c.base, P.o_bandC);
  cpx<R>* tmpC = at<cpx<R>>(c.base, P.o_tmpC);
  const int nx = P.nx, nb = P.b1n, nr = P.b2n;
  const int T = blockDim.x;
  cpx<R>* Bs = c.sbuf;  // [nr][nb]
  for (int i = threadIdx.x; i < nr * nb; i += T) Bs[i] = bandC[i];
  __syncthreads();
  const int ngrp = (nr + 7) >> 3, items = nx * ngrp;
  for (int it = g.rank * T + threadIdx.x; it < items; it += g.G * T) {
    const int rg = it / nx, ix = it - rg * nx, r0 = 8 * rg;
    cpx<R> acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = cmk<R>(0, 0);
    for (int b = 0; b < nb; ++b) {
      const cpx<R> e = Ex[(size_t)b * nx + ix];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (r0 + j < nr) {
          const cpx<R> v = Bs[(r0 + j) * nb + b];
          acc[j].x += v.x * e.x - v.y * e.y;
          acc[j].y += v.x * e.y + v.y * e.x;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (r0 + j < nr) tmpC[(size_t)(r0 + j) * nx + ix] = acc[j];
  }
  __syncthreads();
}

// F7 on the DFT path: a thread takes one image column and 4 image rows.
template <typename R>
__device__ void dft_t1_cols(FgCtx<R>& c, const GroupCtx& g) {
  const ProbDesc& P = *c.P;
  const cpx<R>* Ey = at<cpx<R>>(c.base, P.o_ey);
  const cpx<R>* tmpC = at<cpx<R>>(c.base, P.o_tmpC);
  const double* dc1 = at<double>(c.base, P.o_dc1);
  const double* dc2 = at<double>(c.base, P.o_dc2);
  double* gchi = at<double>(c.base, P.o_gchi);
  const int nx = P.nx, ny = P.ny, nr = P.b2n;
  const int T = blockDim.x, ngrp = (ny + 3) >> 2, items = nx * ngrp;
  for (int it = g.rank * T + threadIdx.x; it < items; it += g.G * T) {
    const int yg = it / nx, ix = it - yg * nx, y0 = 4 * yg;
    R acc[4] = {0, 0, 0, 0};
    for (int r = 0; r < nr; ++r) {
      const cpx<R> t = tmpC[(size_t)r * nx + ix];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        if (y0 + j < ny) {
          const cpx<R> e = Ey[(size_t)r * ny + y0 + j];
          acc[j] += e.x * t.x - e.y * t.y;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (y0 + j < ny) gchi[(size_t)(y0 + j) * nx + ix] = (double)acc[j] * dc1[ix] * dc2[y0 + j];
  }
}

// ---------------------------------------------------------------------------
// F1: type-2 row pass.  Deconvolved image rows -> band columns of the
// row-transformed fine grid (tmpA[iy][b], b < b1n).  Also zeroes bandC.
// Optionally accumulates image moments for the global regularizers.
// ---------------------------------------------------------------------------
template <typename R>
__device__ void fg_t2_rows(FgCtx<R>& c, const GroupCtx& g, double (&mom)[10]) {
  if (c.P->dft) {
    dft_t2_rows(c, g, mom);
    return;
  }
  const ProbDesc& P = *c.P;
  const double* x = at<double>(c.base, P.o_x);
  const int* inv = at<int>(c.base, P.o_inv);
  double* xg = at<double>(c.base, P.o_xg);
  const double* dc1 = at<double>(c.base, P.o_dc1);
  const double* dc2 = at<double>(c.base, P.o_dc2);
  const cpx<R>* tw1 = at<cpx<R>>(c.base, P.o_tw1);
  cpx<R>* tmpA = at<cpx<R>>(c.base, P.o_tmpA);
  cpx<R>* bandC = at<cpx<R>>(c.base, P.o_bandC);
  const int n1 = P.nf1, nx = P.nx, ny = P.ny;
  const FftPlan pl = make_plan(n1);
  const int S = min(fft_batch(n1), c.smem_cpx / n1);
  for (int i = g.rank * blockDim.x + threadIdx.x; i < P.b2n * P.b1n; i += g.G * blockDim.x)
    bandC[i] = cmk<R>(0, 0);
  const bool need_mom = P.has_tfd || P.has_cen || P.has_sm;
  for (int row0 = g.rank * S; row0 < ny; row0 += g.G * S) {
    const int rows = min(S, ny - row0);
    for (int i = threadIdx.x; i < rows * n1; i += blockDim.x) c.sbuf[i] = cmk<R>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < rows * nx; i += blockDim.x) {
      const int s = i / nx, ix = i - s * nx, iy = row0 + s;
      const int pv = P.ident ? iy * nx + ix : inv[iy * nx + ix];
      const double val = pv >= 0 ? x[pv] : 0.0;
      if (!P.ident) xg[(size_t)iy * nx + ix] = val;
      c.sbuf[s * n1 + wrapn(ix - nx / 2, n1)] = cmk<R>((R)(val * dc1[ix] * dc2[iy]), (R)0);
      if (need_mom && pv >= 0) {
        const double fx = ix + 1, fy = iy + 1;  // 1-based pixel numbers as the reference
        mom[0] += val;
        mom[1] += fabs(val);
        mom[2] += val * fx;
        mom[3] += val * fy;
        mom[4] += val * fx * fx;
        mom[5] += val * fy * fy;
        mom[6] += val * fx * fy;
        if (P.has_cen) {
          const double Ip = fabs(P.cen_alpha - 1) < 1e-10 ? smabs(val) : pow(smabs(val), P.cen_alpha);
          mom[7] += Ip * (fx - P.nxref);
          mom[8] += Ip * (fy - P.nyref);
          mom[9] += Ip;
        }
      }
    }
    __syncthreads();
    const cpx<R>* out = smem_fft(c.sbuf, c.swork, pl, rows, tw1);
    for (int i = threadIdx.x; i < rows * P.b1n; i += blockDim.x) {
      const int s = i / P.b1n, b = i - s * P.b1n;
      tmpA[(size_t)(row0 + s) * P.b1n + b] = out[s * n1 + wrapn(P.b1s + b, n1)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// F2: type-2 column pass over band columns -> bandA[b2][b1]
// ---------------------------------------------------------------------------
template <typename R>
__device__ void fg_t2_cols(FgCtx<R>& c, const GroupCtx& g) {
  if (c.P->dft) {
    dft_t2_cols(c, g);
    return;
  }
  const ProbDesc& P = *c.P;
  const cpx<R>* tw2 = at<cpx<R>>(c.base, P.o_tw2);
  const cpx<R>* tmpA = at<cpx<R>>(c.base, P.o_tmpA);
  cpx<R>* bandA = at<cpx<R>>(c.base, P.o_bandA);
  const int n2 = P.nf2, ny = P.ny, b1n = P.b1n;
  const FftPlan pl = make_plan(n2);
  const int S = min(fft_batch(n2), c.smem_cpx / n2);
  for (int b0 = g.rank * S; b0 < b1n; b0 += g.G * S) {
    const int cols = min(S, b1n - b0);
    for (int i = threadIdx.x; i < cols * n2; i += blockDim.x) c.sbuf[i] = cmk<R>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < cols * ny; i += blockDim.x) {
      const int iy = i / cols, s = i - iy * cols;
      c.sbuf[s * n2 + wrapn(iy - ny / 2, n2)] = tmpA[(size_t)iy * b1n + b0 + s];
    }
    __syncthreads();
    const cpx<R>* out = smem_fft(c.sbuf, c.swork, pl, cols, tw2);
    for (int i = threadIdx.x; i < cols * P.b2n; i += blockDim.x) {
      const int b2 = i / cols, s = i - b2 * cols;
      bandA[(size_t)b2 * b1n + b0 + s] = out[s * n2 + wrapn(P.b2s + b2, n2)];
    }
    __syncthreads();
  }
}

// Interpolation of the points j = j0, j0 + dj, ... < nuv from the band:
// V_j = sum_b psi(v_j - l2 - b) sum_a psi(u_j - l1 - a) band[l2 + b][l1 + a].
// The kernel width W is a template constant so both tap vectors stay in
// registers and the W row loads of a tap row issue back to back.
template <int W, typename R>
__device__ __forceinline__ void interp_points(const ProbDesc& P, const R* __restrict__ xu, const R* __restrict__ xv,
                                              const cpx<R>* bandA, cpx<R>* V, cpx<R>* cacc, R beta, int j0,
                                              int dj) {
  const R half = (R)0.5 * (R)W;
  const R inv = (R)1 / half;
  for (int j = j0; j < P.nuv; j += dj) {
    const R x1 = xu[j], x2 = xv[j];
    const int l1 = (int)ceil(x1 - half), l2 = (int)ceil(x2 - half);
    R k1[W], k2[W];
#pragma unroll
    for (int a = 0; a < W; ++a) {
      k1[a] = es_kernel(((R)(l1 + a) - x1) * inv, beta);
      k2[a] = es_kernel(((R)(l2 + a) - x2) * inv, beta);
    }
    const int c1 = imod(l1 - P.b1s, P.nf1), c2 = imod(l2 - P.b2s, P.nf2);
    R ar = 0, ai = 0;
#pragma unroll
    for (int b = 0; b < W; ++b) {
      int rw = c2 + b;  // wraps only when the band spans the whole fine grid
      if (rw >= P.nf2) rw -= P.nf2;
      const cpx<R>* row = bandA + (size_t)rw * P.b1n;
      R rr = 0, ri = 0;
#pragma unroll
      for (int a = 0; a < W; ++a) {
        int cl = c1 + a;
        if (cl >= P.nf1) cl -= P.nf1;
        const cpx<R> q = row[cl];
        rr += k1[a] * q.x;
        ri += k1[a] * q.y;
      }
      ar += k2[b] * rr;
      ai += k2[b] * ri;
    }
    V[j] = cmk(ar, ai);
    if (cacc) cacc[j] = cmk<R>(0, 0);
  }
}

// ---------------------------------------------------------------------------
// F3: type-2 interpolation, V_j = sum psi psi bandA.  With zero_acc it also
// clears the points' derivative accumulators that F4 adds into.
// ---------------------------------------------------------------------------
template <typename R>
__device__ void fg_interp(FgCtx<R>& c, const GroupCtx& g, bool zero_acc) {
  const ProbDesc& P = *c.P;
  const R* xu = at<R>(c.base, P.o_u);
  const R* xv = at<R>(c.base, P.o_v);
  const cpx<R>* gband = at<cpx<R>>(c.base, P.o_bandA);
  cpx<R>* V = at<cpx<R>>(c.base, P.o_V);
  cpx<R>* cacc = zero_acc ? at<cpx<R>>(c.base, P.o_contrib) : nullptr;
  const int w = P.w;
  const R beta = (R)P.beta;
  const int ncell = P.b1n * P.b2n;
  // the band is re-read w*w times per point: stage it in shared memory
  const bool staged = ncell <= c.dyn_cpx;
  const cpx<R>* bandA = gband;
  if (staged) {
    // only CTAs that own points load the band
    if (g.rank * (int)blockDim.x < P.nuv) {
      for (int i = threadIdx.x; i < ncell; i += blockDim.x) c.sbuf[i] = gband[i];
      __syncthreads();
      bandA = c.sbuf;
    }
  }
  const int j0 = g.rank * blockDim.x + threadIdx.x, dj = g.G * blockDim.x;
  switch (w) {
#define SMILI_INTERP_W(W) \
  case W: interp_points<W>(P, xu, xv, bandA, V, cacc, beta, j0, dj); break;
    SMILI_INTERP_W(2) SMILI_INTERP_W(3) SMILI_INTERP_W(4) SMILI_INTERP_W(5) SMILI_INTERP_W(6)
    SMILI_INTERP_W(7) SMILI_INTERP_W(8) SMILI_INTERP_W(9) SMILI_INTERP_W(10) SMILI_INTERP_W(11)
    SMILI_INTERP_W(12) SMILI_INTERP_W(13) SMILI_INTERP_W(14) SMILI_INTERP_W(15)
    default: interp_points<16>(P, xu, xv, bandA, V, cacc, beta, j0, dj); break;  // w <= SMILI_MAXW = 16
#undef SMILI_INTERP_W
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// F4: chi-square terms, and their derivatives with respect to each model
// visibility added into that uv point's accumulator (o_contrib, zeroed by F3)
// with global atomics: one vector reduction per contribution in FP32, two in
// FP64.  The accumulators (one complex value per uv point) are small enough
// to stay in L2 while the data stream past, and spreading then reads them in
// its own point order.
// chi[0..3] = fcv, amp, cp, ca (weighted by the normalised data weights).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void acc_add(cpx<float>* p, cpx<float> v) {
  atomicAdd(reinterpret_cast<float2*>(p), make_float2(v.x, v.y));
}
__device__ __forceinline__ void acc_add(cpx<double>* p, cpx<double> v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

template <typename R>
__device__ void fg_chisq(FgCtx<R>& c, const GroupCtx& g, double (&chi)[4]) {
  const ProbDesc& P = *c.P;
  const cpx<R>* V = at<cpx<R>>(c.base, P.o_V);
  const R* dre = at<R>(c.base, P.o_dre);
  const R* dim = at<R>(c.base, P.o_dim);
  const R* dvar = at<R>(c.base, P.o_dvar);
  const int* didx = at<int>(c.base, P.o_didx);
  const signed char* dsgn = at<signed char>(c.base, P.o_dsgn);
  cpx<R>* cacc = at<cpx<R>>(c.base, P.o_contrib);
  typedef typename std::conditional<sizeof(R) == 8, KSum, KSumF>::type Acc;
  Acc acc[4];
  for (int q = 0; q < 4; ++q) acc[q].s = acc[q].c = 0;
  const int e_amp = P.nfcv, e_cp = e_amp + P.namp, e_ca = e_cp + P.ncp, e_end = e_ca + P.nca;
  const int s_amp = P.nfcv, s_cp = s_amp + P.namp, s_ca = s_cp + 3 * P.ncp;
  const R wf = (R)P.wfcv, wa = (R)P.wamp, wc = (R)P.wcp, wq = (R)P.wca;
  // model_fcv/amp/cp/ca (fftlib.f90:744-1254) also return each datum's model and residual
  double* mres = P.o_model ? at<double>(c.base, P.o_model) : nullptr;
  // One loop per data type over the same items (i = j0 + k dj) in the same
  // order as a single loop, two items per step: both items' gathers are
  // issued before either is evaluated, so their latencies overlap.
  const int j0 = g.rank * blockDim.x + threadIdx.x, dj = g.G * blockDim.x;
  auto first = [&](int a) { return a <= j0 ? j0 : j0 + (a - j0 + dj - 1) / dj * dj; };
  auto put = [&](int i, R model, R model2, R resid, R resid2) {
    if (mres) {
      mres[4 * i] = model;
      mres[4 * i + 1] = model2;
      mres[4 * i + 2] = resid;
      mres[4 * i + 3] = resid2;
    }
  };
  // complex visibilities (fftlib.f90:384-439)
  auto fcv = [&](int i, int k, const cpx<R>& Vk, R sg, R var, R yr, R yi) {
    const R rr = yr - Vk.x, ri = yi - sg * Vk.y;
    acc[0].add(((rr * rr + ri * ri) / var) * wf);
    const R factor = (R)-2 / var * wf;
    acc_add(cacc + k, cmk(factor * rr, factor * ri * sg));
    put(i, Vk.x, sg * Vk.y, rr, ri);
  };
  for (int i = first(0); i < e_amp; i += 2 * dj) {
    const int ib = i + dj;
    const bool two = ib < e_amp;
    const int ka = didx[i], kb = two ? didx[ib] : ka;
    const cpx<R> Va = V[ka], Vb = V[kb];
    const R sa = (R)dsgn[i], sb = two ? (R)dsgn[ib] : sa;
    const R va = dvar[i], vb = two ? dvar[ib] : va;
    const R ra = dre[i], rb = two ? dre[ib] : ra, ia = dim[i], ibm = two ? dim[ib] : ia;
    fcv(i, ka, Va, sa, va, ra, ia);
    if (two) fcv(ib, kb, Vb, sb, vb, rb, ibm);
  }
  // amplitudes (fftlib.f90:442-493)
  auto amp = [&](int i, int k, const cpx<R>& Vk, R var, R y) {
    const R model = sqrt(Vk.x * Vk.x + Vk.y * Vk.y);
    const R resid = y - model;
    acc[1].add((resid * resid / var) * wa);
    const R factor = (R)-2 * resid / var / model * wa;
    acc_add(cacc + k, cmk(factor * Vk.x, factor * Vk.y));
    put(i, model, 0, resid, 0);
  };
  for (int i = first(e_amp); i < e_cp; i += 2 * dj) {
    const int ib = i + dj;
    const bool two = ib < e_cp;
    const int ka = didx[s_amp + (i - e_amp)], kb = two ? didx[s_amp + (ib - e_amp)] : ka;
    const cpx<R> Va = V[ka], Vb = V[kb];
    const R va = dvar[i], vb = two ? dvar[ib] : va;
    const R ya = dre[i], yb = two ? dre[ib] : ya;
    amp(i, ka, Va, va, ya);
    if (two) amp(ib, kb, Vb, vb, yb);
  }
  // closure phases (fftlib.f90:576-655)
  auto cp = [&](int i, const int (&kq)[3], const cpx<R> (&Vq)[3], const R (&sg)[3], R var, R y) {
    R a2[3];
    R model = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      a2[q] = Vq[q].x * Vq[q].x + Vq[q].y * Vq[q].y;
      model = atan2(Vq[q].y, Vq[q].x) * sg[q] + model;
    }
    const R resid = y - model;
    R sr, cr;
    if (sizeof(R) == 8) {
      double s_, c_;
      sincos((double)resid, &s_, &c_);
      sr = (R)s_;
      cr = (R)c_;
    } else {
      float s_, c_;
      sincosf((float)resid, &s_, &c_);
      sr = (R)s_;
      cr = (R)c_;
    }
    acc[2].add(((R)2 * ((R)1 - cr) / var) * wc);
    const R factor = (R)-2 * sr / var * wc;
#pragma unroll
    for (int q = 0; q < 3; ++q)
      acc_add(cacc + kq[q], cmk(-factor / a2[q] * Vq[q].y * sg[q], factor / a2[q] * Vq[q].x * sg[q]));
    put(i, model, 0, resid, 0);  // unwrapped; the host wraps both into (-pi, pi] as model_cp does
  };
  for (int i = first(e_cp); i < e_ca; i += 2 * dj) {
    const int ib = i + dj;
    const bool two = ib < e_ca;
    const int sa = s_cp + 3 * (i - e_cp), sb = two ? s_cp + 3 * (ib - e_cp) : sa;
    int ka[3], kb[3];
    cpx<R> Va[3], Vb[3];
    R ga[3], gb[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      ka[q] = didx[sa + q];
      kb[q] = didx[sb + q];
      ga[q] = (R)dsgn[sa + q];
      gb[q] = (R)dsgn[sb + q];
    }
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      Va[q] = V[ka[q]];
      Vb[q] = V[kb[q]];
    }
    const R va = dvar[i], vb = two ? dvar[ib] : va;
    const R ya = dre[i], yb = two ? dre[ib] : ya;
    cp(i, ka, Va, ga, va, ya);
    if (two) cp(ib, kb, Vb, gb, vb, yb);
  }
  // log closure amplitudes (fftlib.f90:496-573)
  auto ca = [&](int i, const int (&kq)[4], const cpx<R> (&Vq)[4], R var, R y) {
    R a[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) a[q] = sqrt(Vq[q].x * Vq[q].x + Vq[q].y * Vq[q].y);
    const R model = log(a[0]) + log(a[1]) - log(a[2]) - log(a[3]);
    const R resid = y - model;
    acc[3].add((resid * resid / var) * wq);
    const R factor = (R)-2 * resid / var * wq;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const R f = (q < 2 ? factor : -factor) / (a[q] * a[q]);
      acc_add(cacc + kq[q], cmk(f * Vq[q].x, f * Vq[q].y));
    }
    put(i, model, 0, resid, 0);
  };
  for (int i = first(e_ca); i < e_end; i += 2 * dj) {
    const int ib = i + dj;
    const bool two = ib < e_end;
    const int sa = s_ca + 4 * (i - e_ca), sb = two ? s_ca + 4 * (ib - e_ca) : sa;
    int ka[4], kb[4];
    cpx<R> Va[4], Vb[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ka[q] = didx[sa + q];
      kb[q] = didx[sb + q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      Va[q] = V[ka[q]];
      Vb[q] = V[kb[q]];
    }
    const R va = dvar[i], vb = two ? dvar[ib] : va;
    const R ya = dre[i], yb = two ? dre[ib] : ya;
    ca(i, ka, Va, va, ya);
    if (two) ca(ib, kb, Vb, vb, yb);
  }
  for (int q = 0; q < 4; ++q) chi[q] += acc[q].value();
}

// ---------------------------------------------------------------------------
// F5: spread c_j = Vresre_j - i Vresim_j, read from the uv points'
// derivative accumulators in the bin-sorted point order, onto bandC.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_add_r(double* p, double v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_r(float* p, float v) { atomicAdd(p, v); }

template <typename R>
__device__ __forceinline__ R warp_sum(R v) {
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  return v;
}

// Subproblem spreading.  The bin-sorted points are cut into work items of
// at most 128 points that share one 8x8 bin of the band.  A warp owns an item
// and a private (8+w-1)^2 subgrid in shared memory: for every point the
// lanes cover the w*w taps (all lanes hit different cells, and consecutive
// points are ordered by __syncwarp), so the inner loop needs no atomics.  The
// finished subgrid is added to the CTA's band copy (shared atomics, only the
// overlapping halos collide) and the CTA's band to the global band at the end.
// ---------------------------------------------------------------------------
// F5 on the tensor cores (FP32, w <= 9, 8 x 8 tiles).  A tile's subgrid is a
// product of two thin matrices:
//   D[r][c] = sum_p wy_p[r] (c_p wx_p[c]),   r, c < 8 + w - 1 <= 16,
// with wy_p / wx_p the point's kernel weights placed at its offset inside
// the subgrid (zero elsewhere) and c_p = Vres_re - i Vres_im of the point.
// A warp accumulates the real and imaginary parts of one tile's 16 x 16
// subgrid in mma.sync.m16n8k8 TF32 fragments (8 points per k step) with the
// three-term split a b ~ ah bh + ah bl + al bh (a = ah + al in TF32), which
// keeps the products within a few FP32 ulps; the subgrid never touches
// shared memory and no tap waits on another.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ void fg_spread_tc(FgCtx<float>& c, const GroupCtx& g) {
  const ProbDesc& P = *c.P;
  const float* xu = at<float>(c.base, P.o_u);
  const float* xv = at<float>(c.base, P.o_v);
  const int4* items = at<int4>(c.base, P.o_items);
  const cpx<float>* cacc = at<cpx<float>>(c.base, P.o_contrib);
  float* gband = at<float>(c.base, P.o_bandC);
  const int w = P.w;
  const int SG = 8 + w - 1;  // <= 16
  const float beta = (float)P.beta;
  const float half = 0.5f * (float)w, inv = 1.f / half;
  const int ncell = P.b1n * P.b2n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int gq = lane >> 2, t = lane & 3;
  // shared memory: [nw][32 points][2w] kernel weights, then (if it fits) a
  // private copy of the band
  const size_t wt_b = ((size_t)nw * 32 * 2 * w * sizeof(float) + 15) / 16 * 16;
  float* wtab = reinterpret_cast<float*>(c.sbuf) + (size_t)warp * 32 * 2 * w;
  cpx<float>* sband = reinterpret_cast<cpx<float>*>(reinterpret_cast<char*>(c.sbuf) + wt_b);
  const bool staged = wt_b + (size_t)ncell * sizeof(cpx<float>) <= (size_t)c.dyn_cpx * sizeof(cpx<float>);
  float* band = staged ? reinterpret_cast<float*>(sband) : gband;
  if (staged) {
    for (int i = threadIdx.x; i < ncell; i += blockDim.x) sband[i] = cmk<float>(0, 0);
    __syncthreads();
  }
  const int gw = g.rank * nw + warp, nwt = g.G * nw;
  for (int it = gw; it < P.nitems; it += nwt) {
    const int4 item = items[it];
    float dre[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, dim[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    for (int jb = item.x; jb < item.y; jb += 32) {
      // phase 1: every lane prepares one point (zero weights past the item)
      const int jl = jb + lane;
      float cre_l = 0.f, cim_l = 0.f;
      int lr_l = 0, lc_l = 0;
      float* wr = wtab + lane * 2 * w;
      if (jl < item.y) {
        const cpx<float> cj = cacc[jl];
        cre_l = cj.x;
        cim_l = -cj.y;  // c = Vresre - i Vresim
        const float xi1 = xu[jl], xi2 = xv[jl];
        const int l1 = (int)ceilf(xi1 - half), l2 = (int)ceilf(xi2 - half);
        for (int q = 0; q < w; ++q) {
          wr[q] = es_kernel(((float)(l1 + q) - xi1) * inv, beta);
          wr[w + q] = es_kernel(((float)(l2 + q) - xi2) * inv, beta);
        }
        lr_l = imod(l2 - P.b2s, P.nf2) - item.z;
        lc_l = imod(l1 - P.b1s, P.nf1) - item.w;
      } else {
        for (int q = 0; q < 2 * w; ++q) wr[q] = 0.f;
      }
      __syncwarp();
      // phase 2: 8 points per k step; lane (gq, t) feeds points t and t + 4
      const int np = min(32, item.y - jb);
      for (int kb = 0; kb < np; kb += 8) {
        const int p0 = kb + t, p1 = kb + t + 4;
        const int lr0 = __shfl_sync(0xffffffffu, lr_l, p0), lr1 = __shfl_sync(0xffffffffu, lr_l, p1);
        const int lc0 = __shfl_sync(0xffffffffu, lc_l, p0), lc1 = __shfl_sync(0xffffffffu, lc_l, p1);
        const float cr0 = __shfl_sync(0xffffffffu, cre_l, p0), cr1 = __shfl_sync(0xffffffffu, cre_l, p1);
        const float ci0 = __shfl_sync(0xffffffffu, cim_l, p0), ci1 = __shfl_sync(0xffffffffu, cim_l, p1);
        const float* w0 = wtab + p0 * 2 * w;
        const float* w1 = wtab + p1 * 2 * w;
        auto wy = [&](const float* wp, int d) { return (unsigned)d < (unsigned)w ? wp[w + d] : 0.f; };
        auto wx = [&](const float* wp, int d) { return (unsigned)d < (unsigned)w ? wp[d] : 0.f; };
        uint32_t ah[4], al[4];
        split_tf32(wy(w0, gq - lr0), ah[0], al[0]);
        split_tf32(wy(w0, gq + 8 - lr0), ah[1], al[1]);
        split_tf32(wy(w1, gq - lr1), ah[2], al[2]);
        split_tf32(wy(w1, gq + 8 - lr1), ah[3], al[3]);
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int col = 8 * j + gq;
          const float x0 = wx(w0, col - lc0), x1 = wx(w1, col - lc1);
          uint32_t rh0, rl0, rh1, rl1, ih0, il0, ih1, il1;
          split_tf32(x0 * cr0, rh0, rl0);
          split_tf32(x1 * cr1, rh1, rl1);
          split_tf32(x0 * ci0, ih0, il0);
          split_tf32(x1 * ci1, ih1, il1);
          mma_tf32(dre[j], ah, rh0, rh1);
          mma_tf32(dre[j], ah, rl0, rl1);
          mma_tf32(dre[j], al, rh0, rh1);
          mma_tf32(dim[j], ah, ih0, ih1);
          mma_tf32(dim[j], ah, il0, il1);
          mma_tf32(dim[j], al, ih0, ih1);
        }
      }
      __syncwarp();
    }
    // add the subgrid to the band: fragment element e of n-tile j is
    // (row gq + 8 (e >= 2), col 8 j + 2 t + (e & 1))
#pragma unroll
    for (int j = 0; j < 2; ++j) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = gq + (e >= 2 ? 8 : 0), cc = 8 * j + 2 * t + (e & 1);
        const float vr = dre[j][e], vi = dim[j][e];
        if (r >= SG || cc >= SG || (vr == 0.f && vi == 0.f)) continue;
        int rw = item.z + r, cl = item.w + cc;
        if (rw >= P.nf2) rw -= P.nf2;
        if (cl >= P.nf1) cl -= P.nf1;
        if (rw >= P.b2n || cl >= P.b1n) continue;  // beyond the band: only zero taps land here
        float* dst = band + 2 * ((size_t)rw * P.b1n + cl);
        if (staged) {
          atomicAdd(dst, vr);
          atomicAdd(dst + 1, vi);
        } else {
          atomicAdd(reinterpret_cast<float2*>(dst), make_float2(vr, vi));  // one 8-byte global reduction
        }
      }
    }
  }
  if (staged) {
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * ncell; i += blockDim.x) {
      const float vv = band[i];
      if (vv != 0.f) atomicAdd(gband + i, vv);
    }
    __syncthreads();
  }
}

template <typename R>
__device__ void fg_spread(FgCtx<R>& c, const GroupCtx& g) {
  if constexpr (std::is_same<R, float>::value) {
    if (c.P->w <= 9 && c.P->bin == 8) {
      fg_spread_tc(c, g);
      return;
    }
  }
  const ProbDesc& P = *c.P;
  const R* xu = at<R>(c.base, P.o_u);
  const R* xv = at<R>(c.base, P.o_v);
  const int4* items = at<int4>(c.base, P.o_items);
  const cpx<R>* cacc = at<cpx<R>>(c.base, P.o_contrib);
  R* gband = at<R>(c.base, P.o_bandC);
  const int w = P.w, ww = P.w * P.w;
  const int SG = P.bin + w - 1;  // subgrid side
  const R beta = (R)P.beta;
  const R half = (R)0.5 * (R)w, inv = (R)1 / half;
  const int ncell = P.b1n * P.b2n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // shared memory: [nw][SG*SG] complex subgrids, [nw][PB][2w] kernel weights,
  // then (if it fits) a private copy of the band.  nw = the warps that own a
  // subgrid (all of the CTA's when they fit), PB = points prepared per phase,
  // the largest of 32/16/8 that fits.
  const size_t dyn_b = (size_t)c.dyn_cpx * sizeof(cpx<R>);
  int nw = blockDim.x >> 5;
  while (nw > 1 && (size_t)nw * (SG * SG * sizeof(cpx<R>) + 8 * 2 * w * sizeof(R)) + 16 > dyn_b) --nw;
  const size_t sub_b = (size_t)nw * SG * SG * sizeof(cpx<R>);
  int PB = 32;
  while (PB > 8 && sub_b + (size_t)nw * PB * 2 * w * sizeof(R) > dyn_b) PB >>= 1;
  const size_t wt_b = ((size_t)nw * PB * 2 * w * sizeof(R) + 15) / 16 * 16;
  cpx<R>* sub = c.sbuf + (size_t)warp * SG * SG;
  R* wtab = reinterpret_cast<R*>(reinterpret_cast<char*>(c.sbuf) + sub_b) + (size_t)warp * PB * 2 * w;
  cpx<R>* sband = reinterpret_cast<cpx<R>*>(reinterpret_cast<char*>(c.sbuf) + sub_b + wt_b);
  const bool staged = sub_b + wt_b + (size_t)ncell * sizeof(cpx<R>) <= dyn_b;
  R* band = staged ? reinterpret_cast<R*>(sband) : gband;
  if (staged) {
    for (int i = threadIdx.x; i < ncell; i += blockDim.x) sband[i] = cmk<R>(0, 0);
    __syncthreads();
  }
  const int ra = lane % w, rb = lane / w;
  const int gw = g.rank * nw + warp, nwt = g.G * nw;
  for (int it = warp < nw ? gw : P.nitems; it < P.nitems; it += nwt) {
    const int4 item = items[it];
    for (int i = lane; i < SG * SG; i += 32) sub[i] = cmk<R>(0, 0);
    for (int jb = item.x; jb < item.y; jb += PB) {
      // phase 1: lanes < PB prepare one point each (value, cell, kernel weights)
      const int jl = jb + lane;
      R cre_l = 0, cim_l = 0;
      int cell_l = 0;
      if (lane < PB && jl < item.y) {
        const cpx<R> cj = cacc[jl];
        cre_l = cj.x;
        cim_l = cj.y;
        const R xi1 = xu[jl], xi2 = xv[jl];
        const int l1 = (int)ceil(xi1 - half), l2 = (int)ceil(xi2 - half);
        R* wr = wtab + lane * 2 * w;
        for (int q = 0; q < w; ++q) {
          wr[q] = es_kernel(((R)(l1 + q) - xi1) * inv, beta);
          wr[w + q] = es_kernel(((R)(l2 + q) - xi2) * inv, beta);
        }
        // position inside the subgrid (item.z, item.w = subgrid origin row, col)
        const int lr = imod(l2 - P.b2s, P.nf2) - item.z, lc = imod(l1 - P.b1s, P.nf1) - item.w;
        cell_l = lr * SG + lc;
      }
      __syncwarp();
      // phase 2: the lanes cover the taps of one point at a time
      const int np = min(PB, item.y - jb);
      for (int p = 0; p < np; ++p) {
        const R cre = __shfl_sync(0xffffffffu, cre_l, p);
        const R cim = -__shfl_sync(0xffffffffu, cim_l, p);  // c = Vresre - i Vresim
        const int cell0 = __shfl_sync(0xffffffffu, cell_l, p);
        const R* wr = wtab + p * 2 * w;
        int a = ra, b = rb;
        for (int t0 = 0; t0 < ww; t0 += 32) {
          if (t0 + lane < ww) {
            cpx<R>& cell = sub[cell0 + b * SG + a];
            const R wt = wr[a] * wr[w + b];
            cell.x += wt * cre;
            cell.y += wt * cim;
          }
          a += 32 % w;
          b += 32 / w;
          if (a >= w) {
            a -= w;
            b += 1;
          }
        }
        __syncwarp();
      }
    }
    // add the subgrid to the band (rows/cols wrap only for a full-grid band)
    for (int i = lane; i < SG * SG; i += 32) {
      const cpx<R> v = sub[i];
      if (v.x == (R)0 && v.y == (R)0) continue;
      int rw = item.z + i / SG, cl = item.w + i % SG;
      if (rw >= P.nf2) rw -= P.nf2;
      if (cl >= P.nf1) cl -= P.nf1;
      if (rw >= P.b2n || cl >= P.b1n) continue;  // beyond the band: only zero taps land here
      R* dst = band + 2 * ((size_t)rw * P.b1n + cl);
      atomic_add_r(dst, v.x);
      atomic_add_r(dst + 1, v.y);
    }
    __syncwarp();
  }
  if (staged) {
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * ncell; i += blockDim.x) {
      const R vv = band[i];
      if (vv != (R)0) atomic_add_r(gband + i, vv);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// F6: type-1 row pass over band rows -> tmpC[b2][ix] (modes along axis 1)
// ---------------------------------------------------------------------------
template <typename R>
__device__ void fg_t1_rows(FgCtx<R>& c, const GroupCtx& g) {
  if (c.P->dft) {
    dft_t1_rows(c, g);
    return;
  }
  const ProbDesc& P = *c.P;
  const cpx<R>* tw1 = at<cpx<R>>(c.base, P.o_tw1);
  const cpx<R>* bandC = at<cpx<R>>(c.base, P.o_bandC);
  cpx<R>* tmpC = at<cpx<R>>(c.base, P.o_tmpC);
  const int n1 = P.nf1, nx = P.nx, b1n = P.b1n;
  const FftPlan pl = make_plan(n1);
  const int S = min(fft_batch(n1), c.smem_cpx / n1);
  for (int r0 = g.rank * S; r0 < P.b2n; r0 += g.G * S) {
    const int rows = min(S, P.b2n - r0);
    for (int i = threadIdx.x; i < rows * n1; i += blockDim.x) c.sbuf[i] = cmk<R>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < rows * b1n; i += blockDim.x) {
      const int s = i / b1n, b = i - s * b1n;
      c.sbuf[s * n1 + wrapn(P.b1s + b, n1)] = bandC[(size_t)(r0 + s) * b1n + b];
    }
    __syncthreads();
    const cpx<R>* out = smem_fft(c.sbuf, c.swork, pl, rows, tw1);
    for (int i = threadIdx.x; i < rows * nx; i += blockDim.x) {
      const int s = i / nx, ix = i - s * nx;
      tmpC[(size_t)(r0 + s) * nx + ix] = out[s * n1 + wrapn(ix - nx / 2, n1)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// F7: type-1 column pass -> gchi[iy][ix] = Re(F) * dc1 * dc2
// ---------------------------------------------------------------------------
template <typename R>
__device__ void fg_t1_cols(FgCtx<R>& c, const GroupCtx& g) {
  if (c.P->dft) {
    dft_t1_cols(c, g);
    return;
  }
  const ProbDesc& P = *c.P;
  const cpx<R>* tw2 = at<cpx<R>>(c.base, P.o_tw2);
  const cpx<R>* tmpC = at<cpx<R>>(c.base, P.o_tmpC);
  const double* dc1 = at<double>(c.base, P.o_dc1);
  const double* dc2 = at<double>(c.base, P.o_dc2);
  double* gchi = at<double>(c.base, P.o_gchi);
  const int n2 = P.nf2, nx = P.nx, ny = P.ny;
  const FftPlan pl = make_plan(n2);
  const int S = min(fft_batch(n2), c.smem_cpx / n2);
  for (int x0 = g.rank * S; x0 < nx; x0 += g.G * S) {
    const int cols = min(S, nx - x0);
    for (int i = threadIdx.x; i < cols * n2; i += blockDim.x) c.sbuf[i] = cmk<R>(0, 0);
    __syncthreads();
    for (int i = threadIdx.x; i < cols * P.b2n; i += blockDim.x) {
      const int b2 = i / cols, s = i - b2 * cols;
      c.sbuf[s * n2 + wrapn(P.b2s + b2, n2)] = tmpC[(size_t)b2 * nx + x0 + s];
    }
    __syncthreads();
    const cpx<R>* out = smem_fft(c.sbuf, c.swork, pl, cols, tw2);
    for (int i = threadIdx.x; i < cols * ny; i += blockDim.x) {
      const int iy = i / cols, s = i - iy * cols, ix = x0 + s;
      gchi[(size_t)iy * nx + ix] = (double)out[s * n2 + wrapn(iy - ny / 2, n2)].x * dc1[ix] * dc2[iy];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// F8: regularizers + gradient assembly g = gradchisq + gradreg.
// reg[0..7] = l1, tv, tsv, kl, gs, tfd, cen, sm.  Also returns g.d and the
// projected-gradient infinity norm used by the optimiser.
// mom: reduced image moments from F1 (only when tfd/cen/sm are active).
// ---------------------------------------------------------------------------
// Image value at grid cell (ix, iy), 0 outside the image or at a pixel the
// solve does not include: through the pixel map (PxMap) or from the dense
// image grid that the type-2 row pass writes (PxGrid).
struct PxMap {
  const double* x;
  const int* inv;
  int nx, ny;
  __device__ __forceinline__ double operator()(int ix, int iy) const {
    if (ix < 0 || iy < 0 || ix >= nx || iy >= ny) return 0.0;
    const int p = inv[iy * nx + ix];
    return p >= 0 ? x[p] : 0.0;
  }
};
struct PxGrid {
  const double* xg;
  int nx, ny;
  __device__ __forceinline__ double operator()(int ix, int iy) const {
    if (ix < 0 || iy < 0 || ix >= nx || iy >= ny) return 0.0;
    return xg[(size_t)iy * nx + ix];
  }
};
// TV gradient (image.f90:512-612) at pixel (i1, j1) from preloaded values,
// reproducing the gradient reset: I11 = I(i1, j1), xp = I(i1+1, j1),
// yp = I(i1, j1+1), xm = I(i1-1, j1), ym = I(i1, j1-1), xmyp = I(i1-1, j1+1),
// xpym = I(i1+1, j1-1); the has_* flags say which neighbours lie inside the
// image (a value outside is never read).
template <typename T>
__device__ __forceinline__ T tv_grade_vals(T I11, T xp, T yp, T xm, T ym, T xmyp, T xpym, bool has_xp,
                                           bool has_yp, bool has_xm, bool has_ym) {
  T gr = 0;
  T dIx = has_xp ? xp - I11 : (T)0;
  T dIy = has_yp ? yp - I11 : (T)0;
  T e = sqrt(dIx * dIx + dIy * dIy);
  if (e > (T)1e-10) gr -= (dIx + dIy) / e;
  if (has_xm) {
    dIx = I11 - xm;
    dIy = has_yp ? xmyp - xm : (T)0;
    e = sqrt(dIx * dIx + dIy * dIy);
    if (e > (T)1e-10) gr += dIx / e;
    else gr = 0;
  }
  if (has_ym) {
    dIy = I11 - ym;
    dIx = has_xp ? xpym - ym : (T)0;
    e = sqrt(dIx * dIx + dIy * dIy);
    if (e > (T)1e-10) gr += dIy / e;
    else gr = 0;
  }
  return gr;
}
struct RegMoments {
  double Isum_abs, xcen, ycen, Sg[3], mom[2], Sp[3];
  double tfd_resid;
  double cen_sx, cen_sy, cen_sI, cen_cost;
};

__device__ void reg_moments(const ProbDesc& P, const double (&m)[10], RegMoments& r) {
  r.tfd_resid = m[0] - P.tfd_tgtfd;
  r.Isum_abs = m[1];
  r.xcen = m[2] / m[1];
  r.ycen = m[3] / m[1];
  const double S = m[0];
  // second moments about the |I|-normalised centroid from raw moments
  r.Sg[0] = (m[4] - 2 * r.xcen * m[2] + r.xcen * r.xcen * S) / r.Isum_abs;
  r.Sg[1] = (m[5] - 2 * r.ycen * m[3] + r.ycen * r.ycen * S) / r.Isum_abs;
  r.Sg[2] = (m[6] - r.xcen * m[3] - r.ycen * m[2] + r.xcen * r.ycen * S) / r.Isum_abs;
  r.mom[0] = m[2] - r.xcen * S;
  r.mom[1] = m[3] - r.ycen * S;
  const double cp = cos(P.sm_phi), sp = sin(P.sm_phi);
  r.Sp[0] = P.sm_min * cp * cp + P.sm_maj * sp * sp;
  r.Sp[1] = P.sm_min * sp * sp + P.sm_maj * cp * cp;
  r.Sp[2] = (P.sm_maj - P.sm_min) * sp * cp;
  r.cen_sI = m[9] + 1e-10;
  r.cen_sx = m[7] / r.cen_sI;
  r.cen_sy = m[8] / r.cen_sI;
  r.cen_cost = sqrt(r.cen_sx * r.cen_sx + r.cen_sy * r.cen_sy + 1e-10);
}

// image moments of a movie frame that has no data (the row pass of F1
// accumulates the same sums for frames with data); one CTA, per-thread partials
__device__ void frame_moments(const ProbDesc& P, char* base, double (&mom)[10]) {
  const double* x = at<double>(base, P.o_x);
  const int* xi = at<int>(base, P.o_xidx);
  const int* yi = at<int>(base, P.o_yidx);
  for (int p = threadIdx.x; p < P.npix; p += blockDim.x) {
    const double val = x[p], fx = xi[p] + 1, fy = yi[p] + 1;
    mom[0] += val;
    mom[1] += fabs(val);
    mom[2] += val * fx;
    mom[3] += val * fy;
    mom[4] += val * fx * fx;
    mom[5] += val * fy * fy;
    mom[6] += val * fx * fy;
  }
}

// log in the compute type of the regularizer stage
__device__ __forceinline__ double reg_log(double x) { return log(x); }
__device__ __forceinline__ float reg_log(float x) { return logf(x); }

// Per-pixel regularizer terms in the compute type T (float in the FP32 mode):
// L1, TV, TSV, MEM (kl) and the Gaussian-prior entropy (gs).  The moment
// terms (total flux, centroid, second moment) use differences of image-wide
// sums and stay in FP64; so do the regularizer sums, the gradient that the
// optimiser reads and g.d.
template <typename T, class PX>
__device__ void reg_grad_loop(const ProbDesc& P, char* base, const PX& px, const RegMoments& rm, int lo, int hi,
                              double (&reg)[8], double& gd, double& sbg, bool opt_terms) {
  const double* x = at<double>(base, P.o_x);
  const int* xi = at<int>(base, P.o_xidx);
  const int* yi = at<int>(base, P.o_yidx);
  const double* gchi = at<double>(base, P.o_gchi);
  const double* d = at<double>(base, P.o_d);
  double* gout = at<double>(base, P.o_g);
  // a weight array is read only when its weights differ between pixels;
  // otherwise its one value (wu) is used
  const double* l1w = (P.has_l1 && !(P.wuni & 1)) ? at<double>(base, P.o_l1w) : nullptr;
  const double* tvw = (P.has_tv && !(P.wuni & 2)) ? at<double>(base, P.o_tvw) : nullptr;
  const double* tsvw = (P.has_tsv && !(P.wuni & 4)) ? at<double>(base, P.o_tsvw) : nullptr;
  const double* klw = (P.has_kl && !(P.wuni & 8)) ? at<double>(base, P.o_klw) : nullptr;
  const double* gsw = (P.has_gs && !(P.wuni & 16)) ? at<double>(base, P.o_gsw) : nullptr;
  const int nx = P.nx, ny = P.ny;
  const T l1_l = (T)P.l1_l, tv_l = (T)P.tv_l, tsv_l = (T)P.tsv_l, kl_l = (T)P.kl_l, gs_l = (T)P.gs_l;
  const double g_tfd = P.has_tfd ? P.tfd_l * 2 * rm.tfd_resid : 0.0;
  // running sums in registers (the caller's accumulators are written once
  // at the end, so the stores of the loop cannot alias them)
  double r0 = reg[0], r1 = reg[1], r2 = reg[2], r3 = reg[3], r4 = reg[4], gdl = gd, sbgl = sbg;
  const bool nb = P.has_tv || P.has_tsv;
  const bool ident = P.ident;
  for (int p = lo + threadIdx.x; p < hi; p += blockDim.x) {
    // every load of the iteration first (two dependent rounds: the pixel's
    // indices, then its grid cell and neighbours), so that the arithmetic
    // below waits once per round and not once per term
    int ix, iy;
    if (ident) {  // row-major full grid: no index loads, so one round of loads below
      iy = p / nx;
      ix = p - iy * nx;
    } else {
      ix = xi[p];
      iy = yi[p];
    }
    const double I = x[p];
    const double w_l1 = l1w ? l1w[p] : P.wu[0], w_kl = klw ? klw[p] : P.wu[3], w_gs = gsw ? gsw[p] : P.wu[4];
    const double w_tv = tvw ? tvw[p] : P.wu[1], w_tsv = tsvw ? tsvw[p] : P.wu[2];
    const double dp = opt_terms ? d[p] : 0.0;
    const bool hxp = ix + 1 < nx, hyp = iy + 1 < ny, hxm = ix - 1 >= 0, hym = iy - 1 >= 0;
    const double gc = gchi[(size_t)iy * nx + ix];
    double vxp = 0, vyp = 0, vxm = 0, vym = 0, vxmyp = 0, vxpym = 0;
    if (nb) {
      vxp = hxp ? px(ix + 1, iy) : 0.0;
      vyp = hyp ? px(ix, iy + 1) : 0.0;
      vxm = hxm ? px(ix - 1, iy) : 0.0;
      vym = hym ? px(ix, iy - 1) : 0.0;
      if (P.has_tv) {
        vxmyp = (hxm && hyp) ? px(ix - 1, iy + 1) : 0.0;
        vxpym = (hxp && hym) ? px(ix + 1, iy - 1) : 0.0;
      }
    }
    const T It = (T)I;
    // each term is added to one FP64 sum, in the order of image.f90's
    // gradient: total flux, centroid, l1, MEM, gs, TV, TSV, second moment
    double gr = g_tfd;
    if (P.has_cen) {
      const double dix = (ix + 1) - P.nxref, diy = (iy + 1) - P.nyref;
      const double gIp = fabs(P.cen_alpha - 1) < 1e-10
                             ? I / smabs(I)
                             : I / smabs(I) * P.cen_alpha * pow(smabs(I), P.cen_alpha - 1);
      gr += P.cen_l * ((rm.cen_sx * (dix - rm.cen_sx) + rm.cen_sy * (diy - rm.cen_sy)) / rm.cen_sI /
                       rm.cen_cost * gIp);
    }
    if (P.has_l1) {
      const T a = smabs(It), w = l1_l * (T)w_l1;
      r0 += (double)(w * a);
      gr += (double)(w * (It / a));
    }
    if (P.has_kl) {
      const T a = smabs(It), pr = (T)w_kl, lr = reg_log(a / pr);
      r3 += (double)(kl_l * (a * lr + pr / (T)2.718281828459045235));
      gr += (double)(kl_l * (It / a) * (lr + 1));
    }
    if (P.has_gs) {
      const T a = smabs(It), pr = (T)w_gs, lr = reg_log(a / pr);
      r4 += (double)(gs_l * (a * (lr - 1) + pr));
      gr += (double)(gs_l * (It / a) * lr);
    }
    if (nb) {
      const T txp = (T)vxp, typ = (T)vyp, txm = (T)vxm, tym = (T)vym;
      const T dIx = hxp ? txp - It : (T)0;
      const T dIy = hyp ? typ - It : (T)0;
      if (P.has_tv) {
        const T w = tv_l * (T)w_tv;
        r1 += (double)(w * sqrt(dIx * dIx + dIy * dIy));
        gr += (double)(w * tv_grade_vals<T>(It, txp, typ, txm, tym, (T)vxmyp, (T)vxpym, hxp, hyp, hxm, hym));
      }
      if (P.has_tsv) {
        const T w = tsv_l * (T)w_tsv;
        r2 += (double)(w * (dIx * dIx + dIy * dIy));
        T gt = 0;
        if (hxp) gt -= 2 * (txp - It);
        if (hyp) gt -= 2 * (typ - It);
        if (hxm) gt += 2 * (It - txm);
        if (hym) gt += 2 * (It - tym);
        gr += (double)(w * gt);
      }
    }
    if (P.has_sm) {
      const double fx = ix + 1, fy = iy + 1;
      const double xg = (fx - rm.xcen) / rm.Isum_abs, yg = (fy - rm.ycen) / rm.Isum_abs;
      const double dx = fx - rm.xcen, dy = fy - rm.ycen;
      const double s0 = ((dx * dx - 2. * xg * rm.mom[0]) - rm.Sg[0]) / rm.Isum_abs;
      const double s1 = ((dy * dy - 2. * yg * rm.mom[1]) - rm.Sg[1]) / rm.Isum_abs;
      const double s2 = (dx * dy - xg * rm.mom[1] - yg * rm.mom[0] - rm.Sg[2]) / rm.Isum_abs;
      gr += P.sm_l * (2. * (rm.Sg[0] - rm.Sp[0]) * s0 + 2. * (rm.Sg[1] - rm.Sp[1]) * s1 +
                      4. * (rm.Sg[2] - rm.Sp[2]) * s2);
    }
    const double gv = gc + gr;
    gout[p] = gv;
    if (!opt_terms) continue;  // a movie frame: the movie pass forms g.d and the projected gradient
    gdl += gv * dp;
    // projected gradient (projgr, lbfgsb.f:2942-2990) with lower bound 0
    double gi = gv;
    if (P.nonneg && gi >= 0.0) gi = fmin(I, gi);
    sbgl = fmax(sbgl, fabs(gi));
  }
  reg[0] = r0;
  reg[1] = r1;
  reg[2] = r2;
  reg[3] = r3;
  reg[4] = r4;
  gd = gdl;
  sbg = sbgl;
}

// F8: regularizer values and the full gradient g = grad chi2 + grad reg over
// pixels [lo, hi); neighbours come from the dense image grid when F1 wrote
// it in this evaluation (frames without data use the pixel map).
template <typename T>
__device__ void fg_reg_grad(const ProbDesc& P, char* base, const GroupCtx& g, const RegMoments& rm,
                            int lo, int hi, double (&reg)[8], double& gd, double& sbg,
                            bool opt_terms = true) {
  if (P.ident || (P.nuv > 0 && P.o_xg)) {
    // the dense grid: x itself on a row-major full grid, else the copy F1 wrote
    const PxGrid px{at<double>(base, P.ident ? P.o_x : P.o_xg), P.nx, P.ny};
    reg_grad_loop<T>(P, base, px, rm, lo, hi, reg, gd, sbg, opt_terms);
  } else {
    const PxMap px{at<double>(base, P.o_x), at<int>(base, P.o_inv), P.nx, P.ny};
    reg_grad_loop<T>(P, base, px, rm, lo, hi, reg, gd, sbg, opt_terms);
  }
}
