// Shared-memory mixed-radix Stockham FFT with the "+" exponent:
//   out_k = sum_j in_j exp(+2 pi i j k / n).
// Both NUFFT directions of the imaging path use this sign (FINUFFT's iflag >= 0,
// src/wrapfinufft/wrapfinufft.f90:114-124,188-202).  A CTA transforms S
// sequences of length n together; every radix pass is one sweep of n/R
// butterflies per sequence over the block, ping-ponging between two
// shared-memory buffers.  Twiddles come from a per-size table
// tw[k] = exp(+2 pi i k / n) in global memory (L1/L2 resident).
#pragma once
#include "common.cuh"

#define SMILI_MAXRAD 16

struct FftPlan {
  int n, nrad;
  int rad[SMILI_MAXRAD];
};

// radices 8, 4, 2, 3, 5 (n = 2^a 3^b 5^c)
__host__ __device__ inline FftPlan make_plan(int n) {
  FftPlan p;
  p.n = n;
  p.nrad = 0;
  int m = n;
  while (m % 8 == 0 && p.nrad < SMILI_MAXRAD) { p.rad[p.nrad++] = 8; m /= 8; }
  while (m % 4 == 0 && p.nrad < SMILI_MAXRAD) { p.rad[p.nrad++] = 4; m /= 4; }
  while (m % 2 == 0 && p.nrad < SMILI_MAXRAD) { p.rad[p.nrad++] = 2; m /= 2; }
  while (m % 3 == 0 && p.nrad < SMILI_MAXRAD) { p.rad[p.nrad++] = 3; m /= 3; }
  while (m % 5 == 0 && p.nrad < SMILI_MAXRAD) { p.rad[p.nrad++] = 5; m /= 5; }
  if (m != 1) p.nrad = -1;  // unsupported length
  return p;
}

template <typename R>
__device__ __forceinline__ void dft2(cpx<R>* v) {
  const cpx<R> a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename R>
__device__ __forceinline__ void dft4(cpx<R>& a, cpx<R>& b, cpx<R>& c, cpx<R>& d) {
  const cpx<R> s0 = cadd(a, c), s1 = csub(a, c), s2 = cadd(b, d), s3 = cmul_i(csub(b, d));
  a = cadd(s0, s2);
  c = csub(s0, s2);
  b = cadd(s1, s3);
  d = csub(s1, s3);
}

template <typename R>
__device__ __forceinline__ void dft8(cpx<R>* v) {
  // even/odd split into two length-4 transforms, w = exp(+i pi/4)
  cpx<R> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  cpx<R> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3);
  dft4(o0, o1, o2, o3);
  const R h = (R)0.70710678118654752440;
  const cpx<R> t1 = cmk(h * (o1.x - o1.y), h * (o1.x + o1.y));    // w^1 o1
  const cpx<R> t2 = cmul_i(o2);                                    // w^2 o2
  const cpx<R> t3 = cmk(-h * (o3.x + o3.y), h * (o3.x - o3.y));   // w^3 o3
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

template <typename R>
__device__ __forceinline__ void dft3(cpx<R>* v) {
  const R s = (R)0.86602540378443864676;  // sqrt(3)/2
  const cpx<R> a = v[0], t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
  const cpx<R> m = cmk(a.x - (R)0.5 * t1.x, a.y - (R)0.5 * t1.y);
  const cpx<R> it2 = cmk(-s * t2.y, s * t2.x);  // i * s * t2
  v[0] = cadd(a, t1);
  v[1] = cadd(m, it2);
  v[2] = csub(m, it2);
}

template <typename R>
__device__ __forceinline__ void dft5(cpx<R>* v) {
  // direct form with the five roots exp(+2 pi i k/5)
  const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
  const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
  const cpx<R> a = v[0];
  const cpx<R> b14 = cadd(v[1], v[4]), d14 = csub(v[1], v[4]);
  const cpx<R> b23 = cadd(v[2], v[3]), d23 = csub(v[2], v[3]);
  const cpx<R> r1 = cmk(a.x + c1 * b14.x + c2 * b23.x, a.y + c1 * b14.y + c2 * b23.y);
  const cpx<R> r2 = cmk(a.x + c2 * b14.x + c1 * b23.x, a.y + c2 * b14.y + c1 * b23.y);
  // i*(s1 d14 + s2 d23) and i*(s2 d14 - s1 d23)
  const cpx<R> q1 = cmk(-(s1 * d14.y + s2 * d23.y), s1 * d14.x + s2 * d23.x);
  const cpx<R> q2 = cmk(-(s2 * d14.y - s1 * d23.y), s2 * d14.x - s1 * d23.x);
  v[0] = cadd(a, cadd(b14, b23));
  v[1] = cadd(r1, q1);
  v[4] = csub(r1, q1);
  v[2] = cadd(r2, q2);
  v[3] = csub(r2, q2);
}

// One radix-RR pass: n/RR butterflies per sequence for S sequences, src ->
// dst, with Ns the product of the radices already applied.  RR is a
// template constant so the butterfly's values stay in registers.
template <int RR, typename R>
__device__ __forceinline__ void fft_pass(const cpx<R>* src, cpx<R>* dst, int n, int Ns, int S,
                                         const cpx<R>* __restrict__ tw) {
  const int nr = n / RR;
  const int tstep = n / (Ns * RR);
  // (s, j) = divmod(idx, nr) advanced incrementally as idx steps by
  // blockDim.x; one division per step (for k = j mod Ns) instead of three
  int s = threadIdx.x / nr, j = threadIdx.x - (threadIdx.x / nr) * nr;
  const int ds = blockDim.x / nr, dj = blockDim.x - ds * nr;
  int jq = j / Ns, k = j - jq * Ns;
  for (int idx = threadIdx.x; idx < S * nr; idx += blockDim.x) {
    const cpx<R>* in = src + (size_t)s * n;
    cpx<R> v[RR];
#pragma unroll
    for (int r = 0; r < RR; ++r) v[r] = in[j + r * nr];
    if (k) {
#pragma unroll
      for (int r = 1; r < RR; ++r) v[r] = cmul(v[r], tw[k * r * tstep]);
    }
    if constexpr (RR == 8) dft8(v);
    else if constexpr (RR == 4) dft4(v[0], v[1], v[2], v[3]);
    else if constexpr (RR == 2) dft2(v);
    else if constexpr (RR == 3) dft3(v);
    else dft5(v);
    cpx<R>* out = dst + (size_t)s * n + jq * Ns * RR + k;
#pragma unroll
    for (int r = 0; r < RR; ++r) out[r * Ns] = v[r];
    // advance to idx + blockDim.x
    s += ds;
    j += dj;
    if (j >= nr) {
      j -= nr;
      ++s;
    }
    jq = j / Ns;  // Ns is a power of the radices; one division per step
    k = j - jq * Ns;
  }
}

// Transform S sequences (buf[s*n + i]) in shared memory; returns the buffer
// that holds the result (buf or work).  All threads of the block must call.
template <typename R>
__device__ cpx<R>* smem_fft(cpx<R>* buf, cpx<R>* work, const FftPlan& pl, int S,
                            const cpx<R>* __restrict__ tw) {
  cpx<R>* src = buf;
  cpx<R>* dst = work;
  const int n = pl.n;
  int Ns = 1;
  for (int p = 0; p < pl.nrad; ++p) {
    const int Rr = pl.rad[p];
    switch (Rr) {
      case 8: fft_pass<8>(src, dst, n, Ns, S, tw); break;
      case 4: fft_pass<4>(src, dst, n, Ns, S, tw); break;
      case 2: fft_pass<2>(src, dst, n, Ns, S, tw); break;
      case 3: fft_pass<3>(src, dst, n, Ns, S, tw); break;
      default: fft_pass<5>(src, dst, n, Ns, S, tw); break;
    }
    __syncthreads();
    cpx<R>* t = src;
    src = dst;
    dst = t;
    Ns *= Rr;
  }
  return src;
}
