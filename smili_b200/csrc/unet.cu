// BF16 kernels of the warm-start U-Net (no reference counterpart).
//
// Activations are NHWC bf16 with an explicit channel stride (`ld`), so a
// layer can read or write a channel slice of a wider buffer: the decoder's
// concatenation of the upsampled path and the encoder skip is one buffer
// that two producers write into, with no copy.  Weights are [Cout][3][3][Cin]
// bf16 (FP32 master copies live with the optimiser).  Every contraction
// accumulates in FP32 on the tensor cores (mma.sync m16n8k16 bf16).
//
// conv3x3 (pad 1, stride 1) is an implicit GEMM: D[pixel][cout] =
// sum over (ky, kx, cin) of X[pixel + (ky-1, kx-1)][cin] W[cout][ky][kx][cin].
// A CTA owns an 8 x 16 pixel tile (one m16 row block per warp) and a chunk of
// 8*NT output channels; it stages a (8+2) x (16+2) input halo and the weight
// slab of one 16-channel input chunk in shared memory at a time.
// The data gradient is the same kernel on the ReLU-masked output gradient
// with flipped, transposed weights; the weight gradient is a second
// implicit GEMM over pixels with deterministic per-split partial sums.
// Convolutions whose input rows and weights TMA can address (Cin and the
// channel stride multiples of 8, 16-byte aligned bases) run instead on the
// tcgen05 tensor cores with the accumulator in tensor memory (conv_tc.cuh),
// and so do weight gradients whose channel counts and strides are multiples
// of 8; the mma.sync kernels below take the rest (the one-channel input and
// output layers).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/smili_unet.h"
#include "conv_tc.cuh"

namespace {

constexpr int TH = 8, TW = 16;          // pixel tile of one CTA
constexpr int KC = 16;                  // input channels per staged chunk
constexpr int KP = KC + 8;              // padded channel stride in shared memory (conflict-free)
constexpr int HALO_H = TH + 2, HALO_W = TW + 2;

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// ---------------------------------------------------------------------------
// conv3x3 forward / data-gradient
// ---------------------------------------------------------------------------
struct ConvArgs {
  const __nv_bfloat16* x;
  int N, H, W, Cin, ldx;
  const __nv_bfloat16* w;  // [Cout][3][3][Cin]
  const float* bias;       // [Cout] or null
  __nv_bfloat16* y;
  int ldy, Cout;
  int relu, accumulate;
  int tiles_x, tiles_y;
};

template <int NT>
__global__ void __launch_bounds__(256) conv3x3_kernel(ConvArgs a) {
  __shared__ __align__(16) __nv_bfloat16 halo[HALO_H * HALO_W * KP];
  __shared__ __align__(16) __nv_bfloat16 wsm[NT * 8 * 9 * KP];
  const int tile = blockIdx.x;
  const int tx = tile % a.tiles_x;
  const int ty = (tile / a.tiles_x) % a.tiles_y;
  const int n = tile / (a.tiles_x * a.tiles_y);
  const int x0 = tx * TW, y0 = ty * TH;
  const int co0 = blockIdx.y * NT * 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  float acc[NT][4];
#pragma unroll
  for (int i = 0; i < NT; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  const bool vec = (a.Cin % 8 == 0) && (a.ldx % 8 == 0) && ((reinterpret_cast<uintptr_t>(a.x) & 15) == 0);
  const bool wvec = (a.Cin % 8 == 0) && ((reinterpret_cast<uintptr_t>(a.w) & 15) == 0);
  for (int ci0 = 0; ci0 < a.Cin; ci0 += KC) {
    __syncthreads();
    // input halo: HALO_H x HALO_W pixels x KC channels (zero outside the image / channels)
    if (vec) {
      for (int q = threadIdx.x; q < HALO_H * HALO_W * 2; q += blockDim.x) {
        const int pix = q >> 1, half = q & 1;
        const int hy = pix / HALO_W, hx = pix - hy * HALO_W;
        const int iy = y0 + hy - 1, ix = x0 + hx - 1;
        const int c = ci0 + half * 8;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (iy >= 0 && iy < a.H && ix >= 0 && ix < a.W && c < a.Cin)
          v = *reinterpret_cast<const uint4*>(a.x + (((size_t)n * a.H + iy) * a.W + ix) * a.ldx + c);
        *reinterpret_cast<uint4*>(halo + pix * KP + half * 8) = v;
      }
    } else {
      for (int q = threadIdx.x; q < HALO_H * HALO_W * KC; q += blockDim.x) {
        const int pix = q / KC, c = q - pix * KC;
        const int hy = pix / HALO_W, hx = pix - hy * HALO_W;
        const int iy = y0 + hy - 1, ix = x0 + hx - 1;
        __nv_bfloat16 v = zero;
        if (iy >= 0 && iy < a.H && ix >= 0 && ix < a.W && ci0 + c < a.Cin)
          v = a.x[(((size_t)n * a.H + iy) * a.W + ix) * a.ldx + ci0 + c];
        halo[pix * KP + c] = v;
      }
    }
    // weights: (NT*8) output channels x 9 taps x KC input channels
    if (wvec) {
      for (int q = threadIdx.x; q < NT * 8 * 9 * 2; q += blockDim.x) {
        const int row = q >> 1, half = q & 1;  // row = co_local * 9 + tap
        const int col = row / 9, tap = row - col * 9;
        const int co = co0 + col, c = ci0 + half * 8;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (co < a.Cout && c < a.Cin)
          v = *reinterpret_cast<const uint4*>(a.w + ((size_t)co * 9 + tap) * a.Cin + c);
        *reinterpret_cast<uint4*>(wsm + row * KP + half * 8) = v;
      }
    } else {
      for (int q = threadIdx.x; q < NT * 8 * 9 * KC; q += blockDim.x) {
        const int row = q / KC, c = q - row * KC;
        const int col = row / 9, tap = row - col * 9;
        const int co = co0 + col;
        __nv_bfloat16 v = zero;
        if (co < a.Cout && ci0 + c < a.Cin) v = a.w[((size_t)co * 9 + tap) * a.Cin + ci0 + c];
        wsm[row * KP + c] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int ky = tap / 3, kx = tap - ky * 3;
      const __nv_bfloat16* hrow = halo + ((warp + ky) * HALO_W + kx) * KP;
      uint32_t af[4];
      af[0] = ld32(hrow + g * KP + 2 * t);
      af[1] = ld32(hrow + (g + 8) * KP + 2 * t);
      af[2] = ld32(hrow + g * KP + 2 * t + 8);
      af[3] = ld32(hrow + (g + 8) * KP + 2 * t + 8);
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const __nv_bfloat16* wrow = wsm + ((nt * 8 + g) * 9 + tap) * KP;
        mma_bf16(acc[nt], af, ld32(wrow + 2 * t), ld32(wrow + 2 * t + 8));
      }
    }
  }
  // epilogue: bias, ReLU, bf16 store (optionally accumulating)
  const int oy = y0 + warp;
  if (oy >= a.H) return;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
#pragma unroll
    for (int hlf = 0; hlf < 2; ++hlf) {
      const int ox = x0 + g + hlf * 8;
      if (ox >= a.W) continue;
      __nv_bfloat16* dst = a.y + (((size_t)n * a.H + oy) * a.W + ox) * a.ldy;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int co = co0 + nt * 8 + 2 * t + e;
        if (co >= a.Cout) continue;
        float v = acc[nt][hlf * 2 + e];
        if (a.bias) v += a.bias[co];
        if (a.relu) v = fmaxf(v, 0.f);
        if (a.accumulate) v += __bfloat162float(dst[co]);
        dst[co] = __float2bfloat16(v);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// conv3x3 weight gradient: dW[co][tap][ci] = sum_p dY[p][co] X[p + s(tap)][ci]
// A = dY^T (co x pixels), B = shifted X (pixels x ci); one k16 step is one
// tile row of 16 pixels.  A CTA owns 64 output x 16 input channels for all 9
// taps (warp w: co block w%4, ci block w/4) and loops over the pixel tiles
// of its split; each split writes its own partial (deterministic sum later).
// ---------------------------------------------------------------------------
struct WgradArgs {
  const __nv_bfloat16* x;
  int ldx;
  const __nv_bfloat16* dy;
  int lddy;
  int N, H, W, Cin, Cout;
  int tiles_x, tiles_y, ntiles, nsplit;
  float* partial;  // [nsplit][Cout][9][Cin]
};

__global__ void __launch_bounds__(256) conv3x3_wgrad_kernel(WgradArgs a) {
  __shared__ __align__(16) __nv_bfloat16 xt[KC * HALO_H * HALO_W];  // [ci][pixel]
  __shared__ __align__(16) __nv_bfloat16 dyt[64 * TH * TW];         // [co][pixel]
  const int split = blockIdx.x;
  const int co0 = blockIdx.y * 64, ci0 = blockIdx.z * KC;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int mb = warp & 3, nb = warp >> 2;  // 16 co x 8 ci block of this warp
  float acc[9][4];
#pragma unroll
  for (int i = 0; i < 9; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  for (int tile = split; tile < a.ntiles; tile += a.nsplit) {
    const int tx = tile % a.tiles_x;
    const int ty = (tile / a.tiles_x) % a.tiles_y;
    const int n = tile / (a.tiles_x * a.tiles_y);
    const int x0 = tx * TW, y0 = ty * TH;
    __syncthreads();
    for (int q = threadIdx.x; q < KC * HALO_H * HALO_W; q += blockDim.x) {
      const int pix = q / KC, c = q - pix * KC;
      const int hy = pix / HALO_W, hx = pix - hy * HALO_W;
      const int iy = y0 + hy - 1, ix = x0 + hx - 1;
      __nv_bfloat16 v = zero;
      if (iy >= 0 && iy < a.H && ix >= 0 && ix < a.W && ci0 + c < a.Cin)
        v = a.x[(((size_t)n * a.H + iy) * a.W + ix) * a.ldx + ci0 + c];
      xt[c * (HALO_H * HALO_W) + pix] = v;
    }
    for (int q = threadIdx.x; q < 64 * TH * TW; q += blockDim.x) {
      const int pix = q / 64, c = q - pix * 64;
      const int py = pix / TW, px = pix - py * TW;
      const int iy = y0 + py, ix = x0 + px;
      __nv_bfloat16 v = zero;
      if (iy < a.H && ix < a.W && co0 + c < a.Cout)
        v = a.dy[(((size_t)n * a.H + iy) * a.W + ix) * a.lddy + co0 + c];
      dyt[c * (TH * TW) + pix] = v;
    }
    __syncthreads();
    for (int r = 0; r < TH; ++r) {
      // A fragment: rows co (mb*16 + g, +8), k = pixel x of tile row r
      const __nv_bfloat16* arow = dyt + r * TW;
      uint32_t af[4];
      af[0] = ld32(arow + (mb * 16 + g) * (TH * TW) + 2 * t);
      af[1] = ld32(arow + (mb * 16 + g + 8) * (TH * TW) + 2 * t);
      af[2] = ld32(arow + (mb * 16 + g) * (TH * TW) + 2 * t + 8);
      af[3] = ld32(arow + (mb * 16 + g + 8) * (TH * TW) + 2 * t + 8);
      const __nv_bfloat16* bcol = xt + (nb * 8 + g) * (HALO_H * HALO_W);
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int ky = tap / 3, kx = tap - ky * 3;
        const __nv_bfloat16* b = bcol + (r + ky) * HALO_W + kx;
        const uint32_t b0 = pack2(b[2 * t], b[2 * t + 1]);
        const uint32_t b1 = pack2(b[2 * t + 8], b[2 * t + 9]);
        mma_bf16(acc[tap], af, b0, b1);
      }
    }
  }
  float* out = a.partial + (size_t)split * a.Cout * 9 * a.Cin;
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
#pragma unroll
    for (int hlf = 0; hlf < 2; ++hlf) {
      const int co = co0 + mb * 16 + g + hlf * 8;
      if (co >= a.Cout) continue;
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int ci = ci0 + nb * 8 + 2 * t + e;
        if (ci < a.Cin) out[((size_t)co * 9 + tap) * a.Cin + ci] = acc[tap][hlf * 2 + e];
      }
    }
  }
}

// sum the split partials in a fixed order: dw (+)= sum_s partial[s]
__global__ void sum_partials_kernel(const float* partial, int nsplit, size_t count, float* dw, int accumulate) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int k = 0; k < nsplit; ++k) s += partial[(size_t)k * count + i];
    dw[i] = accumulate ? dw[i] + s : s;
  }
}

// bias gradient: db[c] (+)= sum over pixels of dy[p][c] (fixed order per channel)
__global__ void bias_grad_kernel(const __nv_bfloat16* dy, int ld, size_t npix, int C, float* db, int accumulate) {
  __shared__ float red[256];
  const int c = blockIdx.x;
  float s = 0.f;
  for (size_t p = threadIdx.x; p < npix; p += blockDim.x) s += __bfloat162float(dy[p * ld + c]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = accumulate ? db[c] + red[0] : red[0];
}

// wt[ci][ky][kx][co] = w[co][2-ky][2-kx][ci]
__global__ void flip_weights_kernel(const __nv_bfloat16* w, __nv_bfloat16* wt, int Cout, int Cin) {
  const size_t total = (size_t)Cout * 9 * Cin;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin);
    const int tap = (int)((i / Cin) % 9);
    const int co = (int)(i / ((size_t)Cin * 9));
    wt[((size_t)ci * 9 + (8 - tap)) * Cout + co] = w[i];
  }
}

// dy *= (y > 0) over an N*H*W x C slice
__global__ void relu_mask_kernel(const __nv_bfloat16* y, int ldy, __nv_bfloat16* dy, int lddy, size_t npix, int C) {
  const size_t total = npix * C;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t p = i / C;
    const int c = (int)(i - p * C);
    if (!(__bfloat162float(y[p * ldy + c]) > 0.f)) dy[p * lddy + c] = __float2bfloat16(0.f);
  }
}

// 2x2 average pooling (H, W even) and its gradient
__global__ void avgpool2_kernel(const __nv_bfloat16* x, int ldx, __nv_bfloat16* y, int ldy, int N, int H, int W,
                                int C) {
  const int Ho = H / 2, Wo = W / 2;
  const size_t total = (size_t)N * Ho * Wo * C;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    size_t p = i / C;
    const int ox = (int)(p % Wo);
    p /= Wo;
    const int oy = (int)(p % Ho);
    const int n = (int)(p / Ho);
    const size_t b = ((size_t)n * H + 2 * oy) * W + 2 * ox;
    const float s = __bfloat162float(x[b * ldx + c]) + __bfloat162float(x[(b + 1) * ldx + c]) +
                    __bfloat162float(x[(b + W) * ldx + c]) + __bfloat162float(x[(b + W + 1) * ldx + c]);
    y[(((size_t)n * Ho + oy) * Wo + ox) * ldy + c] = __float2bfloat16(0.25f * s);
  }
}

__global__ void avgpool2_bwd_kernel(const __nv_bfloat16* dy, int lddy, __nv_bfloat16* dx, int lddx, int N, int H,
                                    int W, int C, int accumulate) {
  const size_t total = (size_t)N * H * W * C;
  const int Wo = W / 2, Ho = H / 2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    size_t p = i / C;
    const int ix = (int)(p % W);
    p /= W;
    const int iy = (int)(p % H);
    const int n = (int)(p / H);
    float v = 0.25f * __bfloat162float(dy[(((size_t)n * Ho + iy / 2) * Wo + ix / 2) * lddy + c]);
    __nv_bfloat16* d = dx + (((size_t)n * H + iy) * W + ix) * lddx + c;
    if (accumulate) v += __bfloat162float(*d);
    *d = __float2bfloat16(v);
  }
}

// nearest-neighbour 2x upsampling and its gradient (sum of the 4 children)
__global__ void upsample2_kernel(const __nv_bfloat16* x, int ldx, __nv_bfloat16* y, int ldy, int N, int H, int W,
                                 int C) {
  const int Ho = 2 * H, Wo = 2 * W;
  const size_t total = (size_t)N * Ho * Wo * C;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    size_t p = i / C;
    const int ox = (int)(p % Wo);
    p /= Wo;
    const int oy = (int)(p % Ho);
    const int n = (int)(p / Ho);
    y[(((size_t)n * Ho + oy) * Wo + ox) * ldy + c] = x[(((size_t)n * H + oy / 2) * W + ox / 2) * ldx + c];
  }
}

__global__ void upsample2_bwd_kernel(const __nv_bfloat16* dy, int lddy, __nv_bfloat16* dx, int lddx, int N, int H,
                                     int W, int C, int accumulate) {
  const size_t total = (size_t)N * H * W * C;
  const int Wo = 2 * W;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    size_t p = i / C;
    const int ix = (int)(p % W);
    p /= W;
    const int iy = (int)(p % H);
    const int n = (int)(p / H);
    const size_t b = ((size_t)n * 2 * H + 2 * iy) * Wo + 2 * ix;
    float v = __bfloat162float(dy[b * lddy + c]) + __bfloat162float(dy[(b + 1) * lddy + c]) +
              __bfloat162float(dy[(b + Wo) * lddy + c]) + __bfloat162float(dy[(b + Wo + 1) * lddy + c]);
    __nv_bfloat16* d = dx + (((size_t)n * H + iy) * W + ix) * lddx + c;
    if (accumulate) v += __bfloat162float(*d);
    *d = __float2bfloat16(v);
  }
}

// mean squared error of a 1-channel output against an FP32 target:
// loss_part[block] = sum (y - t)^2 over the block's pixels; dy = 2 (y - t) / n
__global__ void mse_kernel(const __nv_bfloat16* y, int ldy, const float* target, size_t n, __nv_bfloat16* dy,
                           int lddy, float* loss_part) {
  __shared__ float red[256];
  float s = 0.f;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float r = __bfloat162float(y[i * ldy]) - target[i];
    s += r * r;
    dy[i * lddy] = __float2bfloat16(2.f * r / (float)n);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss_part[blockIdx.x] = red[0];
}

// Adam with decoupled weight decay on FP32 master weights; writes the bf16 copy
__global__ void adam_kernel(float* w, __nv_bfloat16* w16, const float* g, float* m, float* v, size_t n, float lr,
                            float b1, float b2, float eps, float wd, float bc1, float bc2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = (mi / bc1) / (sqrtf(vi / bc2) + eps);
    const float wi = w[i] * (1.f - lr * wd) - lr * upd;
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
  }
}

__global__ void f32_to_bf16_kernel(const float* x, __nv_bfloat16* y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

// 0: tensor-core (tcgen05) path where it applies, else mma.sync; 1: always
// mma.sync; 2: tcgen05 with one 128-pixel tile per CTA (for comparisons)
int g_conv_path = 0;

int grid_for(size_t n, int block = 256) {
  size_t g = (n + block - 1) / block;
  if (g > 148 * 32) g = 148 * 32;
  return (int)(g < 1 ? 1 : g);
}

int check_launch() {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : SMILI_UNET_ERR_CUDA;
}

}  // namespace

extern "C" {

int smili_unet_conv3x3(const void* x, int N, int H, int W, int Cin, int ldx, const void* w, const float* bias,
                       void* y, int ldy, int Cout, int relu, int accumulate, void* stream) {
  if (!x || !w || !y || N < 1 || H < 1 || W < 1 || Cin < 1 || Cout < 1 || ldx < Cin || ldy < Cout)
    return SMILI_UNET_ERR_ARG;
  ConvArgs a;
  a.x = static_cast<const __nv_bfloat16*>(x);
  a.N = N;
  a.H = H;
  a.W = W;
  a.Cin = Cin;
  a.ldx = ldx;
  a.w = static_cast<const __nv_bfloat16*>(w);
  a.bias = bias;
  a.y = static_cast<__nv_bfloat16*>(y);
  a.ldy = ldy;
  a.Cout = Cout;
  a.relu = relu;
  a.accumulate = accumulate;
  a.tiles_x = (W + TW - 1) / TW;
  a.tiles_y = (H + TH - 1) / TH;
  const long long tiles = (long long)a.tiles_x * a.tiles_y * N;
  if (tiles > 0x7fffffffLL) return SMILI_UNET_ERR_ARG;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g_conv_path != 1 && tc::eligible(x, Cin, ldx, w, Cout))
    return tc::launch(a.x, N, H, W, Cin, ldx, a.w, bias, a.y, ldy, Cout, relu, accumulate, s,
                      g_conv_path == 2 ? 1 : 2) == 0
               ? 0
               : SMILI_UNET_ERR_CUDA;
  if (Cout <= 8) {
    conv3x3_kernel<1><<<dim3((unsigned)tiles, 1), 256, 0, s>>>(a);
  } else if (Cout <= 16) {
    conv3x3_kernel<2><<<dim3((unsigned)tiles, 1), 256, 0, s>>>(a);
  } else if (Cout <= 32) {
    conv3x3_kernel<4><<<dim3((unsigned)tiles, 1), 256, 0, s>>>(a);
  } else {
    conv3x3_kernel<8><<<dim3((unsigned)tiles, (Cout + 63) / 64), 256, 0, s>>>(a);
  }
  return check_launch();
}

int smili_unet_conv3x3_wgrad(const void* x, int ldx, const void* dy, int lddy, int N, int H, int W, int Cin,
                             int Cout, float* partial, int nsplit, float* dw, int accumulate, void* stream) {
  if (!x || !dy || !partial || !dw || N < 1 || H < 1 || W < 1 || Cin < 1 || Cout < 1 || nsplit < 1 || ldx < Cin ||
      lddy < Cout)
    return SMILI_UNET_ERR_ARG;
  WgradArgs a;
  a.x = static_cast<const __nv_bfloat16*>(x);
  a.ldx = ldx;
  a.dy = static_cast<const __nv_bfloat16*>(dy);
  a.lddy = lddy;
  a.N = N;
  a.H = H;
  a.W = W;
  a.Cin = Cin;
  a.Cout = Cout;
  a.tiles_x = (W + TW - 1) / TW;
  a.tiles_y = (H + TH - 1) / TH;
  a.ntiles = a.tiles_x * a.tiles_y * N;
  a.nsplit = nsplit;
  a.partial = partial;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (g_conv_path != 1 && tc::wgrad_eligible(x, ldx, dy, lddy, Cin, Cout)) {
    if (tc::launch_wgrad(a.x, ldx, a.dy, lddy, N, H, W, Cin, Cout, partial, nsplit, s) != 0)
      return SMILI_UNET_ERR_CUDA;
  } else {
    conv3x3_wgrad_kernel<<<dim3(nsplit, (Cout + 63) / 64, (Cin + KC - 1) / KC), 256, 0, s>>>(a);
  }
  const size_t count = (size_t)Cout * 9 * Cin;
  sum_partials_kernel<<<grid_for(count), 256, 0, s>>>(partial, nsplit, count, dw, accumulate);
  return check_launch();
}

int smili_unet_bias_grad(const void* dy, int ld, long long npix, int C, float* db, int accumulate, void* stream) {
  if (!dy || !db || npix < 1 || C < 1 || ld < C) return SMILI_UNET_ERR_ARG;
  bias_grad_kernel<<<C, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(dy), ld,
                                                                      (size_t)npix, C, db, accumulate);
  return check_launch();
}

int smili_unet_flip_weights(const void* w, void* wt, int Cout, int Cin, void* stream) {
  if (!w || !wt || Cout < 1 || Cin < 1) return SMILI_UNET_ERR_ARG;
  flip_weights_kernel<<<grid_for((size_t)Cout * 9 * Cin), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(w), static_cast<__nv_bfloat16*>(wt), Cout, Cin);
  return check_launch();
}

int smili_unet_relu_mask(const void* y, int ldy, void* dy, int lddy, long long npix, int C, void* stream) {
  if (!y || !dy || npix < 1 || C < 1 || ldy < C || lddy < C) return SMILI_UNET_ERR_ARG;
  relu_mask_kernel<<<grid_for((size_t)npix * C), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(y), ldy, static_cast<__nv_bfloat16*>(dy), lddy, (size_t)npix, C);
  return check_launch();
}

int smili_unet_avgpool2(const void* x, int ldx, void* y, int ldy, int N, int H, int W, int C, void* stream) {
  if (!x || !y || N < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || ldx < C || ldy < C)
    return SMILI_UNET_ERR_ARG;
  avgpool2_kernel<<<grid_for((size_t)N * H * W * C / 4), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), ldx, static_cast<__nv_bfloat16*>(y), ldy, N, H, W, C);
  return check_launch();
}

int smili_unet_avgpool2_bwd(const void* dy, int lddy, void* dx, int lddx, int N, int H, int W, int C,
                            int accumulate, void* stream) {
  if (!dy || !dx || N < 1 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || lddx < C || lddy < C)
    return SMILI_UNET_ERR_ARG;
  avgpool2_bwd_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(dy), lddy, static_cast<__nv_bfloat16*>(dx), lddx, N, H, W, C, accumulate);
  return check_launch();
}

int smili_unet_upsample2(const void* x, int ldx, void* y, int ldy, int N, int H, int W, int C, void* stream) {
  if (!x || !y || N < 1 || H < 1 || W < 1 || C < 1 || ldx < C || ldy < C) return SMILI_UNET_ERR_ARG;
  upsample2_kernel<<<grid_for((size_t)N * H * W * C * 4), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(x), ldx, static_cast<__nv_bfloat16*>(y), ldy, N, H, W, C);
  return check_launch();
}

int smili_unet_upsample2_bwd(const void* dy, int lddy, void* dx, int lddx, int N, int H, int W, int C,
                             int accumulate, void* stream) {
  if (!dy || !dx || N < 1 || H < 1 || W < 1 || C < 1 || lddx < C || lddy < C) return SMILI_UNET_ERR_ARG;
  upsample2_bwd_kernel<<<grid_for((size_t)N * H * W * C), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(dy), lddy, static_cast<__nv_bfloat16*>(dx), lddx, N, H, W, C, accumulate);
  return check_launch();
}

int smili_unet_mse(const void* y, int ldy, const float* target, long long n, void* dy, int lddy, float* loss_part,
                   int nblocks, void* stream) {
  if (!y || !target || !dy || !loss_part || n < 1 || nblocks < 1 || ldy < 1 || lddy < 1) return SMILI_UNET_ERR_ARG;
  mse_kernel<<<nblocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(y), ldy,
                                                                      target, (size_t)n,
                                                                      static_cast<__nv_bfloat16*>(dy), lddy,
                                                                      loss_part);
  return check_launch();
}

int smili_unet_adam(float* w, void* w16, const float* g, float* m, float* v, long long n, float lr, float b1,
                    float b2, float eps, float wd, int step, void* stream) {
  if (!w || !g || !m || !v || n < 1 || step < 1) return SMILI_UNET_ERR_ARG;
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<grid_for((size_t)n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      w, static_cast<__nv_bfloat16*>(w16), g, m, v, (size_t)n, lr, b1, b2, eps, wd, bc1, bc2);
  return check_launch();
}

int smili_unet_set_conv_path(int path) {
  if (path < 0 || path > 2) return SMILI_UNET_ERR_ARG;
  g_conv_path = path;
  return 0;
}

const char* smili_unet_last_error(void) { return tc::last_error().c_str(); }

int smili_unet_tc_status(void) {
  int e = 0;
  if (cudaMemcpyFromSymbol(&e, tc::g_tc_err, sizeof(int)) != cudaSuccess) return SMILI_UNET_ERR_CUDA;
  if (e) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(tc::g_tc_err, &zero, sizeof(int)) != cudaSuccess) return SMILI_UNET_ERR_CUDA;
  }
  return e;
}

int smili_unet_f32_to_bf16(const float* x, void* y, long long n, void* stream) {
  if (!x || !y || n < 1) return SMILI_UNET_ERR_ARG;
  f32_to_bf16_kernel<<<grid_for((size_t)n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      x, static_cast<__nv_bfloat16*>(y), (size_t)n);
  return check_launch();
}

}  // extern "C"
