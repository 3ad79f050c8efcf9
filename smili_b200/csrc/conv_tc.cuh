// conv3x3 (pad 1, stride 1) on the fifth-generation tensor cores: tcgen05.mma
// with the accumulator in tensor memory, operands staged by TMA.
//
// Implicit GEMM D[pixel][cout] = sum over (tap, cin) of X[pixel + s(tap)][cin]
// W[cout][tap][cin] with one CTA per tile of 128 output pixels (8 rows x 16
// columns of one image), or two such tiles stacked (16 x 16 pixels, two
// accumulators sharing each weight stage), and up to 256 output channels:
//
// - A (128 pixels x 16 input channels, bf16, K-major) is one TMA box of the
//   NHWC input viewed as a 4-D tensor (C, W, H, N) at (cin0, x0 + kx - 1,
//   y0 + ky - 1, n).  Pixels outside the image and channels past Cin come in
//   as zeros (TMA out-of-bounds fill), which is the zero padding; the
//   innermost coordinate cin0 is a multiple of 16 channels (32 bytes).
// - B (ntile output channels x 16 input channels, K-major) is one TMA box of
//   the weights viewed as (Cin, 9, Cout) at (cin0, tap, cout0).
// - Both land in shared memory with the 32-byte swizzle, which is the
//   canonical K-major SWIZZLE_32B layout of the UMMA descriptors (8-row
//   atoms of 256 bytes).  One tcgen05.mma (M 128, N ntile, K 16) consumes a
//   stage; 9 * ceil(Cin / 16) of them accumulate into ntile FP32 columns of
//   tensor memory.
//
// Warp roles: lane 0 of warp 0 issues the TMA loads into a ring of STAGES
// stages; lane 0 of warp 1 issues the MMAs and releases each stage with
// tcgen05.commit; warp 2 allocates and frees the tensor memory.  All four
// warps then read the accumulator (warp w owns lanes 32w..32w+31, i.e.
// pixels 32w..32w+31 of the tile) and apply bias, ReLU and the optional
// accumulation into the bf16 output.
//
// Every wait on an mbarrier is bounded.  A wait that runs out records a
// code in g_tc_err (smili_unet_tc_status reads and clears it), the role
// stops issuing, outstanding copies are waited for (again bounded) and the
// tensor memory is freed before the CTA exits.  No load here reads another
// GPU's memory, and none uses cluster multicast.
#include <cuda.h>

#include <mutex>
#include <string>

namespace tc {

constexpr int TILE_H = 8, TILE_W = 16, BM = TILE_H * TILE_W;  // 128 pixels: the UMMA M
constexpr int KCH = 16;                                        // input channels per stage (one UMMA K)
constexpr int STAGES = 8;
constexpr uint32_t A_BYTES = BM * KCH * 2;                      // 4096
constexpr uint32_t kSpinLimit = 1u << 21;                       // polls of one bounded wait

__device__ int g_tc_err;  // first error code of a bounded wait that ran out (0: none)

struct Params {
  int H, W, Cin, Cout, ldy, relu, accumulate;
  int tiles_x, tiles_y;
  int msub;     // 128-pixel sub-tiles per CTA (1 or 2): one accumulator each (the second at column
                // tmem_cols / 2), sharing every B stage
  int ntile;    // UMMA N: output channels per CTA (multiple of 16, <= 256)
  int tmem_cols;
  int kiters;   // 9 * ceil(Cin / 16)
  const float* bias;
  __nv_bfloat16* y;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for the phase with the given parity to complete; gives up
// early once any CTA has recorded an error
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
  for (uint32_t i = 0; i < kSpinLimit; ++i) {
    if (mbar_try_wait(b, parity)) return true;
    if ((i & 1023u) == 1023u && *reinterpret_cast<volatile int*>(&g_tc_err) != 0) return false;
  }
  return false;
}

__device__ __forceinline__ void set_err(int code) { atomicCAS(&g_tc_err, 0, code); }

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, "
      "%6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

// K-major operand in the 32-byte swizzle: rows of 32 bytes (16 bf16 of K),
// 8-row atoms 256 bytes apart (stride byte offset), descriptor version 1,
// layout type 6 (SWIZZLE_32B).  The leading byte offset is unused for a
// swizzled K-major operand and set to 1.
__device__ __forceinline__ uint64_t sdesc_k_sw32(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major,
// N = ntile, M = 128
__host__ __device__ constexpr uint32_t idesc_bf16(int ntile) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(ntile >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(128) conv3x3_tc_kernel(const __grid_constant__ CUtensorMap tmx,
                                                         const __grid_constant__ CUtensorMap tmw, Params p) {
  extern __shared__ unsigned char dyn_raw[];
  __shared__ __align__(8) uint64_t full_bar[STAGES], empty_bar[STAGES], done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int consumed;
  // 1024-byte aligned ring: STAGES A tiles, then STAGES B tiles
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dyn_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t b_bytes = (uint32_t)p.ntile * KCH * 2;
  const uint32_t a_bytes = A_BYTES * (uint32_t)p.msub;
  unsigned char* a_ring = base;
  unsigned char* b_ring = base + STAGES * a_bytes;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tile = blockIdx.x;
  const int tx = tile % p.tiles_x;
  const int ty = (tile / p.tiles_x) % p.tiles_y;
  const int n = tile / (p.tiles_x * p.tiles_y);
  const int x0 = tx * TILE_W, y0 = ty * TILE_H * p.msub;
  const int co0 = blockIdx.y * p.ntile;
  const int cchunks = (p.Cin + KCH - 1) / KCH;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"((uint32_t)p.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_slot;

  int issued = 0;
  if (warp == 0 && lane == 0) {
    // producer: TMA loads of A and B for k = 0 .. kiters-1 into stage k % STAGES
    for (int k = 0; k < p.kiters; ++k) {
      const int s = k % STAGES;
      if (k >= STAGES && !mbar_wait(&empty_bar[s], ((k / STAGES) - 1) & 1)) {
        set_err(1);
        break;
      }
      const int tap = k / cchunks, ci0 = (k - tap * cchunks) * KCH;
      const int ky = tap / 3, kx = tap - ky * 3;
      mbar_expect_tx(&full_bar[s], a_bytes + b_bytes);
      tma_load_4d(a_ring + s * a_bytes, &tmx, &full_bar[s], ci0, x0 + kx - 1, y0 + ky - 1, n);
      tma_load_3d(b_ring + s * b_bytes, &tmw, &full_bar[s], ci0, tap, co0);
      issued = k + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // MMA issuer
    const uint32_t idesc = idesc_bf16(p.ntile);
    int k = 0;
    for (; k < p.kiters; ++k) {
      const int s = k % STAGES;
      if (!mbar_wait(&full_bar[s], (k / STAGES) & 1)) {
        set_err(2);
        break;
      }
      fence_after();
      const uint64_t bdesc = sdesc_k_sw32(smem_u32(b_ring + s * b_bytes));
      for (int sub = 0; sub < p.msub; ++sub)  // sub-tile sub: A rows 128 sub .., accumulator at column half sub
        umma_bf16(tmem + (uint32_t)(sub * (p.tmem_cols / 2)),
                  sdesc_k_sw32(smem_u32(a_ring + s * a_bytes + sub * A_BYTES)), bdesc, idesc, k > 0 ? 1u : 0u);
      umma_commit(&empty_bar[s]);
    }
    consumed = k;
    umma_commit(&done_bar);  // arrives once every MMA issued above has completed
  }
  __syncwarp();
  if (!mbar_wait(&done_bar, 0)) set_err(3);
  fence_after();
  __syncthreads();
  if (warp == 0 && lane == 0) {
    // copies issued but never consumed (only after an error): wait for them
    for (int k = consumed; k < issued; ++k)
      if (!mbar_wait(&full_bar[k % STAGES], (k / STAGES) & 1)) set_err(4);
  }

  // epilogue: warp w reads the accumulator rows (pixels) 32w .. 32w+31 of
  // each sub-tile
  const bool vec = (p.ldy % 8 == 0) && ((reinterpret_cast<uintptr_t>(p.y) & 15) == 0) && ((co0 & 7) == 0);
  for (int sub = 0; sub < p.msub; ++sub) {
  const int r = warp * 32 + lane;
  const int oy = y0 + sub * TILE_H + r / TILE_W, ox = x0 + r % TILE_W;
  const bool in = oy < p.H && ox < p.W;
  __nv_bfloat16* dst = p.y + (((size_t)n * p.H + (in ? oy : 0)) * p.W + (in ? ox : 0)) * p.ldy;
  for (int c = 0; c < p.ntile; c += 16) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(sub * (p.tmem_cols / 2) + c), v);
    if (!in) continue;
    if (vec && co0 + c + 16 <= p.Cout) {
      uint4 old[2] = {make_uint4(0, 0, 0, 0), make_uint4(0, 0, 0, 0)};
      if (p.accumulate) {
        old[0] = *reinterpret_cast<const uint4*>(dst + co0 + c);
        old[1] = *reinterpret_cast<const uint4*>(dst + co0 + c + 8);
      }
      const __nv_bfloat16* ob = reinterpret_cast<const __nv_bfloat16*>(old);
      uint4 out[2];
      __nv_bfloat16* o = reinterpret_cast<__nv_bfloat16*>(out);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        float x = v[i];
        if (p.bias) x += __ldg(p.bias + co0 + c + i);
        if (p.relu) x = fmaxf(x, 0.f);
        if (p.accumulate) x += __bfloat162float(ob[i]);
        o[i] = __float2bfloat16(x);
      }
      *reinterpret_cast<uint4*>(dst + co0 + c) = out[0];
      *reinterpret_cast<uint4*>(dst + co0 + c + 8) = out[1];
      continue;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int co = co0 + c + i;
      if (co >= p.Cout) break;
      float x = v[i];
      if (p.bias) x += p.bias[co];
      if (p.relu) x = fmaxf(x, 0.f);
      if (p.accumulate) x += __bfloat162float(dst[co]);
      dst[co] = __float2bfloat16(x);
    }
  }
  }
  fence_before();
  __syncthreads();
  if (warp == 2) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)p.tmem_cols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// conv3x3 weight gradient on tcgen05:
//   dW[co][tap][ci] = sum over pixels p of dY[p][co] X[p + s(tap)][ci]
// One CTA per (split, tap, M tile, N tile); the K dimension is pixels, one
// 8 x 16 pixel tile (128 K rows) per stage, eight UMMA K-steps of 16.  Both
// operands are MN-major: a TMA box of 64 channels x 16 x 8 pixels of the NHWC
// tensor is 128 rows (pixels, the K index) of 128 bytes (64 channels of the
// M or N index) in the 128-byte swizzle, the canonical MN-major SWIZZLE_128B
// layout (8-row atoms 1024 bytes apart along K: the stride byte offset; the
// next 64 channels in the next box, 16 KB on: the leading byte offset).
// The larger of (Cout, Cin) is the M side (128, padded by TMA zero fill),
// the smaller the N side (a multiple of 16 up to 256): with 24 channels an
// N of 32 wastes far less than an M of 128.  X is read at the tap-shifted
// coordinates (zeros outside the image), dY unshifted.  Each split writes
// its own FP32 partial [split][co][tap][ci]; the splits are summed later in
// a fixed order, so the result is deterministic.
// ---------------------------------------------------------------------------
constexpr int WG_BOX = 64;                       // channels per TMA box (128 bytes)
constexpr uint32_t WG_BOX_BYTES = 128 * 128;     // 128 pixels x 128 bytes

struct WgParams {
  int H, W, Cin, Cout;
  int tiles_x, tiles_y, ntiles, nsplit;
  int m_is_ci;            // 0: M = output channels (A = dY); 1: M = input channels (A = X)
  int mtiles, ntile, nboxes_n, ntiles_n;
  int tmem_cols, stages;
  float* partial;
};

__device__ __forceinline__ uint64_t sdesc_mn_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(WG_BOX_BYTES >> 4) << 16) |
         ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both MN-major
__host__ __device__ constexpr uint32_t idesc_bf16_mn(int ntile) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(ntile >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__global__ void __launch_bounds__(128) conv3x3_wgrad_tc_kernel(const __grid_constant__ CUtensorMap tmdy,
                                                               const __grid_constant__ CUtensorMap tmx,
                                                               WgParams p) {
  extern __shared__ unsigned char dyn_raw[];
  __shared__ __align__(8) uint64_t full_bar[4], empty_bar[4], done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int consumed;
  unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(dyn_raw) + 1023) & ~uintptr_t(1023));
  const int S = p.stages;
  const uint32_t stage_bytes = (uint32_t)(2 + p.nboxes_n) * WG_BOX_BYTES;  // A: 2 boxes (M = 128)

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int split = blockIdx.x;
  int rest = blockIdx.y;
  const int tap = rest % 9;
  rest /= 9;
  const int mt = rest % p.mtiles;
  const int nt = rest / p.mtiles;
  const int ky = tap / 3, kx = tap - ky * 3;
  const int m0 = mt * 128, n0 = nt * p.ntile;
  int nk = 0;  // pixel tiles of this split
  if (split < p.ntiles) nk = (p.ntiles - 1 - split) / p.nsplit + 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"((uint32_t)p.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = tmem_slot;

  int issued = 0;
  if (warp == 0 && lane == 0) {
    for (int k = 0; k < nk; ++k) {
      const int s = k % S;
      if (k >= S && !mbar_wait(&empty_bar[s], ((k / S) - 1) & 1)) {
        set_err(5);
        break;
      }
      const int t = split + k * p.nsplit;
      const int tx = t % p.tiles_x, ty = (t / p.tiles_x) % p.tiles_y, n = t / (p.tiles_x * p.tiles_y);
      const int x0 = tx * TILE_W, y0 = ty * TILE_H;
      unsigned char* st = base + (size_t)s * stage_bytes;
      mbar_expect_tx(&full_bar[s], stage_bytes);
      // A (M side, 2 boxes of 64 channels) then B (N side)
      for (int b = 0; b < 2 + p.nboxes_n; ++b) {
        const bool is_a = b < 2;
        const int c0 = is_a ? m0 + b * WG_BOX : n0 + (b - 2) * WG_BOX;
        const bool use_x = is_a == (p.m_is_ci != 0);  // which tensor this box comes from
        if (use_x)
          tma_load_4d(st + b * WG_BOX_BYTES, &tmx, &full_bar[s], c0, x0 + kx - 1, y0 + ky - 1, n);
        else
          tma_load_4d(st + b * WG_BOX_BYTES, &tmdy, &full_bar[s], c0, x0, y0, n);
      }
      issued = k + 1;
    }
  } else if (warp == 1 && lane == 0) {
    const uint32_t idesc = idesc_bf16_mn(p.ntile);
    int k = 0;
    for (; k < nk; ++k) {
      const int s = k % S;
      if (!mbar_wait(&full_bar[s], (k / S) & 1)) {
        set_err(6);
        break;
      }
      fence_after();
      const uint32_t a = smem_u32(base + (size_t)s * stage_bytes);
      const uint32_t b = a + 2 * WG_BOX_BYTES;
#pragma unroll
      for (int ks = 0; ks < 8; ++ks)  // 16 pixels (K rows) of 128 bytes per step
        umma_bf16(tmem, sdesc_mn_sw128(a + ks * 2048), sdesc_mn_sw128(b + ks * 2048), idesc,
                  (k > 0 || ks > 0) ? 1u : 0u);
      umma_commit(&empty_bar[s]);
    }
    consumed = k;
    umma_commit(&done_bar);
  }
  __syncwarp();
  if (!mbar_wait(&done_bar, 0)) set_err(7);
  fence_after();
  __syncthreads();
  if (warp == 0 && lane == 0) {
    for (int k = consumed; k < issued; ++k)
      if (!mbar_wait(&full_bar[k % S], (k / S) & 1)) set_err(8);
  }

  // epilogue: accumulator row (M index) 32w + lane, columns the N index
  const int mrow = m0 + warp * 32 + lane;
  const int mlim = p.m_is_ci ? p.Cin : p.Cout, nlim = p.m_is_ci ? p.Cout : p.Cin;
  float* part = p.partial + (size_t)split * p.Cout * 9 * p.Cin;
  for (int c = 0; c < p.ntile; c += 16) {
    float v[16];
    tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
    if (mrow >= mlim || nk == 0) {
      if (nk == 0 && mrow < mlim) {  // a split without pixels still writes its (zero) partial
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = 0.f;
      } else {
        continue;
      }
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int ncol = n0 + c + i;
      if (ncol >= nlim) break;
      const int co = p.m_is_ci ? ncol : mrow, ci = p.m_is_ci ? mrow : ncol;
      part[((size_t)co * 9 + tap) * p.Cin + ci] = v[i];
    }
  }
  fence_before();
  __syncthreads();
  if (warp == 2) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)p.tmem_cols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  });
  return fn;
}

// Whether the tensor-core path takes this convolution: TMA needs 16-byte
// aligned bases and row strides (Cin, ldx multiples of 8 bf16).
inline bool eligible(const void* x, int Cin, int ldx, const void* w, int Cout) {
  return Cin % 8 == 0 && ldx % 8 == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
         (reinterpret_cast<uintptr_t>(w) & 15) == 0 && Cout >= 1 && encode_fn() != nullptr;
}

inline size_t dyn_bytes(int ntile, int msub) {
  return 1024 + (size_t)STAGES * ((size_t)A_BYTES * msub + (size_t)ntile * KCH * 2);
}

inline std::string& last_error() {
  static thread_local std::string e;
  return e;
}

inline int fail(const std::string& msg) {
  last_error() = msg;
  return -3;
}

// returns 0 or a negative code (the reason in last_error())
// msub_max 2 lets a CTA own two 128-pixel sub-tiles (16 x 16 pixels) that
// share every weight stage, halving the weight traffic per flop, when the
// image has at least 16 rows.
inline int launch(const __nv_bfloat16* x, int N, int H, int W, int Cin, int ldx, const __nv_bfloat16* w,
                  const float* bias, __nv_bfloat16* y, int ldy, int Cout, int relu, int accumulate,
                  cudaStream_t stream, int msub_max = 2) {
  last_error().clear();
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail("cuTensorMapEncodeTiled is not available from the driver");
  const int ntile = std::min(256, (Cout + 15) / 16 * 16);
  const int msub = (msub_max >= 2 && H >= 2 * TILE_H) ? 2 : 1;
  int cols = 32;
  while (cols < msub * ntile) cols *= 2;
  CUtensorMap mx, mw;
  {
    const cuuint64_t dims[4] = {(cuuint64_t)Cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)ldx * 2, (cuuint64_t)W * ldx * 2, (cuuint64_t)H * W * ldx * 2};
    const cuuint32_t box[4] = {KCH, TILE_W, (cuuint32_t)(TILE_H * msub), 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    const CUresult r = enc(&mx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(x), dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail("tensor map of the input: CUresult " + std::to_string((int)r));
  }
  {
    const cuuint64_t dims[3] = {(cuuint64_t)Cin, 9, (cuuint64_t)Cout};
    const cuuint64_t strides[2] = {(cuuint64_t)Cin * 2, (cuuint64_t)9 * Cin * 2};
    const cuuint32_t box[3] = {KCH, 1, (cuuint32_t)ntile};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = enc(&mw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(w), dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail("tensor map of the weights: CUresult " + std::to_string((int)r));
  }
  Params p;
  p.H = H;
  p.W = W;
  p.Cin = Cin;
  p.Cout = Cout;
  p.ldy = ldy;
  p.relu = relu;
  p.accumulate = accumulate;
  p.tiles_x = (W + TILE_W - 1) / TILE_W;
  p.tiles_y = (H + TILE_H * msub - 1) / (TILE_H * msub);
  p.msub = msub;
  p.ntile = ntile;
  p.tmem_cols = cols;
  p.kiters = 9 * ((Cin + KCH - 1) / KCH);
  p.bias = bias;
  p.y = y;
  const long long tiles = (long long)p.tiles_x * p.tiles_y * N;
  if (tiles > 0x7fffffffLL) {
    last_error() = "too many pixel tiles";
    return -1;
  }
  // shared memory sized so that the CTAs one SM can hold never ask for more
  // than the SM's 512 tensor-memory columns (an allocation beyond them would
  // wait for another CTA to free its columns)
  size_t smem = dyn_bytes(ntile, msub);
  const size_t sm_total = 228 * 1024;                               // shared memory of one SM
  const size_t min_for_tmem = sm_total / (512 / cols + 1) + 1024;  // at most 512 / cols CTAs fit
  if (smem < min_for_tmem) smem = min_for_tmem;
  if (smem > 200 * 1024) {
    last_error() = "shared memory of the stage ring too large";
    return -1;
  }
  // the dynamic shared memory of this launch (set per launch: the attribute
  // is per device and the size depends on ntile)
  cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  conv3x3_tc_kernel<<<dim3((unsigned)tiles, (Cout + ntile - 1) / ntile), 128, smem, stream>>>(mx, mw, p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(std::string("launch: ") + cudaGetErrorString(e));
  return 0;
}

// Whether the tensor-core weight gradient applies: TMA needs 16-byte row
// strides and bases (channel strides multiples of 8).
inline bool wgrad_eligible(const void* x, int ldx, const void* dy, int lddy, int Cin, int Cout) {
  return ldx % 8 == 0 && lddy % 8 == 0 && Cin % 8 == 0 && Cout % 8 == 0 &&
         (reinterpret_cast<uintptr_t>(x) & 15) == 0 && (reinterpret_cast<uintptr_t>(dy) & 15) == 0 &&
         encode_fn() != nullptr;
}

inline int encode_act(CUtensorMap* m, const __nv_bfloat16* t, int C, int ld, int W, int H, int N) {
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
  const cuuint64_t strides[3] = {(cuuint64_t)ld * 2, (cuuint64_t)W * ld * 2, (cuuint64_t)H * W * ld * 2};
  const cuuint32_t box[4] = {WG_BOX, TILE_W, TILE_H, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult r = encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(t), dims,
                                 strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : (int)r;
}

// partial[nsplit][Cout][9][Cin] (FP32); returns 0 or a negative code
inline int launch_wgrad(const __nv_bfloat16* x, int ldx, const __nv_bfloat16* dy, int lddy, int N, int H, int W,
                        int Cin, int Cout, float* partial, int nsplit, cudaStream_t stream) {
  last_error().clear();
  if (!encode_fn()) return fail("cuTensorMapEncodeTiled is not available from the driver");
  WgParams p;
  p.H = H;
  p.W = W;
  p.Cin = Cin;
  p.Cout = Cout;
  p.tiles_x = (W + TILE_W - 1) / TILE_W;
  p.tiles_y = (H + TILE_H - 1) / TILE_H;
  const long long ntiles = (long long)p.tiles_x * p.tiles_y * N;
  if (ntiles > 0x7fffffffLL) {
    last_error() = "too many pixel tiles";
    return -1;
  }
  p.ntiles = (int)ntiles;
  p.nsplit = nsplit;
  p.m_is_ci = Cin > Cout;
  const int mdim = p.m_is_ci ? Cin : Cout, ndim = p.m_is_ci ? Cout : Cin;
  p.mtiles = (mdim + 127) / 128;
  p.ntiles_n = (ndim + 255) / 256;
  const int nper = (ndim + p.ntiles_n - 1) / p.ntiles_n;
  p.ntile = (nper + 15) / 16 * 16;
  p.nboxes_n = (p.ntile + WG_BOX - 1) / WG_BOX;
  int cols = 32;
  while (cols < p.ntile) cols *= 2;
  p.tmem_cols = cols;
  const size_t stage = (size_t)(2 + p.nboxes_n) * WG_BOX_BYTES;
  p.stages = (int)std::max<size_t>(2, std::min<size_t>(4, (200 * 1024 - 1024) / stage));
  size_t smem = 1024 + stage * p.stages;
  const size_t min_for_tmem = (size_t)228 * 1024 / (512 / cols + 1) + 1024;
  if (smem < min_for_tmem) smem = min_for_tmem;
  if (smem > 227 * 1024) {
    last_error() = "shared memory of the weight-gradient stages too large";
    return -1;
  }
  p.partial = partial;
  CUtensorMap mdy, mx;
  int r = encode_act(&mdy, dy, Cout, lddy, W, H, N);
  if (r) return fail("tensor map of the output gradient: CUresult " + std::to_string(r));
  r = encode_act(&mx, x, Cin, ldx, W, H, N);
  if (r) return fail("tensor map of the input: CUresult " + std::to_string(r));
  cudaError_t e =
      cudaFuncSetAttribute(conv3x3_wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return fail(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  const long long gy = 9LL * p.mtiles * p.ntiles_n;
  conv3x3_wgrad_tc_kernel<<<dim3((unsigned)nsplit, (unsigned)gy), 128, smem, stream>>>(mdy, mx, p);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(std::string("launch: ") + cudaGetErrorString(e));
  return 0;
}

}  // namespace tc
