// Common device helpers: complex arithmetic, block reductions and the
// intra-group barrier of the persistent solver.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

#include "layout.h"

// CTA shape of the solver kernel per precision.  FP32 runs 512 threads
// (two CTAs per SM at 64 registers: 32 resident warps to hide the latency of
// the gather-heavy stages), FP64 256 threads (two CTAs per SM at 128
// registers; its shared-memory staging is twice as large).  Device code
// strides by blockDim.x; buffers shared by both shapes are sized for the
// larger one.
template <typename R>
struct Shape {
  static constexpr int threads = sizeof(R) == 4 ? 512 : 256;
  static constexpr int warps = threads / 32;
  static constexpr int min_blocks = 2;
};
#define SMILI_MAX_THREADS 512
#define SMILI_MAX_WARPS (SMILI_MAX_THREADS / 32)

template <typename R>
struct cpx {
  R x, y;
};
template <typename R>
__device__ __forceinline__ cpx<R> cmk(R a, R b) {
  cpx<R> c;
  c.x = a;
  c.y = b;
  return c;
}
template <typename R>
__device__ __forceinline__ cpx<R> cadd(cpx<R> a, cpx<R> b) {
  return cmk(a.x + b.x, a.y + b.y);
}
template <typename R>
__device__ __forceinline__ cpx<R> csub(cpx<R> a, cpx<R> b) {
  return cmk(a.x - b.x, a.y - b.y);
}
template <typename R>
__device__ __forceinline__ cpx<R> cmul(cpx<R> a, cpx<R> b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R>
__device__ __forceinline__ cpx<R> cscale(cpx<R> a, R s) {
  return cmk(a.x * s, a.y * s);
}
// multiply by +i
template <typename R>
__device__ __forceinline__ cpx<R> cmul_i(cpx<R> a) {
  return cmk(-a.y, a.x);
}

template <typename T>
__device__ __forceinline__ T* at(char* base, int64_t off) {
  return reinterpret_cast<T*>(base + off);
}

// ---------------------------------------------------------------------------
// block reductions of K values per thread (deterministic order)
// ---------------------------------------------------------------------------
enum { RED_SUM = 0, RED_MAX = 1, RED_MIN = 2 };

__device__ __forceinline__ double red_op(double a, double b, int op) {
  return op == RED_SUM ? a + b : (op == RED_MAX ? fmax(a, b) : fmin(a, b));
}

// Reduce v[0..K) over the block; result valid in every thread's out[].
// scratch: (blockDim.x / 32) * K doubles of shared memory.
template <int K>
__device__ __forceinline__ void block_reduce(const double (&v)[K], const int (&op)[K],
                                             double (&out)[K], double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double a = v[k];
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) a = red_op(a, __shfl_xor_sync(0xffffffffu, a, s), op[k]);
    if (lane == 0) scratch[wid * K + k] = a;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double a = scratch[k];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) a = red_op(a, scratch[w * K + k], op[k]);
    out[k] = a;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Group context: the CTAs that cooperate on one problem.
// ---------------------------------------------------------------------------
struct GroupCtx {
  int rank, G;
  unsigned* bar;       // [0] arrival counter, [1] generation
  double* red_part;    // [G][SMILI_REDK] partials
  double* red_out;     // [SMILI_REDK] reduced values
  int* abort_flag;     // global abort (set on a barrier timeout)
  long long spin_limit;
};

// Spin budget of one barrier wait.  A healthy barrier completes in
// microseconds; the limit only ends a wait that can never complete.
#define SMILI_SPIN_LIMIT (1LL << 24)

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned atom_acqrel_add(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

// Wait until the generation counter moves past gen.  Polls without sleeping
// for a short while (barriers normally complete within microseconds), then
// backs off; gives up after spin_limit polls or when another CTA aborted.
__device__ __forceinline__ bool wait_generation(GroupCtx& g, unsigned gen) {
  long long spins = 0;
  while (ld_acquire(&g.bar[1]) == gen) {
    if (++spins > g.spin_limit || *((volatile int*)g.abort_flag)) {
      atomicExch(g.abort_flag, 1);
      return false;
    }
    if (spins > 4096) __nanosleep(64);
  }
  return true;
}

// Returns false when the wait timed out (abort flag set): callers stop work.
// Arrival is an acquire-release atomic on the group's counter (it orders this
// CTA's earlier writes before the arrival and the last arriver's reads after
// it); the last arriver resets the counter and releases the generation.
__device__ bool group_sync(GroupCtx& g) {
  __syncthreads();
  if (g.G == 1) return true;
  __shared__ int ok_s;
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();  // writes of the whole block (ordered by bar.sync) before the arrival
    const unsigned gen = ld_acquire(&g.bar[1]);
    const unsigned arrived = atom_acqrel_add(&g.bar[0], 1u);
    if (arrived == (unsigned)(g.G - 1)) {
      g.bar[0] = 0;
      red_release_add(&g.bar[1], 1u);
    } else {
      ok = wait_generation(g, gen) ? 1 : 0;
    }
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// Group-wide reduction of K values held in shared memory (vals[0..K),
// already reduced over the block).  Every CTA passes its partials; the last
// CTA to arrive combines them in rank order and publishes the result, so the
// value is identical in every CTA and independent of arrival order.  On
// return vals[] holds the group result in every CTA.  K <= SMILI_REDK.
#define SMILI_REDK 128
__device__ bool group_reduce(GroupCtx& g, double* vals, const unsigned char* ops, int K) {
  if (g.G == 1) {
    __syncthreads();
    return true;
  }
  __shared__ int last_s, ok_s;
  for (int k = threadIdx.x; k < K; k += blockDim.x) g.red_part[(size_t)g.rank * SMILI_REDK + k] = vals[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    ok_s = 1;
    last_s = 0;
    __threadfence();  // the block's partials (written by other threads) before the arrival
    const unsigned gen = ld_acquire(&g.bar[1]);
    const unsigned arrived = atom_acqrel_add(&g.bar[0], 1u);
    if (arrived == (unsigned)(g.G - 1)) {
      last_s = 1;
    } else {
      ok_s = wait_generation(g, gen) ? 1 : 0;
    }
  }
  __syncthreads();
  if (last_s) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      const volatile double* rp = g.red_part;
      double a = rp[k];
      for (int r = 1; r < g.G; ++r) a = red_op(a, rp[(size_t)r * SMILI_REDK + k], ops[k]);
      g.red_out[k] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();  // the reduced values before the release
      g.bar[0] = 0;
      red_release_add(&g.bar[1], 1u);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) vals[k] = ((const volatile double*)g.red_out)[k];
  __syncthreads();
  return ok_s != 0;
}

// Block reduction of K per-thread values (v[k] in each thread, op per entry)
// into shared out[0..K).  scratch: (blockDim.x / 32) * K doubles.
__device__ void block_reduce_arr(const double* v, const unsigned char* ops, int K, double* out,
                                 double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int k = 0; k < K; ++k) {
    double a = v[k];
    const int op = ops[k];
    for (int s = 16; s > 0; s >>= 1) a = red_op(a, __shfl_xor_sync(0xffffffffu, a, s), op);
    if (lane == 0) scratch[wid * K + k] = a;
  }
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double a = scratch[k];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) a = red_op(a, scratch[w * K + k], ops[k]);
    out[k] = a;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Stage profiler: CTA 0 (thread 0) accumulates the time between consecutive
// marks into acc[stage] (nanoseconds, from %globaltimer).  Off when acc is 0.
// ---------------------------------------------------------------------------
enum {
  PR_F1 = 0, PR_F2, PR_F3, PR_F4, PR_F5, PR_F6, PR_F7, PR_F8, PR_LB_POST, PR_CAUCHY, PR_FORMK,
  PR_SUBSM, PR_LNSRCH, PR_INIT, PR_OTHER, PR_COUNT, PR_C_SEL, PR_C_GATHER, PR_C_SORT, PR_C_SCAN,
  PR_C_ROUNDS, PR_NSTAGE
};

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

struct Prof {
  unsigned long long* acc;
  unsigned long long t;
  __device__ void start() {
    if (acc) t = gtimer();
  }
  __device__ void mark(int st) {
    if (acc) {
      const unsigned long long now = gtimer();
      acc[st] += now - t;
      t = now;
    }
  }
  __device__ void count(int st) {
    if (acc) acc[st] += 1;
  }
};
