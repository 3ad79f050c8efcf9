// Non-redundant uv list on the device: the compute core of get_uvlist
// (smili/uvdata/uvtable/tools.py:12-132).
//
// Input: the uv points of all data terms stacked in the reference's order
// (fcv, amp, cp uv12/uv23/uv31, ca uv1..uv4).  Each point with v < 0 becomes
// (-u, -v) with sign -1 (tools.py:47-95); the distinct folded points are
// listed in the order np.unique gives complex values (u, then v; -0 and +0
// are one value), each represented by its first occurrence in the stack; each
// input point gets sign * (1 + its point's position in that list).
//
// Device work: fold and key every point (order-preserving 64-bit keys of u
// and v, ties broken by stack position), a bitonic sort of the keys (blocks
// of UV_BLK in shared memory, longer merges in global memory), head flags
// where the key changes, a three-kernel scan of the flags into list
// positions, and two scatters.  Included by solver.cu (error reporting).
#pragma once
#include <mutex>

struct UvKey {
  unsigned long long ku, kv;
  unsigned idx, pad;
};

constexpr int UV_BLK = 2048;  // keys sorted per CTA in shared memory (48 KB)
constexpr int UV_SCAN = 1024; // flags per CTA in the scan

// IEEE bits of a finite double -> unsigned key with the same order; -0 -> +0
__device__ __forceinline__ unsigned long long uv_order_key(double x) {
  unsigned long long b = (unsigned long long)__double_as_longlong(x);
  if ((b << 1) == 0) b = 0;
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

__device__ __forceinline__ bool uv_less(const UvKey& a, const UvKey& b) {
  if (a.ku != b.ku) return a.ku < b.ku;
  if (a.kv != b.kv) return a.kv < b.kv;
  return a.idx < b.idx;
}

__global__ void uv_fold_kernel(int n, long npad, const double* __restrict__ u, const double* __restrict__ v,
                               double* fu, double* fv, signed char* sg, UvKey* keys) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < npad; i += (long)gridDim.x * blockDim.x) {
    UvKey k;
    k.pad = 0;
    if (i < n) {
      double a = u[i], b = v[i];
      signed char s = 1;
      if (b < 0.0) {
        a = -a;
        b = -b;
        s = -1;
      }
      fu[i] = a;
      fv[i] = b;
      sg[i] = s;
      k.ku = uv_order_key(a);
      k.kv = uv_order_key(b);
      k.idx = (unsigned)i;
    } else {  // padding sorts after every finite point
      k.ku = k.kv = ~0ULL;
      k.idx = 0xffffffffu;
    }
    keys[i] = k;
  }
}

// compare-exchange of the pair (i, i + j) in the bitonic stage k; ascending
// where the global index has bit k clear
__device__ __forceinline__ void uv_cmpx(UvKey* s, int i, int j, long gi, long k) {
  const UvKey a = s[i], b = s[i + j];
  const bool up = (gi & k) == 0;
  if (uv_less(b, a) == up) {
    s[i] = b;
    s[i + j] = a;
  }
}

// stages k = 2 .. UV_BLK of every UV_BLK-key block, in shared memory
__global__ void __launch_bounds__(1024) uv_sort_local(UvKey* keys) {
  __shared__ UvKey s[UV_BLK];
  const long base = (long)blockIdx.x * UV_BLK;
  for (int i = threadIdx.x; i < UV_BLK; i += blockDim.x) s[i] = keys[base + i];
  __syncthreads();
  for (int k = 2; k <= UV_BLK; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < UV_BLK / 2; t += blockDim.x) {
        const int i = 2 * t - (t & (j - 1));
        uv_cmpx(s, i, j, base + i, k);
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < UV_BLK; i += blockDim.x) keys[base + i] = s[i];
}

// one step j >= UV_BLK of stage k, in global memory
__global__ void uv_sort_global(UvKey* keys, long npad, long k, long j) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < npad / 2; t += (long)gridDim.x * blockDim.x) {
    const long i = 2 * t - (t & (j - 1));
    const UvKey a = keys[i], b = keys[i + j];
    const bool up = (i & k) == 0;
    if (uv_less(b, a) == up) {
      keys[i] = b;
      keys[i + j] = a;
    }
  }
}

// steps j = UV_BLK/2 .. 1 of stage k, in shared memory
__global__ void __launch_bounds__(1024) uv_sort_merge_local(UvKey* keys, long k) {
  __shared__ UvKey s[UV_BLK];
  const long base = (long)blockIdx.x * UV_BLK;
  for (int i = threadIdx.x; i < UV_BLK; i += blockDim.x) s[i] = keys[base + i];
  __syncthreads();
  for (int j = UV_BLK / 2; j > 0; j >>= 1) {
    for (int t = threadIdx.x; t < UV_BLK / 2; t += blockDim.x) {
      const int i = 2 * t - (t & (j - 1));
      uv_cmpx(s, i, j, base + i, k);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < UV_BLK; i += blockDim.x) keys[base + i] = s[i];
}

// head flags of the sorted keys, scanned per CTA (inclusive); bsum[block] =
// the CTA's total
__global__ void __launch_bounds__(UV_SCAN) uv_scan_local(const UvKey* keys, int n, int* head, int* rank, int* bsum) {
  __shared__ int wsum[UV_SCAN / 32];
  const int i = blockIdx.x * UV_SCAN + threadIdx.x;
  int h = 0;
  if (i < n) {
    h = (i == 0) || keys[i].ku != keys[i - 1].ku || keys[i].kv != keys[i - 1].kv;
    head[i] = h;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = h;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  if (wid > 0) x += wsum[wid - 1];
  if (i < n) rank[i] = x;
  if (threadIdx.x == UV_SCAN - 1) bsum[blockIdx.x] = x;
}

// exclusive scan of the nb CTA totals, in place (one CTA)
__global__ void __launch_bounds__(1024) uv_scan_sums(int* bsum, int nb) {
  __shared__ int part[1024];
  const int per = (nb + blockDim.x - 1) / blockDim.x, b0 = threadIdx.x * per;
  int s = 0;
  for (int q = 0; q < per && b0 + q < nb; ++q) s += bsum[b0 + q];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const int v = part[t];
      part[t] = run;
      run += v;
    }
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int q = 0; q < per && b0 + q < nb; ++q) {
    const int v = bsum[b0 + q];
    bsum[b0 + q] = run;
    run += v;
  }
}

// list position of every sorted key; the first key of each run writes its
// point into the list; every stack position learns its point's position
__global__ void uv_scatter(const UvKey* keys, int n, const int* head, const int* rank, const int* bsum,
                           const double* fu, const double* fv, int* inv, double* uo, double* vo) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int pos = rank[i] + bsum[i / UV_SCAN] - 1;
    const unsigned orig = keys[i].idx;
    inv[orig] = pos;
    if (head[i]) {
      uo[pos] = fu[orig];
      vo[pos] = fv[orig];
    }
  }
}

__global__ void uv_sign(int n, const int* inv, const signed char* sg, int* uvidx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    uvidx[i] = (int)sg[i] * (inv[i] + 1);
}

// Device work space per device, kept between calls and grown when a larger
// list arrives (allocation and release of tens of MB cost up to tens of ms
// each, more than the listing itself).  Calls hold g_uv_mu for their whole
// duration, so the space is never shared by two calls at once.
struct UvWork {
  char* d = nullptr;
  size_t cap = 0;
};
static std::mutex g_uv_mu;
static UvWork g_uv_work[64];

// Host side: validates, runs the kernels on `st` and copies the results back.
static int uvlist_run(int n, const double* u, const double* v, int device, cudaStream_t st, int* nuv,
                      double* u_out, double* v_out, int* uvidx) {
  if (n < 1 || n > (1 << 26) || !u || !v || !nuv || !u_out || !v_out || !uvidx)
    return fail(SMILI_ERR_ARG, "get_uvlist: need 1 <= n <= 2^26 points and non-null arrays");
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(u[i]) || !std::isfinite(v[i])) return fail(SMILI_ERR_DATA, "get_uvlist: non-finite u or v");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SMILI_ERR_NODEV, "no CUDA device");
  if (device < 0 || device >= ndev || device >= 64 || cudaSetDevice(device) != cudaSuccess)
    return fail(SMILI_ERR_NODEV, "cannot select the CUDA device");
  std::lock_guard<std::mutex> lock(g_uv_mu);
  long npad = UV_BLK;
  while (npad < n) npad <<= 1;
  const int nb = (n + UV_SCAN - 1) / UV_SCAN;
  // one allocation: keys, folded u/v, signs, flags, ranks, CTA sums, inverse, outputs
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_keys = take(sizeof(UvKey) * npad), o_fu = take(8 * (size_t)n), o_fv = take(8 * (size_t)n),
               o_sg = take(n), o_head = take(4 * (size_t)n), o_rank = take(4 * (size_t)n),
               o_bsum = take(4 * (size_t)nb), o_inv = take(4 * (size_t)n), o_uo = take(8 * (size_t)n),
               o_vo = take(8 * (size_t)n), o_idx = take(4 * (size_t)n), o_u = take(8 * (size_t)n),
               o_v = take(8 * (size_t)n);
  UvWork& wk = g_uv_work[device];
  if (wk.cap < off) {
    if (wk.d) cudaFree(wk.d);
    wk.d = nullptr;
    wk.cap = 0;
    const size_t want = off + off / 4;  // headroom for slightly larger lists
    if (cudaMalloc(&wk.d, want) != cudaSuccess) {
      wk.d = nullptr;
      return fail(SMILI_ERR_CUDA, "get_uvlist: cudaMalloc of the work space failed");
    }
    wk.cap = want;
  }
  char* d = wk.d;
  auto at_ = [&](size_t o) { return d + o; };
  UvKey* keys = reinterpret_cast<UvKey*>(at_(o_keys));
  double *fu = reinterpret_cast<double*>(at_(o_fu)), *fv = reinterpret_cast<double*>(at_(o_fv));
  signed char* sg = reinterpret_cast<signed char*>(at_(o_sg));
  int *head = reinterpret_cast<int*>(at_(o_head)), *rank = reinterpret_cast<int*>(at_(o_rank));
  int *bsum = reinterpret_cast<int*>(at_(o_bsum)), *inv = reinterpret_cast<int*>(at_(o_inv));
  double *uo = reinterpret_cast<double*>(at_(o_uo)), *vo = reinterpret_cast<double*>(at_(o_vo));
  int* idx = reinterpret_cast<int*>(at_(o_idx));
  double *du = reinterpret_cast<double*>(at_(o_u)), *dv = reinterpret_cast<double*>(at_(o_v));
  cudaError_t e = cudaSuccess;
  auto chk = [&](cudaError_t r) {
    if (e == cudaSuccess && r != cudaSuccess) e = r;
  };
  chk(cudaMemcpyAsync(du, u, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
  chk(cudaMemcpyAsync(dv, v, 8 * (size_t)n, cudaMemcpyHostToDevice, st));
  const int gb = (int)std::min<long>((npad + 255) / 256, 148L * 16);
  uv_fold_kernel<<<gb, 256, 0, st>>>(n, npad, du, dv, fu, fv, sg, keys);
  chk(cudaGetLastError());
  const int nblk = (int)(npad / UV_BLK);
  uv_sort_local<<<nblk, 1024, 0, st>>>(keys);
  chk(cudaGetLastError());
  for (long k = 2L * UV_BLK; k <= npad; k <<= 1) {
    for (long j = k >> 1; j >= UV_BLK; j >>= 1) {
      uv_sort_global<<<(int)std::min<long>((npad / 2 + 255) / 256, 148L * 16), 256, 0, st>>>(keys, npad, k, j);
      chk(cudaGetLastError());
    }
    uv_sort_merge_local<<<nblk, 1024, 0, st>>>(keys, k);
    chk(cudaGetLastError());
  }
  uv_scan_local<<<nb, UV_SCAN, 0, st>>>(keys, n, head, rank, bsum);
  chk(cudaGetLastError());
  uv_scan_sums<<<1, 1024, 0, st>>>(bsum, nb);
  chk(cudaGetLastError());
  const int gn = (int)std::min<long>((n + 255) / 256, 148L * 16);
  uv_scatter<<<gn, 256, 0, st>>>(keys, n, head, rank, bsum, fu, fv, inv, uo, vo);
  chk(cudaGetLastError());
  uv_sign<<<gn, 256, 0, st>>>(n, inv, sg, idx);
  chk(cudaGetLastError());
  // the list length: position of the last sorted key + 1
  int last_rank = 0, last_sum = 0;
  chk(cudaMemcpyAsync(&last_rank, rank + (n - 1), 4, cudaMemcpyDeviceToHost, st));
  chk(cudaMemcpyAsync(&last_sum, bsum + (n - 1) / UV_SCAN, 4, cudaMemcpyDeviceToHost, st));
  chk(cudaStreamSynchronize(st));
  const int m = last_rank + last_sum;
  if (e == cudaSuccess && (m < 1 || m > n)) e = cudaErrorUnknown;
  if (e == cudaSuccess) {
    chk(cudaMemcpyAsync(u_out, uo, 8 * (size_t)m, cudaMemcpyDeviceToHost, st));
    chk(cudaMemcpyAsync(v_out, vo, 8 * (size_t)m, cudaMemcpyDeviceToHost, st));
    chk(cudaMemcpyAsync(uvidx, idx, 4 * (size_t)n, cudaMemcpyDeviceToHost, st));
    chk(cudaStreamSynchronize(st));
  }
  if (e != cudaSuccess) return fail(SMILI_ERR_CUDA, std::string("get_uvlist: ") + cudaGetErrorString(e));
  *nuv = m;
  return SMILI_OK;
}
