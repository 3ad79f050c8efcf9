// CPU oracle, part 1: FFT, exponential-of-semicircle NUFFT and exact DFT.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; never
// linked by the product).
//
// Restates the published FINUFFT method (Barnett, Magland & af Klinteberg,
// SIAM J. Sci. Comput. 41(5) C479-C504, 2019) that the reference calls
// through src/wrapfinufft/wrapfinufft.f90:94-206:
//   type 2 (finufft2d2, iflag=0 -> "+" sign, wrapfinufft.f90:114-124):
//     V_j = sum_{k1,k2} f(k1,k2) exp(+i (k1 x_j + k2 y_j)),
//   type 1 (finufft2d1, iflag=1 -> "+" sign, wrapfinufft.f90:188-202):
//     F(k1,k2) = sum_j c_j exp(+i (k1 x_j + k2 y_j)),
// with modes k = -N/2 .. (N-1)/2 mapped to pixels 1..N (fk bounds at
// wrapfinufft.f90:20,31).  FINUFFT itself is not in the reference tree and
// its version is unpinned (docker/Dockerfile clones HEAD); the kernel-width
// and shape rules below follow the paper (w = ceil(log10(10/eps)),
// beta = 2.30 w for upsampling 2) and FINUFFT's defaults.
#include "oracle.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

// ---------------------------------------------------------------------------
// Stockham mixed-radix FFT with the "+" exponent: out_k = sum_j in_j e^{+2 pi i jk/n}
// ---------------------------------------------------------------------------
namespace {

struct FFT1 {
  int n = 0;
  std::vector<int> radix;
  explicit FFT1(int n_) : n(n_) {
    int m = n;
    for (int r : {4, 2, 3, 5}) {
      while (m % r == 0) { radix.push_back(r); m /= r; }
    }
    for (int p = 7; m > 1; p += 2) {
      while (m % p == 0) { radix.push_back(p); m /= p; }
    }
  }
  // small DFT of length R with + sign, in place
  static void dft_small(cplx* v, int R) {
    if (R == 2) {
      cplx a = v[0], b = v[1];
      v[0] = a + b; v[1] = a - b;
    } else if (R == 4) {
      cplx a = v[0], b = v[1], c = v[2], d = v[3];
      cplx s0 = a + c, s1 = a - c, s2 = b + d, s3 = b - d;
      cplx is3(-s3.imag(), s3.real());  // i * s3
      v[0] = s0 + s2; v[2] = s0 - s2; v[1] = s1 + is3; v[3] = s1 - is3;
    } else {
      cplx tmp[64];
      for (int k = 0; k < R; ++k) {
        cplx acc = 0;
        for (int j = 0; j < R; ++j) {
          double ang = 2.0 * M_PI * double((long)j * k % R) / R;
          acc += v[j] * cplx(std::cos(ang), std::sin(ang));
        }
        tmp[k] = acc;
      }
      for (int k = 0; k < R; ++k) v[k] = tmp[k];
    }
  }
  // transform `data` (length n, unit stride); `work` is scratch of length n
  void run(cplx* data, cplx* work) const {
    cplx* src = data;
    cplx* dst = work;
    int Ns = 1;
    for (int R : radix) {
      const int nr = n / R;
      for (int j = 0; j < nr; ++j) {
        cplx v[64];
        const int k = j % Ns;
        const double ang = 2.0 * M_PI * double(k) / double(Ns * R);
        for (int r = 0; r < R; ++r) {
          v[r] = src[j + r * nr];
          if (r) v[r] *= cplx(std::cos(ang * r), std::sin(ang * r));
        }
        dft_small(v, R);
        const int base = (j / Ns) * Ns * R + k;
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
      }
      std::swap(src, dst);
      Ns *= R;
    }
    if (src != data) std::memcpy(data, src, sizeof(cplx) * n);
  }
};

// 2-D transform of a grid stored [row = index 2][col = index 1], n1 x n2
void fft2d(cplx* grid, int n1, int n2) {
  FFT1 f1(n1), f2(n2);
#pragma omp parallel
  {
    std::vector<cplx> w(std::max(n1, n2)), col(n2);
#pragma omp for schedule(static)
    for (int r = 0; r < n2; ++r) f1.run(grid + (size_t)r * n1, w.data());
#pragma omp for schedule(static)
    for (int c = 0; c < n1; ++c) {
      for (int r = 0; r < n2; ++r) col[r] = grid[(size_t)r * n1 + c];
      f2.run(col.data(), w.data());
      for (int r = 0; r < n2; ++r) grid[(size_t)r * n1 + c] = col[r];
    }
  }
}

// ---------------------------------------------------------------------------
// kernel parameters and Fourier series of the kernel
// ---------------------------------------------------------------------------
struct EsParams {
  int w;
  double beta;
};

EsParams es_params(double eps) {
  int w = (int)std::ceil(std::log10(10.0 / eps));
  if (w < 2) w = 2;
  if (w > 16) w = 16;
  double c = 2.30;
  if (w == 2) c = 2.20;
  else if (w == 3) c = 2.26;
  else if (w == 4) c = 2.38;
  return {w, c * w};
}

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

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_q.
void gauss_legendre(int q, std::vector<double>& x, std::vector<double>& wts) {
  x.resize(q);
  wts.resize(q);
  for (int i = 0; i < q; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (q + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= q; ++k) {
        double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      double dp = q * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= q; ++k) {
      double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    double dp = q * (z * p1 - p0) / (z * z - 1.0);
    x[i] = z;
    wts[i] = 2.0 / ((1 - z * z) * dp * dp);
  }
}

inline double es_kernel(double z, double beta) {
  double s = 1.0 - z * z;
  return s > 0 ? std::exp(beta * (std::sqrt(s) - 1.0)) : 0.0;
}

// psi_hat(k) = int psi(s) e^{2 pi i k s / n} ds with psi(s) = phi(2s/w)
std::vector<double> kernel_fseries(int N, int nf, const EsParams& p) {
  std::vector<double> gx, gw;
  gauss_legendre(64, gx, gw);
  std::vector<double> out(N);
  for (int i = 0; i < N; ++i) {
    int k = i - N / 2;
    double acc = 0;
    for (int q = 0; q < 64; ++q) {
      if (gx[q] <= 0) continue;  // symmetric: integrate over (0, 1] and double
      acc += gw[q] * es_kernel(gx[q], p.beta) * std::cos(M_PI * k * p.w * gx[q] / nf);
    }
    out[i] = p.w * acc;  // (w/2) * 2 * int_0^1
  }
  return out;
}

inline int wrap(long l, int n) {
  long r = l % n;
  return (int)(r < 0 ? r + n : r);
}

}  // namespace

// ---------------------------------------------------------------------------
// exact DFTs (the definitions the NUFFT approximates)
// ---------------------------------------------------------------------------
static void dft2(int nuv, const double* u, const double* v, int nx, int ny, const double* img,
                 double* vre, double* vim) {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nuv; ++j) {
    cplx acc = 0;
    for (int iy = 0; iy < ny; ++iy) {
      const int k2 = iy - ny / 2;
      cplx row = 0;
      for (int ix = 0; ix < nx; ++ix) {
        const int k1 = ix - nx / 2;
        const double ph = u[j] * k1;
        row += img[(size_t)iy * nx + ix] * cplx(std::cos(ph), std::sin(ph));
      }
      const double ph2 = v[j] * k2;
      acc += row * cplx(std::cos(ph2), std::sin(ph2));
    }
    vre[j] = acc.real();
    vim[j] = acc.imag();
  }
}

static void dft1(int nuv, const double* u, const double* v, const double* cre, const double* cim,
                 int nx, int ny, double* ore, double* oim) {
#pragma omp parallel for schedule(static)
  for (int p = 0; p < nx * ny; ++p) {
    const int k1 = p % nx - nx / 2, k2 = p / nx - ny / 2;
    cplx acc = 0;
    for (int j = 0; j < nuv; ++j) {
      const double ph = u[j] * k1 + v[j] * k2;
      acc += cplx(cre[j], cim[j]) * cplx(std::cos(ph), std::sin(ph));
    }
    ore[p] = acc.real();
    oim[p] = acc.imag();
  }
}

// ---------------------------------------------------------------------------
// NUFFT type 2: deconvolve + pad, FFT, interpolate
// ---------------------------------------------------------------------------
extern "C" int orc_nufft2d2(int nuv, const double* u, const double* v, int nx, int ny,
                            const double* img, double eps, double* vre, double* vim) {
  if (eps <= 0) {
    dft2(nuv, u, v, nx, ny, img, vre, vim);
    return 0;
  }
  const EsParams p = es_params(eps);
  const int n1 = next235even(std::max(2 * nx, 2 * p.w));
  const int n2 = next235even(std::max(2 * ny, 2 * p.w));
  const std::vector<double> ph1 = kernel_fseries(nx, n1, p), ph2 = kernel_fseries(ny, n2, p);
  std::vector<cplx> grid((size_t)n1 * n2, 0.0);
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix)
      grid[(size_t)wrap(iy - ny / 2, n2) * n1 + wrap(ix - nx / 2, n1)] =
          img[(size_t)iy * nx + ix] / (ph1[ix] * ph2[iy]);
  fft2d(grid.data(), n1, n2);
  const double half = p.w / 2.0;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < nuv; ++j) {
    const double xi1 = u[j] * n1 / (2 * M_PI), xi2 = v[j] * n2 / (2 * M_PI);
    const long l1 = (long)std::ceil(xi1 - half), l2 = (long)std::ceil(xi2 - half);
    double k1[16], k2[16];
    for (int a = 0; a < p.w; ++a) {
      k1[a] = es_kernel((l1 + a - xi1) / half, p.beta);
      k2[a] = es_kernel((l2 + a - xi2) / half, p.beta);
    }
    cplx acc = 0;
    for (int b = 0; b < p.w; ++b) {
      const cplx* row = grid.data() + (size_t)wrap(l2 + b, n2) * n1;
      cplx racc = 0;
      for (int a = 0; a < p.w; ++a) racc += k1[a] * row[wrap(l1 + a, n1)];
      acc += k2[b] * racc;
    }
    vre[j] = acc.real();
    vim[j] = acc.imag();
  }
  return 0;
}

// ---------------------------------------------------------------------------
// NUFFT type 1: spread, FFT, deconvolve + crop
// ---------------------------------------------------------------------------
extern "C" int orc_nufft2d1(int nuv, const double* u, const double* v, const double* cre,
                            const double* cim, int nx, int ny, double eps, double* ore,
                            double* oim) {
  if (eps <= 0) {
    dft1(nuv, u, v, cre, cim, nx, ny, ore, oim);
    return 0;
  }
  const EsParams p = es_params(eps);
  const int n1 = next235even(std::max(2 * nx, 2 * p.w));
  const int n2 = next235even(std::max(2 * ny, 2 * p.w));
  const std::vector<double> ph1 = kernel_fseries(nx, n1, p), ph2 = kernel_fseries(ny, n2, p);
  const size_t ng = (size_t)n1 * n2;
  std::vector<cplx> grid(ng, 0.0);
  const double half = p.w / 2.0;
  int nth = 1;
#ifdef _OPENMP
  nth = omp_get_max_threads();
#endif
  std::vector<std::vector<cplx>> priv(nth);
#pragma omp parallel
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    std::vector<cplx>& gl = priv[tid];
    gl.assign(ng, 0.0);
#pragma omp for schedule(static)
    for (int j = 0; j < nuv; ++j) {
      const double xi1 = u[j] * n1 / (2 * M_PI), xi2 = v[j] * n2 / (2 * M_PI);
      const long l1 = (long)std::ceil(xi1 - half), l2 = (long)std::ceil(xi2 - half);
      double k1[16], k2[16];
      for (int a = 0; a < p.w; ++a) {
        k1[a] = es_kernel((l1 + a - xi1) / half, p.beta);
        k2[a] = es_kernel((l2 + a - xi2) / half, p.beta);
      }
      const cplx c(cre[j], cim[j]);
      for (int b = 0; b < p.w; ++b) {
        cplx* row = gl.data() + (size_t)wrap(l2 + b, n2) * n1;
        const cplx cb = c * k2[b];
        for (int a = 0; a < p.w; ++a) row[wrap(l1 + a, n1)] += cb * k1[a];
      }
    }
  }
  // deterministic reduction of the per-thread grids (thread order)
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)ng; ++i) {
    cplx s = 0;
    for (int t = 0; t < nth; ++t) s += priv[t][i];
    grid[i] = s;
  }
  fft2d(grid.data(), n1, n2);
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      const cplx g = grid[(size_t)wrap(iy - ny / 2, n2) * n1 + wrap(ix - nx / 2, n1)] /
                     (ph1[ix] * ph2[iy]);
      ore[(size_t)iy * nx + ix] = g.real();
      oim[(size_t)iy * nx + ix] = g.imag();
    }
  return 0;
}

extern "C" int orc_nthreads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
