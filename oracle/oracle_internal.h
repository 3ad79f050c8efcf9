// Internal helpers shared by the oracle's translation units (test
// infrastructure only): the chi-square kernels of fftlib.f90:384-655 and
// calc_cost_reg of image.f90:12-200, as restated in oracle_fortlib.cpp.
#pragma once
#include <cmath>
#include <complex>

#include "oracle.h"

typedef std::complex<double> cplx;

namespace orc {

extern const double kZeroEps;
inline double smabs(double x) { return std::sqrt(x * x + 1e-10); }
inline int isign(int v) { return v >= 0 ? 1 : -1; }

void chisq_fcv(const cplx* V, const int* uvidx, const cplx* Vd, const double* var, double fnorm, int n,
               double& chisq, double* rre, double* rim);
void chisq_amp(const cplx* V, const int* uvidx, const double* A, const double* var, double fnorm, int n,
               double& chisq, double* rre, double* rim);
void chisq_ca(const cplx* V, const int* uvidx, const double* CA, const double* var, double fnorm, int n,
              double& chisq, double* rre, double* rim);
void chisq_cp(const cplx* V, const int* uvidx, const double* CP, const double* var, double fnorm, int n,
              double& chisq, double* rre, double* rim);
// reg[9] = cost, l1, tv, tsv, kl, gs, tfd, cen, sm; grad[npix] overwritten
void calc_cost_reg(const orc_args* a, const double* I1d, double* reg, double* grad);

}  // namespace orc
