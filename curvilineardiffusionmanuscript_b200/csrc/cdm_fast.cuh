// cdm_fast.cuh — arithmetic of the reciprocal ("fast") FP64 form shared by
// the 2D and 3D marching kernels.
#pragma once
#include "cdm_device.cuh"

namespace cdm {
namespace fastmath {

// Newton–Raphson refinement of the hardware reciprocal approximation; the
// approximation's own result is kept for 0 and ±inf arguments (1/0 = inf,
// 1/inf = 0), where the refinement would produce NaN.
__device__ __forceinline__ double rcp_nr(double b) {
  double y0;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(b));
  double e = fma(-b, y0, 1.0);
  double y = fma(y0, e, y0);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  return (y0 == 0.0 || fabs(y0) == __longlong_as_double(0x7ff0000000000000ll)) ? y0 : y;
}

// the same refinement without the 0 / ±inf fix-ups, for arguments known to be
// positive, finite and normal
__device__ __forceinline__ double rcp_pos(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  return fma(y, e, y);
}

// general exponents go through pow() out of line, keeping its temporaries out
// of the sweep's register budget
static __device__ __noinline__ double pow_general(double x, double n) { return pow(x, n); }

__device__ __forceinline__ double pow_fast(double x, int mode, int m, int half, double n) {
  if (mode == 0) return 1.0;
  if (mode == 1) {
    // x^m by repeated products (predicated for the common m <= 3), times √x for half exponents
    double p = m >= 1 ? x : 1.0;
    if (m >= 2) p *= x;
    if (m >= 3) p *= x;
    for (int e = 3; e < m; ++e) p *= x;
    if (half) p = (m >= 1) ? p * sqrt(x) : sqrt(x);
    return p;
  }
  return pow_general(x, n);
}

}  // namespace fastmath
}  // namespace cdm
