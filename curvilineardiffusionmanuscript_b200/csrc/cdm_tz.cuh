// cdm_tz.cuh — twilight-zone (manufactured-solution) forcing of the reference's
// wavy-mesh verification: define_forcing_wavy (twilight_zone.jl:54-195), added
// to the update by _update_kernel_tz! (update.jl:23-71) and to the residual by
// _update_resid_kernel_tz! (residuals.jl:49-99).
//
// The forcing of cell (i, j) is
//   f = ut − orth_ξ − orth_η − cross − non_orth_ξ − non_orth_η − s      (:191)
// with orth_ξ = g11·(αξ·uξ + α·uξξ), orth_η = g22·(αη·uη + α·uηη),
// cross = g12·(2α·uξη + αη·uξ + αξ·uη), non_orth_ξ = α·αᵢⱼ·uξ,
// non_orth_η = α·βᵢⱼ·uη (:182-188), where α is the diffusivity of the current
// pseudo-iteration and everything else depends only on the mesh, ρ, cₚ, the
// source term and t.  `terms` evaluates those α-independent parts once per
// time step; `combine` adds α in the kernel, in the reference's operation
// order, so that the result equals the reference expression evaluated at once.
//
// Elementary functions.  exp and sinpi are evaluated by the methods below,
// not by the platform's libraries, so that the device and a CPU restatement of
// the same methods give the same bits:
//   exp:   Cody–Waite reduction x = k·ln2 + r, |r| ≤ ln2/2, with ln2 split into
//          its nearest double and the remainder (the first product subtracted
//          by a fused multiply-add is exact), then the Taylor polynomial of e^r
//          to degree 13 by Horner's rule with fused multiply-adds, scaled by 2^k;
//   sinpi: exact reduction of x modulo 2, folding to a ∈ [0, ½], then the
//          Taylor polynomial of sin(πa) (a ≤ ¼) or of cos(π(½ − a)) in the
//          square of the reduced argument, Horner with fused multiply-adds.
// Coefficients are 1/n!, (−1)^k π^(2k+1)/(2k+1)! and (−1)^k π^(2k)/(2k)! and
// ln2, 1/ln2 rounded to the nearest double.  Both stay within 2 ulp of the
// correctly rounded results.  exy^(3/2) is evaluated as exy·√exy.
#pragma once
#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define CDM_TZ_HD __host__ __device__ __forceinline__
#else
#define CDM_TZ_HD inline
#endif

namespace cdm {
namespace tz {

CDM_TZ_HD double exp_cw(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return INFINITY;
  if (x < -745.1332191019412) return 0.0;
  const double k = nearbyint(x * 0x1.71547652b82fep+0);
  const double r = fma(-k, 0x1.abc9e3b39803fp-56, fma(-k, 0x1.62e42fefa39efp-1, x));
  double p = 0x1.6124613a86d09p-33;  // 1/13!
  p = fma(p, r, 0x1.1eed8eff8d898p-29);
  p = fma(p, r, 0x1.ae64567f544e4p-26);
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);
  p = fma(p, r, 0x1.71de3a556c734p-19);
  p = fma(p, r, 0x1.a01a01a01a01ap-16);
  p = fma(p, r, 0x1.a01a01a01a01ap-13);
  p = fma(p, r, 0x1.6c16c16c16c17p-10);
  p = fma(p, r, 0x1.1111111111111p-7);
  p = fma(p, r, 0x1.5555555555555p-5);
  p = fma(p, r, 0x1.5555555555555p-3);
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  return ldexp(p, (int)k);
}

CDM_TZ_HD double sinpi_poly(double a) {  // sin(πa), 0 <= a <= 1/4
  const double z = a * a;
  double p = 0x1.aaec32af93359p-21;
  p = fma(p, z, -0x1.6fadb9f155744p-16);
  p = fma(p, z, 0x1.e8f434d018d63p-12);
  p = fma(p, z, -0x1.e3074fde8871fp-8);
  p = fma(p, z, 0x1.50783487ee782p-4);
  p = fma(p, z, -0x1.32d2cce62bd86p-1);
  p = fma(p, z, 0x1.466bc6775aae2p+1);
  p = fma(p, z, -0x1.4abbce625be53p+2);
  p = fma(p, z, 0x1.921fb54442d18p+1);
  return a * p;
}

CDM_TZ_HD double cospi_poly(double b) {  // cos(πb), 0 <= b <= 1/4
  const double z = b * b;
  double p = 0x1.20c62c2f2d7f5p-18;
  p = fma(p, z, -0x1.b6e24f44b128fp-14);
  p = fma(p, z, 0x1.f9d38a3763cc3p-10);
  p = fma(p, z, -0x1.a6d1f2a204a8cp-6);
  p = fma(p, z, 0x1.e1f506891babbp-3);
  p = fma(p, z, -0x1.55d3c7e3cbffap+0);
  p = fma(p, z, 0x1.03c1f081b5ac4p+2);
  p = fma(p, z, -0x1.3bd3cc9be45dep+2);
  return fma(p, z, 1.0);
}

CDM_TZ_HD double sinpi(double x) {
  if (!isfinite(x)) return x - x;  // NaN
  const double y = x - 2.0 * nearbyint(0.5 * x);  // exact, y in [-1, 1]
  const double s = y < 0.0 ? -1.0 : 1.0;
  double a = fabs(y);
  if (a > 0.5) a = 1.0 - a;  // exact
  const double v = a <= 0.25 ? sinpi_poly(a) : cospi_poly(0.5 - a);
  return s * v;
}

// the α-independent parts of the forcing of one cell, in the order the
// combination reads them
struct Terms {
  double ut;   // ∂u/∂t of the exact solution (0 with no_t)
  double p1;   // αξ·uξ
  double uxx;  // uξξ
  double p2;   // αη·uη
  double uee;  // uηη
  double uxe;  // uξη
  double p3;   // αη·uξ
  double p4;   // αξ·uη
  double ux;   // uξ
  double ue;   // uη
};
constexpr int kNumTerms = 10;

// twilight_zone.jl:69-183 for the cell at 0-based full-array index (I, J):
// centroid (x, y), forward metrics xξ, xη, yξ, yη, density rho, cₚ, time t,
// no_t, and the domain node counts nnx, nny (mesh.nnodes).  Julia's integer
// literals and constants enter as the doubles its promotion rules give.
CDM_TZ_HD Terms terms(double x, double y, double xxi, double xeta, double yxi, double yeta, double rho, double cp,
                      double t, int no_t, int64_t I, int64_t J, int nnx, int nny) {
  const double Lx = 12.0, Ly = 12.0, n_xy = 6.0, n_yx = 6.0, fwhm = 1.0, damp = 4.0;
  const double pi = 3.141592653589793;
  const double dx0 = Lx / (double)(nnx - 1);
  const double dy0 = Ly / (double)(nny - 1);
  const double Ax = 0.2 / dx0;
  const double Ay = 0.4 / dy0;
  // indi = (i - 5) + 1/2 with the reference's 1-based full-array index i = I + 1
  const double indi = (double)(I + 1 - 5) + 0.5;
  const double indj = (double)(J + 1 - 5) + 0.5;
  const double xi_xi = 0.0, xi_eta = 0.0;  // xξξ, xξη
  const double Kx = ((pi * n_xy) * dy0) / Ly;
  const double xee = (((-dx0) * Ax) * (Kx * Kx)) * sinpi(((n_xy * (indj - 1.0)) * dy0) / Ly);
  const double Ky = ((pi * n_yx) * dx0) / Lx;
  const double yxx = (((-dy0) * Ay) * (Ky * Ky)) * sinpi(((n_yx * (indi - 1.0)) * dx0) / Lx);
  const double yxe = 0.0, yee = 0.0;  // yξη, yηη
  const double xm = x - 0.0, ym = y - 0.0;  // x - x0, y - y0
  double exy = exp_cw(-((xm * xm) / fwhm + (ym * ym) / fwhm));
  Terms o;
  if (no_t) {
    o.ut = 0.0;
  } else {
    exy = exy * exp_cw((-damp) * t);
    o.ut = (-damp) * exy;
  }
  const double A = ((2.0 * xm) / fwhm) * xxi + ((2.0 * ym) / fwhm) * yxi;
  const double B = ((2.0 * xm) / fwhm) * xeta + ((2.0 * ym) / fwhm) * yeta;
  const double ux = ((-2.0 / fwhm) * (xm * xxi + ym * yxi)) * exy;
  const double uxx = (A * A - (2.0 / fwhm) * (((xxi * xxi + yxi * yxi) + xm * xi_xi) + ym * yxx)) * exy;
  const double ue = ((-2.0 / fwhm) * (xm * xeta + ym * yeta)) * exy;
  const double uee = (B * B - (2.0 / fwhm) * (((xeta * xeta + yeta * yeta) + xm * xee) + ym * yee)) * exy;
  const double uxe = (A * B - (2.0 / fwhm) * (((xxi * xeta + yxi * yeta) + xm * xi_eta) + ym * yxe)) * exy;
  // nonlinear diffusivity α = u^(5/2)/(ρcₚ): its ξ and η derivatives (:182-183)
  const double e15 = exy * sqrt(exy);
  const double rc = rho * cp;
  const double ax = ((2.5 * e15) * ux) / rc;
  const double ae = ((2.5 * e15) * ue) / rc;
  o.p1 = ax * ux;
  o.uxx = uxx;
  o.p2 = ae * ue;
  o.uee = uee;
  o.uxe = uxe;
  o.p3 = ae * ux;
  o.p4 = ax * ue;
  o.ux = ux;
  o.ue = ue;
  return o;
}

// the forcing of one cell from its terms and the current diffusivity α
// (:184-191); g11 = ξx² + ξy², g22 = ηx² + ηy², g12 = ξx·ηx + ξy·ηy, aij and
// bij the metric cache (∇²ξ, ∇²η), s the source term
CDM_TZ_HD double combine(const Terms& T, double alpha, double g11, double g22, double g12, double aij, double bij,
                         double s) {
  const double orth_x = g11 * (T.p1 + alpha * T.uxx);
  const double orth_e = g22 * (T.p2 + alpha * T.uee);
  const double cross = g12 * (((2.0 * alpha) * T.uxe + T.p3) + T.p4);
  const double no_x = (alpha * aij) * T.ux;
  const double no_e = (alpha * bij) * T.ue;
  return (((((T.ut - orth_x) - orth_e) - cross) - no_x) - no_e) - s;
}

}  // namespace tz
}  // namespace cdm
