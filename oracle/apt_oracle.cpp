// apt_oracle.cpp — CPU restatement of the reference APT solver.
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle and the CPU
// baseline of the B200 APT library.  Only the tests, the smoke check and the
// CPU-baseline leg of the benchmark may load it; the product path never does.
//
// It restates, stage by stage and operation by operation, the accelerated
// pseudo-transient solver of CurvilinearDiffusion
// (smillerc/CurvilinearDiffusionManuscript, pure Julia; no Julia toolchain is
// available, so the reference itself cannot be run here).  Every function
// cites the reference file:line it follows.  Floating-point expressions keep
// the reference's evaluation order (Julia evaluates `a + b + c` left to right,
// `x^2` as x*x, `0.25(e)` as 0.25*e), and the file is compiled with
// -ffp-contract=off so that no multiply-add is fused.
//
// Parity status: the reference publishes no golden vectors for this path and
// its mesh library (CurvilinearGrids 0.6) is not vendored, so the restatement
// is pinned by known-answer tests (boundary-condition semantics of
// test/unit/test_bc.jl, uniform-mesh Laplacian, manufactured-solution order,
// backward-Euler fixed point) rather than by reference outputs.
//
// Threads: loops over the slowest axis are OpenMP-parallel; results do not
// depend on the thread count except the optional RMS norm's summation order.
//
// Twilight zone: define_forcing_wavy (twilight_zone.jl:54-195) is restated
// literally and evaluated per cell inside the update and the residual with the
// iteration's diffusivity, as _update_kernel_tz! / _update_resid_kernel_tz!
// do.  Its exp and sinpi are evaluated by a Cody–Waite/Taylor exp and an
// exactly reduced Taylor sinpi (below) rather than libm, the same published
// methods the CUDA library evaluates, so that the twilight-zone path can be
// compared bit for bit; both stay within 2 ulp of the correctly rounded
// values (checked against high-precision values by the test-suite).  Julia's
// own exp/sinpi may differ from them in the last bit, and exy^(3/2) is taken
// as exy*sqrt(exy).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.14159265358979323846;

enum { BC_NEUMANN = 0, BC_DIRICHLET = 1, BC_PERIODIC = 2, BC_NEG_SYMMETRY = 3 };
enum { ST_OK = 0, ST_MAX_ITER = 1, ST_NONFINITE = 2, ST_BAD_INPUT = 3 };

struct Mesh {
  int ndim, ni, nj, nk, nh;
  int64_t nx, ny, nz, n;  // full sizes
  // cell-centre inverse metrics [3*a + c]
  std::vector<double> inv[9];
  std::vector<double> edgeJ[3];
  std::vector<double> edgehat[3][9];
  std::vector<double> cellJ;
  double L;
  double spacing[3];
  inline int64_t id(int64_t i, int64_t j, int64_t k = 0) const { return i + nx * (j + ny * k); }
};

struct Solver {
  Mesh m;
  // PseudoTransientSolver.jl:28-46
  std::vector<double> u, u_prev, S, res, alpha, theta_dtau, dtau_rho;
  std::vector<double> q[3], qp[3];
  std::vector<double> cache[3];
  int bc_kind[6];
  double bc_val[6];
  int mean;  // 0 harmonic, 1 arithmetic
  int last_err_check;
  // twilight zone: mesh.centroid_coordinates.{x,y} and the forward metrics
  // cell_center_metrics.{x₁,x₂}.{ξ,η} (twilight_zone.jl:74-75, :115-118), mesh.nnodes
  std::vector<double> tz_x, tz_y, tz_xxi, tz_xeta, tz_yxi, tz_yeta;
  int tz_nn[2] = {0, 0};
  bool tz_set = false;
};

struct StepOpts {
  double t;
  int max_iter;
  double rtol, atol;
  int apply_cutoff, calculate_next_dt, subcycle_conductivity, enforce_positivity;
  double CFL;
  double ndt_tol, maximum_u_change, timestep_growth_factor;
  int norm;         // 0 max (GPU reference), 1 rms (CPU reference)
  int check_every;  // 0 = reference schedule
  int tz, no_t;     // twilight-zone forcing (step! keywords tz, no_t)
};

struct StepStats {
  double rel_err, abs_err;
  int niter, status;
  double energy_before, energy_after, source_work;
  int n_checks;
  double next_dt;
};

// averaging.jl:7-8
inline double harmonic_mean(double a, double b) { return (2.0 * a * b) / (a + b); }
inline double arithmetic_mean(double a, double b) { return (a + b) / 2.0; }
inline double face_mean(int mean, double a, double b) {
  return mean == 0 ? harmonic_mean(a, b) : arithmetic_mean(a, b);
}

// |T|^n for the power-law conductivity; integer and half-integer exponents by
// products (Julia's literal_pow for `abs(T)^3`) and one correctly rounded sqrt.
inline double pow_model(double x, double n) {
  if (n == 0.0) return 1.0;
  double twice = 2.0 * n;
  if (n > 0.0 && n <= 16.0 && twice == std::floor(twice)) {
    int m = (int)std::floor(n);
    double p = 1.0;
    if (m >= 1) {
      p = x;
      for (int e = 1; e < m; ++e) p = p * x;
    }
    if (twice != 2.0 * m) p = (m >= 1) ? p * std::sqrt(x) : std::sqrt(x);
    return p;
  }
  return std::pow(x, n);
}

// driver closures, e.g. test/integrated/2d/gaussian/run.jl:129-135
inline double kappa_model(double k0, double n, double T) {
  if (!std::isfinite(T)) return 0.0;
  return k0 * pow_model(std::fabs(T), n);
}

// ----------------------------------------------------------------------------
// boundary_operators.jl:26-263 — applybcs!(bcs, mesh, u, nhalo=1) applied in
// the order of the bcs tuple (loc = 1..2N); Periodic acts on LO locs only.
void applybcs(const Mesh& m, const int* kind, const double* val, double* u) {
  const int64_t nh = m.nh;
  const int64_t ilo = nh, ihi = nh + m.ni - 1, jlo = nh, jhi = nh + m.nj - 1;
  const int64_t klo = (m.ndim == 3) ? nh : 0, khi = (m.ndim == 3) ? nh + m.nk - 1 : 0;
  const int nloc = 2 * m.ndim;
  for (int loc = 0; loc < nloc; ++loc) {
    const int axis = loc / 2;
    const bool lo = (loc % 2) == 0;
    const int k = kind[loc];
    // iterate over the boundary slab of the given axis; the other axes run
    // over the domain only (corners are never written)
    auto slab = [&](auto&& f) {
      if (axis == 0) {
        for (int64_t kk = klo; kk <= khi; ++kk)
          for (int64_t j = jlo; j <= jhi; ++j) f(j, kk);
      } else if (axis == 1) {
        for (int64_t kk = klo; kk <= khi; ++kk)
          for (int64_t i = ilo; i <= ihi; ++i) f(i, kk);
      } else {
        for (int64_t j = jlo; j <= jhi; ++j)
          for (int64_t i = ilo; i <= ihi; ++i) f(i, j);
      }
    };
    // full index of (layer position p along axis, slab coords a,b)
    auto at = [&](int64_t p, int64_t a, int64_t b) -> int64_t {
      if (axis == 0) return m.id(p, a, b);
      if (axis == 1) return m.id(a, p, b);
      return m.id(a, b, p);
    };
    const int64_t dlo = (axis == 0) ? ilo : (axis == 1) ? jlo : klo;
    const int64_t dhi = (axis == 0) ? ihi : (axis == 1) ? jhi : khi;
    const int64_t nfull = (axis == 0) ? m.nx : (axis == 1) ? m.ny : m.nz;
    if (k == BC_NEUMANN) {  // :55-119, one layer (nhalo = 1 from step!)
      slab([&](int64_t a, int64_t b) {
        if (lo) u[at(dlo - 1, a, b)] = u[at(dlo, a, b)];
        else u[at(dhi + 1, a, b)] = u[at(dhi, a, b)];
      });
    } else if (k == BC_DIRICHLET) {
      const double v = val[loc];
      if (m.ndim == 2) {  // :137-155, every halo layer
        slab([&](int64_t a, int64_t b) {
          if (lo)
            for (int64_t p = 0; p <= dlo - 1; ++p) u[at(p, a, b)] = v;
          else
            for (int64_t p = dhi + 1; p < nfull; ++p) u[at(p, a, b)] = v;
        });
      } else {  // :178-200, one layer
        slab([&](int64_t a, int64_t b) {
          if (lo) u[at(dlo - 1, a, b)] = v;
          else u[at(dhi + 1, a, b)] = v;
        });
      }
    } else if (k == BC_PERIODIC) {  // :220-263, LO locations only
      if (lo) {
        slab([&](int64_t a, int64_t b) { u[at(dlo - 1, a, b)] = u[at(dhi, a, b)]; });
        slab([&](int64_t a, int64_t b) { u[at(dhi + 1, a, b)] = u[at(dlo, a, b)]; });
      }
    } else if (k == BC_NEG_SYMMETRY) {  // :157-175
      slab([&](int64_t a, int64_t b) {
        if (lo) u[at(dlo - 1, a, b)] = -u[at(dlo, a, b)];
        else u[at(dhi + 1, a, b)] = -u[at(dhi, a, b)];
      });
    }
  }
}

// ----------------------------------------------------------------------------
// mesh_metric_cache.jl:39-102 (2D) and :104-250 (3D)
void update_metric_cache(Solver& s) {
  const Mesh& m = s.m;
  const int64_t nh = m.nh;
  const int nd = m.ndim;
  const int64_t k0 = (nd == 3) ? nh : 0, k1 = (nd == 3) ? nh + m.nk : 1;
#pragma omp parallel for schedule(static)
  for (int64_t k = k0; k < k1; ++k)
    for (int64_t j = nh; j < nh + m.nj; ++j)
      for (int64_t i = nh; i < nh + m.ni; ++i) {
        const int64_t c = m.id(i, j, k);
        const int64_t cm[3] = {m.id(i - 1, j, k), m.id(i, j - 1, k),
                               nd == 3 ? m.id(i, j, k - 1) : 0};
        // terms summed in the reference's order: for each derivative family b
        // (the cache entry), sum over face family f and component comp of
        // metric[f][comp] * (hat_b.comp/J |_{f+1/2} - hat_b.comp/J |_{f-1/2})
        for (int b = 0; b < nd; ++b) {
          double acc = 0.0;
          bool first = true;
          for (int f = 0; f < nd; ++f) {
            const double Jp = m.edgeJ[f][c];
            const double Jm = m.edgeJ[f][cm[f]];
            for (int comp = 0; comp < nd; ++comp) {
              const double metric = m.inv[3 * f + comp][c];  // xi_x, xi_y, (eta_x, ...)
              const double plus = m.edgehat[f][3 * b + comp][c] / Jp;
              const double minus = m.edgehat[f][3 * b + comp][cm[f]] / Jm;
              const double term = metric * (plus - minus);
              acc = first ? term : acc + term;
              first = false;
            }
          }
          s.cache[b][c] = acc;
        }
      }
}

// ----------------------------------------------------------------------------
// pseudo_transient/conductivity.jl:15-23 (GPU form, no abs) over the full array
void update_conductivity(Solver& s, const double* rho, double cp, double k0, double n) {
  const int64_t N = s.m.n;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < N; ++c) s.alpha[c] = kappa_model(k0, n, s.u[c]) / (rho[c] * cp);
}

// iteration_parameters.jl:2-15 over the full array
void update_iteration_params(Solver& s, const double* rho, double Vpdtau, double dt) {
  const int64_t N = s.m.n;
  const double L = s.m.L;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < N; ++c) {
    const double a = s.alpha[c];
    const double Re = kPi + std::sqrt(kPi * kPi + (L * L * rho[c]) / (a * dt));
    const double dtau_rho = (Vpdtau * L / (a * Re));
    const double theta = (L / (Vpdtau * Re));
    // :13-14 keep only the isfinite masks (Julia: x * false == 0)
    s.dtau_rho[c] = std::isfinite(dtau_rho) ? dtau_rho : 0.0;
    s.theta_dtau[c] = std::isfinite(theta) ? theta : 0.0;
  }
}

// flux/fluxes.jl:5-26 with the face ranges of flux/fluxes_cpu.jl:33-115
// (expand_lower(domain, axis, +1)): q and q' on faces f in [lo-1, hi] along
// the axis and over the domain in the other axes.
void compute_flux(Solver& s) {
  const Mesh& m = s.m;
  const int nd = m.ndim;
  const int64_t nh = m.nh;
  for (int ax = 0; ax < nd; ++ax) {
    const int64_t i0 = nh - (ax == 0), j0 = nh - (ax == 1), k0 = (nd == 3) ? nh - (ax == 2) : 0;
    const int64_t i1 = nh + m.ni, j1 = nh + m.nj, k1 = (nd == 3) ? nh + m.nk : 1;
    const int64_t stride = (ax == 0) ? 1 : (ax == 1) ? m.nx : m.nx * m.ny;
    double* q = s.q[ax].data();
    double* qp = s.qp[ax].data();
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t k = k0; k < k1; ++k)
      for (int64_t j = j0; j < j1; ++j)
        for (int64_t i = i0; i < i1; ++i) {
          const int64_t c = m.id(i, j, k), cp1 = c + stride;
          const double a_f = face_mean(s.mean, s.alpha[c], s.alpha[cp1]);
          const double th_f = face_mean(s.mean, s.theta_dtau[c], s.theta_dtau[cp1]);
          const double du = s.u[cp1] - s.u[c];
          const double q_new = -a_f * du;
          q[c] = (q[c] * th_f + q_new) / (1.0 + th_f);
          qp[c] = -a_f * du;
        }
  }
}

// flux_divergence.jl:7-42 (2D)
inline double flux_divergence_2d(const Solver& s, const double* qi, const double* qj, int64_t i,
                                 int64_t j) {
  const Mesh& m = s.m;
  const int64_t c = m.id(i, j);
  const double xx = m.inv[0][c], xy = m.inv[1][c], ex = m.inv[3][c], ey = m.inv[4][c];
  const int64_t im = m.id(i - 1, j), jm = m.id(i, j - 1), jp = m.id(i, j + 1), ip = m.id(i + 1, j);
  const int64_t imjp = m.id(i - 1, j + 1), imjm = m.id(i - 1, j - 1), ipjm = m.id(i + 1, j - 1);
  const double dqi = qi[c] - qi[im];
  const double dqj = qj[c] - qj[jm];
  const double t1 = (xx * xx + xy * xy) * dqi;
  const double t2 = (ex * ex + ey * ey) * dqj;
  const double t3 = 0.25 * (ex * xx + ey * xy) * ((qi[jp] + qi[imjp]) - (qi[jm] + qi[imjm]));
  const double t4 = 0.25 * (ex * xx + ey * xy) * ((qj[ip] + qj[ipjm]) - (qj[im] + qj[imjm]));
  const double t5 = s.cache[0][c] * (0.5 * (qi[c] + qi[im]));
  const double t6 = s.cache[1][c] * (0.5 * (qj[c] + qj[jm]));
  return t1 + t2 + t3 + t4 + t5 + t6;
}

// flux_divergence.jl:119-239 (3D)
inline double flux_divergence_3d(const Solver& s, const double* qi, const double* qj,
                                 const double* qk, int64_t i, int64_t j, int64_t k) {
  const Mesh& m = s.m;
  const int64_t c = m.id(i, j, k);
  const double xx = m.inv[0][c], xy = m.inv[1][c], xz = m.inv[2][c];
  const double ex = m.inv[3][c], ey = m.inv[4][c], ez = m.inv[5][c];
  const double zx = m.inv[6][c], zy = m.inv[7][c], zz = m.inv[8][c];
  auto I = [&](int64_t a, int64_t b, int64_t d) { return m.id(a, b, d); };
  const double dqi = qi[c] - qi[I(i - 1, j, k)];
  const double dqj = qj[c] - qj[I(i, j - 1, k)];
  const double dqk = qk[c] - qk[I(i, j, k - 1)];
  const double t_ii = (xx * xx + xy * xy + xz * xz) * dqi;
  const double t_jj = (ex * ex + ey * ey + ez * ez) * dqj;
  const double t_kk = (zx * zx + zy * zy + zz * zz) * dqk;
  const double c_xe = 0.5 * (ex * xx + ey * xy + ez * xz);
  const double c_ez = 0.5 * (zx * ex + zy * ey + zz * ez);
  const double c_xz = 0.5 * (zx * xx + zy * xy + zz * xz);
  const double qi_eta = c_xe * (0.5 * (qi[I(i, j + 1, k)] + qi[I(i - 1, j + 1, k)]) -
                                0.5 * (qi[I(i, j - 1, k)] + qi[I(i - 1, j - 1, k)]));
  const double qj_xi = c_xe * (0.5 * (qj[I(i + 1, j, k)] + qj[I(i + 1, j - 1, k)]) -
                               0.5 * (qj[I(i - 1, j, k)] + qj[I(i - 1, j - 1, k)]));
  const double qj_zeta = c_ez * (0.5 * (qj[I(i, j, k + 1)] + qj[I(i, j - 1, k + 1)]) -
                                 0.5 * (qj[I(i, j, k - 1)] + qj[I(i, j - 1, k - 1)]));
  const double qk_eta = c_ez * (0.5 * (qk[I(i, j + 1, k)] + qk[I(i, j + 1, k - 1)]) -
                                0.5 * (qk[I(i, j - 1, k)] + qk[I(i, j - 1, k - 1)]));
  const double qi_zeta = c_xz * (0.5 * (qi[I(i, j, k + 1)] + qi[I(i - 1, j, k + 1)]) -
                                 0.5 * (qi[I(i, j, k - 1)] + qi[I(i - 1, j, k - 1)]));
  const double qk_xi = c_xz * (0.5 * (qk[I(i + 1, j, k)] + qk[I(i + 1, j, k - 1)]) -
                               0.5 * (qk[I(i - 1, j, k)] + qk[I(i - 1, j, k - 1)]));
  const double h_a = s.cache[0][c] * (0.5 * (qi[c] + qi[I(i - 1, j, k)]));
  const double h_b = s.cache[1][c] * (0.5 * (qj[c] + qj[I(i, j - 1, k)]));
  const double h_c = s.cache[2][c] * (0.5 * (qk[c] + qk[I(i, j, k - 1)]));
  return t_ii + t_jj + t_kk + qi_eta + qi_zeta + qj_xi + qj_zeta + qk_eta + qk_xi + h_a + h_b + h_c;
}

inline double divergence(const Solver& s, const std::vector<double>* q, int64_t i, int64_t j,
                         int64_t k) {
  if (s.m.ndim == 2) return flux_divergence_2d(s, q[0].data(), q[1].data(), i, j);
  return flux_divergence_3d(s, q[0].data(), q[1].data(), q[2].data(), i, j, k);
}

// ----------------------------------------------------------------------------
// Elementary functions of the twilight-zone forcing (see the header note).
// exp: Cody–Waite reduction x = k·ln2 + r with ln2 = LN2_HI + LN2_LO (nearest
// double and remainder), Taylor polynomial of e^r to degree 13, Horner with
// fused multiply-adds, times 2^k.
double exp_cw(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return std::numeric_limits<double>::infinity();
  if (x < -745.1332191019412) return 0.0;
  const double k = std::nearbyint(x * 0x1.71547652b82fep+0);
  const double r = std::fma(-k, 0x1.abc9e3b39803fp-56, std::fma(-k, 0x1.62e42fefa39efp-1, x));
  static const double inv_fact[14] = {
      0x1.0000000000000p+0,  0x1.0000000000000p+0,  0x1.0000000000000p-1,  0x1.5555555555555p-3,
      0x1.5555555555555p-5,  0x1.1111111111111p-7,  0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
      0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26,
      0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33};
  double p = inv_fact[13];
  for (int n = 12; n >= 0; --n) p = std::fma(p, r, inv_fact[n]);
  return std::ldexp(p, (int)k);
}

// sinpi: x reduced exactly modulo 2 and folded to a in [0, 1/2]; sin(πa) for
// a <= 1/4, else cos(π(1/2 - a)), each a Taylor polynomial in the square of the
// argument with coefficients (−1)^k π^(2k+1)/(2k+1)! and (−1)^k π^(2k)/(2k)!.
double sinpi(double x) {
  if (!std::isfinite(x)) return x - x;
  const double y = x - 2.0 * std::nearbyint(0.5 * x);
  const double sg = y < 0.0 ? -1.0 : 1.0;
  double a = std::fabs(y);
  if (a > 0.5) a = 1.0 - a;
  double v;
  if (a <= 0.25) {
    static const double c[9] = {0x1.921fb54442d18p+1,  -0x1.4abbce625be53p+2, 0x1.466bc6775aae2p+1,
                                -0x1.32d2cce62bd86p-1, 0x1.50783487ee782p-4,  -0x1.e3074fde8871fp-8,
                                0x1.e8f434d018d63p-12, -0x1.6fadb9f155744p-16, 0x1.aaec32af93359p-21};
    const double z = a * a;
    double p = c[8];
    for (int k = 7; k >= 0; --k) p = std::fma(p, z, c[k]);
    v = a * p;
  } else {
    static const double d[9] = {0x1.0000000000000p+0,  -0x1.3bd3cc9be45dep+2, 0x1.03c1f081b5ac4p+2,
                                -0x1.55d3c7e3cbffap+0, 0x1.e1f506891babbp-3,  -0x1.a6d1f2a204a8cp-6,
                                0x1.f9d38a3763cc3p-10, -0x1.b6e24f44b128fp-14, 0x1.20c62c2f2d7f5p-18};
    const double b = 0.5 - a;
    const double z = b * b;
    double p = d[8];
    for (int k = 7; k >= 0; --k) p = std::fma(p, z, d[k]);
    v = p;
  }
  return sg * v;
}

// twilight_zone.jl:54-195, the wavy-mesh manufactured solution with the
// nonlinear diffusivity branch (non_lin_α = true, :86).  (i, j) is the 0-based
// full-array index of a domain cell; the reference's 1-based index is i + 1.
double define_forcing_wavy(const Solver& s, const double* rho, double cp, double t, int no_t, int64_t i,
                           int64_t j) {
  const Mesh& m = s.m;
  const int64_t c = m.id(i, j);
  const int nx = s.tz_nn[0], ny = s.tz_nn[1];  // :72
  const double x = s.tz_x[c], y = s.tz_y[c];  // :74-75
  const double sv = s.S[c];                    // :77
  const double xi_x = m.inv[0][c], xi_y = m.inv[1][c], eta_x = m.inv[3][c], eta_y = m.inv[4][c];  // :80-83
  const double Lx = 12, Ly = 12;  // :89-98
  const double n_xy = 6, n_yx = 6;
  const double dx0 = Lx / (double)(nx - 1);
  const double dy0 = Ly / (double)(ny - 1);
  const double Ax = 0.2 / dx0;
  const double Ay = 0.4 / dy0;
  const double indi = (double)((i + 1) - 5) + 0.5;  // :100-101
  const double indj = (double)((j + 1) - 5) + 0.5;
  const double fwhm = 1.0, x0 = 0, y0 = 0;  // :103-105
  const double damp = 4;                    // :107
  const double pi = 3.141592653589793;
  const double xxi = s.tz_xxi[c], xeta = s.tz_xeta[c], yxi = s.tz_yxi[c], yeta = s.tz_yeta[c];  // :115-118
  const double xxixi = 0, xxieta = 0;  // :121-122
  const double K1 = pi * n_xy * dy0 / Ly;
  const double xetaeta = -dx0 * Ax * (K1 * K1) * sinpi(n_xy * (indj - 1) * dy0 / Ly);  // :123
  const double K2 = pi * n_yx * dx0 / Lx;
  const double yxixi = -dy0 * Ay * (K2 * K2) * sinpi(n_yx * (indi - 1) * dx0 / Lx);  // :124
  const double yxieta = 0, yetaeta = 0;  // :125-126
  double exy, ut;
  if (no_t) {  // :128-131
    exy = exp_cw(-(((x - x0) * (x - x0)) / fwhm + ((y - y0) * (y - y0)) / fwhm));
    ut = 0;
  } else {  // :150-153
    exy = exp_cw(-(((x - x0) * (x - x0)) / fwhm + ((y - y0) * (y - y0)) / fwhm)) * exp_cw(-damp * t);
    ut = -damp * exy;
  }
  // :132-149 (the same expressions in both branches)
  const double uxi = (-2 / fwhm) * ((x - x0) * xxi + (y - y0) * yxi) * exy;
  const double sxi = 2 * (x - x0) / fwhm * xxi + 2 * (y - y0) / fwhm * yxi;
  const double uxixi =
      (sxi * sxi - (2 / fwhm) * (xxi * xxi + yxi * yxi + (x - x0) * xxixi + (y - y0) * yxixi)) * exy;
  const double ueta = (-2 / fwhm) * ((x - x0) * xeta + (y - y0) * yeta) * exy;
  const double seta = 2 * (x - x0) / fwhm * xeta + 2 * (y - y0) / fwhm * yeta;
  const double uetaeta =
      (seta * seta - (2 / fwhm) * (xeta * xeta + yeta * yeta + (x - x0) * xetaeta + (y - y0) * yetaeta)) * exy;
  const double uxieta =
      (sxi * seta - (2 / fwhm) * (xxi * xeta + yxi * yeta + (x - x0) * xxieta + (y - y0) * yxieta)) * exy;
  // :181-189, non_lin_α = true
  const double a = s.alpha[c];
  const double e15 = exy * std::sqrt(exy);  // exy^(3/2)
  const double axi = ((5.0 / 2) * e15 * uxi) / (rho[c] * cp);
  const double aeta = ((5.0 / 2) * e15 * ueta) / (rho[c] * cp);
  const double orth_xi = (xi_x * xi_x + xi_y * xi_y) * (axi * uxi + a * uxixi);
  const double orth_eta = (eta_x * eta_x + eta_y * eta_y) * (aeta * ueta + a * uetaeta);
  const double cross = (xi_x * eta_x + xi_y * eta_y) * (2 * a * uxieta + aeta * uxi + axi * ueta);
  const double non_orth_xi = a * s.cache[0][c] * uxi;
  const double non_orth_eta = a * s.cache[1][c] * ueta;
  return ut - orth_xi - orth_eta - cross - non_orth_xi - non_orth_eta - sv;  // :191
}

// update.jl:2-21 over the domain (in place: each cell reads only its own u);
// with the twilight zone, update.jl:23-71
void compute_update(Solver& s, double dt, const double* rho, double cp, const StepOpts& o) {
  const Mesh& m = s.m;
  const int64_t nh = m.nh;
  const int64_t k0 = (m.ndim == 3) ? nh : 0, k1 = (m.ndim == 3) ? nh + m.nk : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = k0; k < k1; ++k)
    for (int64_t j = nh; j < nh + m.nj; ++j)
      for (int64_t i = nh; i < nh + m.ni; ++i) {
        const int64_t c = m.id(i, j, k);
        const double dq = divergence(s, s.q, i, j, k);
        if (o.tz) {
          const double f = define_forcing_wavy(s, rho, cp, o.t, o.no_t, i, j);
          s.u[c] = ((s.u[c] + s.dtau_rho[c] * (s.u_prev[c] / dt - dq + s.S[c] + f)) /
                    (1.0 + s.dtau_rho[c] / dt));
        } else {
          s.u[c] = ((s.u[c] + s.dtau_rho[c] * (s.u_prev[c] / dt - dq + s.S[c])) /
                    (1.0 + s.dtau_rho[c] / dt));
        }
      }
}

// Julia isapprox(x, y; rtol) with atol = 0
inline bool isapprox(double x, double y, double rtol) {
  if (x == y) return true;
  if (!(std::isfinite(x) && std::isfinite(y))) return false;
  return std::fabs(x - y) <= rtol * std::max(std::fabs(x), std::fabs(y));
}

// residuals.jl:24-47 over the domain (res halo stays 0); with the twilight
// zone, residuals.jl:49-99
void update_residual(Solver& s, double dt, const double* rho, double cp, const StepOpts& o) {
  const Mesh& m = s.m;
  const int64_t nh = m.nh;
  const double eps = std::numeric_limits<double>::epsilon();
  const int64_t k0 = (m.ndim == 3) ? nh : 0, k1 = (m.ndim == 3) ? nh + m.nk : 1;
#pragma omp parallel for collapse(2) schedule(static)
  for (int64_t k = k0; k < k1; ++k)
    for (int64_t j = nh; j < nh + m.nj; ++j)
      for (int64_t i = nh; i < nh + m.ni; ++i) {
        const int64_t c = m.id(i, j, k);
        const double dq = divergence(s, s.qp, i, j, k);
        const double un = s.u[c], unm1 = s.u_prev[c];
        double du = un - unm1;
        if (isapprox(un, unm1, eps)) du = 0.0;  // du * !isapprox (strong zero)
        if (o.tz) s.res[c] = -du / dt - dq + s.S[c] + define_forcing_wavy(s, rho, cp, o.t, o.no_t, i, j);
        else s.res[c] = -du / dt - dq + s.S[c];
      }
}

// residuals.jl:1-22
double residual_norm(const Solver& s, int kind) {
  const int64_t N = s.m.n;
  if (kind == 0) {  // GPU: norm(A, Inf) / sqrt(length(A)); NaN propagates
    double mx = 0.0;
    bool nan = false;
    for (int64_t c = 0; c < N; ++c) {
      const double a = std::fabs(s.res[c]);
      if (a != a) nan = true;
      else if (a > mx) mx = a;
    }
    if (nan) return std::numeric_limits<double>::quiet_NaN();
    return mx / std::sqrt((double)N);
  }
  double acc = 0.0;  // CPU: sqrt(sum(a^2) / length(a))
#pragma omp parallel for reduction(+ : acc) schedule(static)
  for (int64_t c = 0; c < N; ++c) acc += s.res[c] * s.res[c];
  return std::sqrt(acc / (double)N);
}

// validity_checks.jl:1-43 on the domain and the first halo layer of each side
// (corners excluded).  Returns false when the field is invalid.
bool validate_scalar(const Mesh& m, const double* a, bool positivity) {
  const int64_t nh = m.nh;
  const int nd = m.ndim;
  auto ok = [&](double v) { return std::isfinite(v) && (!positivity || v >= 0.0); };
  const int64_t k0 = (nd == 3) ? nh - 1 : 0, k1 = (nd == 3) ? nh + m.nk + 1 : 1;
  for (int64_t k = k0; k < k1; ++k)
    for (int64_t j = nh - 1; j < nh + m.nj + 1; ++j)
      for (int64_t i = nh - 1; i < nh + m.ni + 1; ++i) {
        const int outside = (i < nh || i >= nh + m.ni) + (j < nh || j >= nh + m.nj) +
                            (nd == 3 ? (k < nh || k >= nh + m.nk) : 0);
        if (outside > 1) continue;  // corner / edge of the halo shell
        if (!ok(a[m.id(i, j, k)])) return false;
      }
  return true;
}

// timestep_control.jl:33-73
double next_dt(const Solver& s, double dt, double tol, double max_change, double growth) {
  const int64_t N = s.m.n;
  double umax = -std::numeric_limits<double>::infinity();
  bool nan = false;
  for (int64_t c = 0; c < N; ++c) {  // maximum(u^n), NaN propagates
    const double v = s.u_prev[c];
    if (v != v) nan = true;
    else if (v > umax) umax = v;
  }
  if (nan) umax = std::numeric_limits<double>::quiet_NaN();
  const double u0 = umax * tol;
  double mx = -std::numeric_limits<double>::infinity();
  for (int64_t c = 0; c < N; ++c) {  // GPU mapreduce(f, max, u^{n+1}, u^n)
    const double a = s.u[c], b = s.u_prev[c];
    double d = std::fabs(a - b) / (a + u0);
    d = std::isfinite(d) ? d : 0.0;
    if (d > mx) mx = d;
  }
  const double cand = dt * std::sqrt(std::fabs(max_change / mx));
  const double cap = growth * dt;
  return (cand < cap) ? cand : cap;  // min(); cand is never NaN here
}

double energy(const Solver& s, const double* T, const double* rho, double cp) {
  const Mesh& m = s.m;
  const int64_t nh = m.nh;
  const int64_t k0 = (m.ndim == 3) ? nh : 0, k1 = (m.ndim == 3) ? nh + m.nk : 1;
  double acc = 0.0;
  for (int64_t k = k0; k < k1; ++k)
    for (int64_t j = nh; j < nh + m.nj; ++j)
      for (int64_t i = nh; i < nh + m.ni; ++i) {
        const int64_t c = m.id(i, j, k);
        acc += rho[c] * cp * T[c] * m.cellJ[c];
      }
  return acc;
}

double source_integral(const Solver& s) {
  const Mesh& m = s.m;
  const int64_t nh = m.nh;
  const int64_t k0 = (m.ndim == 3) ? nh : 0, k1 = (m.ndim == 3) ? nh + m.nk : 1;
  double acc = 0.0;
  for (int64_t k = k0; k < k1; ++k)
    for (int64_t j = nh; j < nh + m.nj; ++j)
      for (int64_t i = nh; i < nh + m.ni; ++i) {
        const int64_t c = m.id(i, j, k);
        acc += s.S[c] * m.cellJ[c];
      }
  return acc;
}

// PseudoTransientSolver.jl:180-351
int step(Solver& s, double* T, const double* rho, double cp, double k0, double n, double dt,
         const StepOpts& o, StepStats* st) {
  const Mesh& m = s.m;
  const int64_t N = m.n;
  // :206-208 adaptive check schedule from the previous step's iteration count
  const int last = s.last_err_check;
  const int min_err_check = (int)std::nearbyint(last * 0.9);  // round-half-even
  const int err_interval = std::max(1, (last - min_err_check) / 2);

  int iter = 0;
  double rel_error = 2 * o.rtol, abs_error = 2 * o.atol;
  double init_L2 = std::numeric_limits<double>::infinity();
  double min_spacing = m.spacing[0];
  for (int d = 1; d < m.ndim; ++d) min_spacing = std::min(min_spacing, m.spacing[d]);
  const double Vpdtau = o.CFL * min_spacing;  // :223
  st->n_checks = 0;
  if (!(dt > 0) || !(Vpdtau > 0)) {  // :225-227
    st->status = ST_BAD_INPUT;
    return ST_BAD_INPUT;
  }
  if (o.tz && (m.ndim != 2 || !s.tz_set)) {  // the forcing is 2D (twilight_zone.jl:70)
    st->status = ST_BAD_INPUT;
    return ST_BAD_INPUT;
  }
  std::memcpy(s.u.data(), T, sizeof(double) * N);  // :229-230
  std::memcpy(s.u_prev.data(), T, sizeof(double) * N);
  update_metric_cache(s);  // :232
  st->energy_before = energy(s, T, rho, cp);
  st->source_work = dt * source_integral(s);
  // :238-250
  if (!validate_scalar(m, s.alpha.data(), o.enforce_positivity != 0) ||
      !validate_scalar(m, s.S.data(), false)) {
    st->status = ST_BAD_INPUT;
    return ST_BAD_INPUT;
  }
  int status = ST_OK;
  while (true) {  // :253-319
    applybcs(m, s.bc_kind, s.bc_val, s.u.data());
    if (o.subcycle_conductivity || iter == 0) {
      update_conductivity(s, rho, cp, k0, n);
      update_iteration_params(s, rho, Vpdtau, dt);
    }
    iter += 1;
    compute_flux(s);
    compute_update(s, dt, rho, cp, o);
    bool check;
    if (o.check_every > 0) check = (iter % o.check_every == 0) || iter == 1;
    else check = (iter >= min_err_check && iter % err_interval == 0) || iter == 1;
    if (check) {
      update_residual(s, dt, rho, cp, o);
      st->n_checks++;
      const double L2 = residual_norm(s, o.norm);
      if (iter == 1) init_L2 = L2;
      rel_error = L2 / init_L2;
      abs_error = L2;
    }
    if (!std::isfinite(rel_error) || !std::isfinite(abs_error)) {
      status = ST_NONFINITE;
      break;
    }
    if (iter > o.max_iter) {
      status = ST_MAX_ITER;
      break;
    }
    if (rel_error <= o.rtol || abs_error <= o.atol) break;
  }
  // :321 is reached only when the loop ends without error()
  if (status == ST_OK) s.last_err_check = iter;
  st->rel_err = rel_error;
  st->abs_err = abs_error;
  st->niter = iter;
  st->status = status;
  if (status != ST_OK) return status;
  if (o.enforce_positivity)  // :323-327
    for (int64_t c = 0; c < N; ++c) s.u[c] = std::fabs(s.u[c]);
  if (o.apply_cutoff)  // :329-331, cutoff! :357-368
    for (int64_t c = 0; c < N; ++c) {
      const double a = s.u[c];
      s.u[c] = std::isfinite(a) ? 0.5 * (std::fabs(a) + a) : 0.0;
    }
  st->next_dt = o.calculate_next_dt
                    ? next_dt(s, dt, o.ndt_tol, o.maximum_u_change, o.timestep_growth_factor)
                    : dt;
  std::memcpy(T, s.u.data(), sizeof(double) * N);  // :346
  st->energy_after = energy(s, T, rho, cp);
  return ST_OK;
}

void alloc_fields(Solver& s) {
  const int64_t N = s.m.n;
  for (auto* v : {&s.u, &s.u_prev, &s.S, &s.res, &s.alpha, &s.theta_dtau, &s.dtau_rho})
    v->assign(N, 0.0);
  for (int d = 0; d < s.m.ndim; ++d) {
    s.q[d].assign(N, 0.0);
    s.qp[d].assign(N, 0.0);
    s.cache[d].assign(N, 0.0);
  }
}

}  // namespace

// ============================================================================
// extern "C" surface used by the test-suite (ctypes)
extern "C" {

// cell_inv: 9 pointers (a*3+c), edge_J: 3 pointers, edge_hat: 27 pointers
// (f*9 + a*3 + c); unused components may be NULL.
void* oracle_create(int ndim, int ni, int nj, int nk, int nhalo, const double* const* cell_inv,
                    const double* cellJ, const double* const* edge_J,
                    const double* const* edge_hat, double L, const double* spacing,
                    const int* bc_kind, const double* bc_val, int mean) {
  Solver* s = new Solver();
  Mesh& m = s->m;
  m.ndim = ndim;
  m.ni = ni;
  m.nj = nj;
  m.nk = (ndim == 3) ? nk : 1;
  m.nh = nhalo;
  m.nx = ni + 2 * nhalo;
  m.ny = nj + 2 * nhalo;
  m.nz = (ndim == 3) ? nk + 2 * nhalo : 1;
  m.n = m.nx * m.ny * m.nz;
  for (int a = 0; a < ndim; ++a)
    for (int c = 0; c < ndim; ++c) m.inv[3 * a + c].assign(cell_inv[3 * a + c], cell_inv[3 * a + c] + m.n);
  m.cellJ.assign(cellJ, cellJ + m.n);
  for (int f = 0; f < ndim; ++f) {
    m.edgeJ[f].assign(edge_J[f], edge_J[f] + m.n);
    for (int a = 0; a < ndim; ++a)
      for (int c = 0; c < ndim; ++c) {
        const double* p = edge_hat[9 * f + 3 * a + c];
        m.edgehat[f][3 * a + c].assign(p, p + m.n);
      }
  }
  m.L = L;
  for (int d = 0; d < 3; ++d) m.spacing[d] = (d < ndim) ? spacing[d] : 0.0;
  for (int l = 0; l < 2 * ndim; ++l) {
    s->bc_kind[l] = bc_kind[l];
    s->bc_val[l] = bc_val[l];
  }
  s->mean = mean;
  s->last_err_check = 0;
  alloc_fields(*s);
  return s;
}

void oracle_destroy(void* h) { delete static_cast<Solver*>(h); }

void oracle_set_source(void* h, const double* S) {
  Solver* s = static_cast<Solver*>(h);
  std::memcpy(s->S.data(), S, sizeof(double) * s->m.n);
}

void oracle_get_state(void* h, double* q, int* last) {
  Solver* s = static_cast<Solver*>(h);
  for (int d = 0; d < s->m.ndim; ++d) std::memcpy(q + d * s->m.n, s->q[d].data(), sizeof(double) * s->m.n);
  *last = s->last_err_check;
}

void oracle_set_state(void* h, const double* q, int last) {
  Solver* s = static_cast<Solver*>(h);
  for (int d = 0; d < s->m.ndim; ++d) std::memcpy(s->q[d].data(), q + d * s->m.n, sizeof(double) * s->m.n);
  s->last_err_check = last;
}

void oracle_get_cache(void* h, double* out) {
  Solver* s = static_cast<Solver*>(h);
  update_metric_cache(*s);
  for (int d = 0; d < s->m.ndim; ++d) std::memcpy(out + d * s->m.n, s->cache[d].data(), sizeof(double) * s->m.n);
}

// opts: doubles {t, rtol, atol, CFL, ndt_tol, maximum_u_change, timestep_growth_factor}
//       ints    {max_iter, apply_cutoff, calculate_next_dt, subcycle_conductivity,
//                enforce_positivity, norm, check_every, tz, no_t}
// out:  doubles {rel_err, abs_err, next_dt, energy_before, energy_after, source_work}
//       ints    {niter, status, n_checks}
int oracle_step(void* h, double* T, const double* rho, double cp, double k0, double n, double dt,
                const double* od, const int* oi, double* outd, int* outi) {
  Solver* s = static_cast<Solver*>(h);
  StepOpts o;
  o.t = od[0];
  o.rtol = od[1];
  o.atol = od[2];
  o.CFL = od[3];
  o.ndt_tol = od[4];
  o.maximum_u_change = od[5];
  o.timestep_growth_factor = od[6];
  o.max_iter = oi[0];
  o.apply_cutoff = oi[1];
  o.calculate_next_dt = oi[2];
  o.subcycle_conductivity = oi[3];
  o.enforce_positivity = oi[4];
  o.norm = oi[5];
  o.check_every = oi[6];
  o.tz = oi[7];
  o.no_t = oi[8];
  StepStats st{};
  st.next_dt = dt;
  int rc = step(*s, T, rho, cp, k0, n, dt, o, &st);
  outd[0] = st.rel_err;
  outd[1] = st.abs_err;
  outd[2] = st.next_dt;
  outd[3] = st.energy_before;
  outd[4] = st.energy_after;
  outd[5] = st.source_work;
  outi[0] = st.niter;
  outi[1] = st.status;
  outi[2] = st.n_checks;
  return rc;
}

// twilight-zone inputs: centroids, forward metrics (full-size arrays) and mesh.nnodes
void oracle_set_tz(void* h, const double* x, const double* y, const double* xxi, const double* xeta,
                   const double* yxi, const double* yeta, int nnx, int nny) {
  Solver* s = static_cast<Solver*>(h);
  const int64_t n = s->m.n;
  s->tz_x.assign(x, x + n);
  s->tz_y.assign(y, y + n);
  s->tz_xxi.assign(xxi, xxi + n);
  s->tz_xeta.assign(xeta, xeta + n);
  s->tz_yxi.assign(yxi, yxi + n);
  s->tz_yeta.assign(yeta, yeta + n);
  s->tz_nn[0] = nnx;
  s->tz_nn[1] = nny;
  s->tz_set = true;
}

// the elementary functions of the forcing, for the test-suite's accuracy checks
double oracle_exp_cw(double x) { return exp_cw(x); }
double oracle_sinpi(double x) { return sinpi(x); }

// standalone applybcs! on a full-size array (BC known-answer tests)
void oracle_applybcs(int ndim, int ni, int nj, int nk, int nhalo, const int* bc_kind,
                     const double* bc_val, double* u) {
  Mesh m;
  m.ndim = ndim;
  m.ni = ni;
  m.nj = nj;
  m.nk = (ndim == 3) ? nk : 1;
  m.nh = nhalo;
  m.nx = ni + 2 * nhalo;
  m.ny = nj + 2 * nhalo;
  m.nz = (ndim == 3) ? nk + 2 * nhalo : 1;
  m.n = m.nx * m.ny * m.nz;
  applybcs(m, bc_kind, bc_val, u);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
