// cdm_device.cuh — device-side data structures and the per-cell arithmetic of
// the APT path, shared by the FP64 sweep, the auxiliary kernels and the host.
//
// Floating-point expressions keep the operation order of the reference
// (src/pseudo_transient/*.jl); the FP64 translation units are compiled with
// -fmad=false so that no multiply-add is contracted, which makes the FP64 path
// reproduce the CPU restatement bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cdm {

constexpr double kPi = 3.14159265358979323846;
// wavefront schedule: added to a problem's launch iteration count once it is done
constexpr int kWaveDone = 1 << 24;

// Resolved ghost-cell rule of one boundary side (applybcs! order semantics,
// boundary_operators.jl:26-30, folded into one rule per side on the host).
enum GhostRule : int { GR_NEUMANN = 0, GR_DIRICHLET = 1, GR_PERIODIC = 2, GR_NEGSYM = 3, GR_NONE = 4 };

enum Status : int { ST_OK = 0, ST_MAX_ITER = 1, ST_NONFINITE = 2, ST_BAD_INPUT = 3 };

// Per-problem control block: the state of step!'s pseudo-time loop
// (PseudoTransientSolver.jl:206-221, :280-318) kept on the device so that the
// stopping rule is evaluated without a host round trip.
struct Ctrl {
  int iter;          // completed pseudo-iterations of this step
  int done;          // 1 once converged or failed
  int status;        // enum Status
  int min_err_check; // :207
  int err_interval;  // :208
  int max_iter;
  int check_every;   // 0: reference schedule
  int norm_kind;     // 0 max (GPU reference), 1 rms
  double rtol, atol;
  double init_L2, rel, abs;
  unsigned int arrive;  // blocks of the current iteration that finished
  int n_checks;
  int abad[2];          // diffusivity validity bits of the last two iterations
  int init_fixed;       // 1: init_L2 was set before the loop (guessed start)
  double sqrtN;         // sqrt(length(res)) over the full array
  double nfull;
  // mixed precision bookkeeping
  int n_restarts;
  int inner_iter;       // FP32 sweeps since the last restart
  double restart_L2;    // FP64 residual max|R| at the last restart (not normalised)
  double inner_L2;      // FP32 correction residual max|r| at the last inner check
  double inner_target;  // inner cycle ends when max|r| <= inner_target
  int inner_done;       // set on the device when the inner target is met
  int inner_check_every;
  int restart_nan;
  int inner_stall;      // inner checks since the last new best
  double inner_best;    // best max|r| of the cycle
  // wavefront schedule: the iteration count this step is expected to take
  // (the previous step's, last_err_check); 0 when unknown
  int est_iter;
};

// Kernel-facing description of one problem (one mesh, one step! call).
struct Problem {
  int ndim, ni, nj, nk, nh;
  int nx, ny, nz;                   // full sizes
  int tiles_i, tiles_j, tiles_k, ntiles;
  int strip_h;                      // row-marching kernels: rows per strip
  int mean;                         // 0 harmonic, 1 arithmetic
  int subcycle;                     // subcycle_conductivity
  int kmode, km, khalf;             // conductivity exponent decomposition
  int qpar;                         // ping-pong index of q holding the state
  int item0;                        // wavefront schedule: index of the problem's first strip in the
                                    // item list, -1 when it has none
  int rule[6];
  double val[6];
  double dt, cp, k0, kn, L, LL, Vpdtau, VpL;
  double* u[2];                     // ping-pong temperature iterates
  double* q[2][3];                  // ping-pong damped fluxes
  const double* u_prev;             // T^n
  const double* S;                  // source term
  const double* rho;                // density (user or staged)
  const double* coef[9];            // packed metric coefficients (see coef_layout)
  double* partial;                  // per-tile reduction partials
  Ctrl* ctrl;
  // mixed precision (FP32 correction sweeps)
  float* d32[2];                    // correction iterates
  float* e32[2][3];                 // damped-flux corrections
  float* ub32;                      // base temperature (FP32 copy)
  float* ab32;                      // diffusivity at the base state
  float* R32;                       // FP64 residual of the base state, rounded
  const float* rho32;
  const float* coef32[9];
  double* ub64[2];                  // base temperature, FP64 ping-pong
  // twilight zone: the α-independent forcing terms of the step (tz::kNumTerms
  // full-size arrays back to back, nx*ny apart), NULL when the forcing is off
  const double* tz;
};

// Copy of a problem descriptor into shared memory by the whole block, ending
// with a barrier.  The 3D plane marches (FP64 and the FP32 correction sweep)
// read the descriptor's sizes, scalars and array pointers throughout their
// loops; from shared memory those reads are short-latency loads instead of L1
// round trips (their register budgets do not hold all of them), and one copy
// serves a whole strip.  The 2D wavefront
// kernel changes problem at every ticket and keeps reading the descriptor
// from global memory: there the copy's latency, exposed once per ticket, cost
// more than it saved.  The descriptor is constant during a launch.
template <int NT>
__device__ __forceinline__ void stage_problem(Problem& dst, const Problem* __restrict__ src) {
  static_assert(sizeof(Problem) % 8 == 0, "descriptor copied in 8-byte words");
  const long long* s = reinterpret_cast<const long long*>(src);
  long long* d = reinterpret_cast<long long*>(&dst);
  for (int w = threadIdx.x; w < (int)(sizeof(Problem) / 8); w += NT) d[w] = s[w];
  __syncthreads();
}

// asynchronous 8-byte copy global -> shared memory (cp.async, L1-allocating:
// for arrays no block writes during the launch), its group commit and wait
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__host__ __device__ inline int64_t fidx(const Problem& P, int a, int b, int c = 0) {
  // domain coordinates (a, b, c) -> full-array offset
  return (int64_t)(a + P.nh) + (int64_t)P.nx * ((int64_t)(b + P.nh) + (int64_t)P.ny * (int64_t)(c + (P.ndim == 3 ? P.nh : 0)));
}

// |T|^n: integer and half-integer exponents by left-to-right products and one
// correctly rounded sqrt (same expression as the CPU restatement).
__device__ __forceinline__ double pow_model(double x, int mode, int m, int half, double n) {
  if (mode == 0) return 1.0;
  if (mode == 1) {
    double p = 1.0;
    if (m >= 1) {
      p = x;
      for (int e = 1; e < m; ++e) p = __dmul_rn(p, x);
    }
    if (half) p = (m >= 1) ? __dmul_rn(p, sqrt(x)) : sqrt(x);
    return p;
  }
  return pow(x, n);
}

// kappa(rho, T) of the drivers (e.g. test/integrated/2d/gaussian/run.jl:129-135)
// divided by rho*cp as in pseudo_transient/conductivity.jl:20
__device__ __forceinline__ double diffusivity(const Problem& P, double T, double rho) {
  double kap = isfinite(T) ? __dmul_rn(P.k0, pow_model(fabs(T), P.kmode, P.km, P.khalf, P.kn)) : 0.0;
  return kap / (rho * P.cp);
}

// iteration_parameters.jl:2-15
__device__ __forceinline__ void iter_params(const Problem& P, double alpha, double rho, double& dtau_rho,
                                            double& theta) {
  const double Re = kPi + sqrt(kPi * kPi + (P.LL * rho) / (alpha * P.dt));
  const double d = P.VpL / (alpha * Re);
  const double t = P.L / (P.Vpdtau * Re);
  dtau_rho = isfinite(d) ? d : 0.0;
  theta = isfinite(t) ? t : 0.0;
}

// averaging.jl:7-8
__device__ __forceinline__ double face_mean(int mean, double a, double b) {
  return mean == 0 ? (2.0 * a * b) / (a + b) : (a + b) / 2.0;
}

// Julia isapprox(x, y; rtol) with atol = 0 (residuals.jl:44)
__device__ __forceinline__ bool isapprox_eps(double x, double y) {
  if (x == y) return true;
  if (!(isfinite(x) && isfinite(y))) return false;
  return fabs(x - y) <= 2.220446049250313e-16 * fmax(fabs(x), fabs(y));
}

// reference check schedule (PseudoTransientSolver.jl:280)
__device__ __forceinline__ bool is_check_iter(const Ctrl* C, int it) {
  if (C->check_every > 0) return (it % C->check_every == 0) || it == 1;
  return (it >= C->min_err_check && it % C->err_interval == 0) || it == 1;
}

__device__ __forceinline__ int ld_cg_int(const int* p) {
  int v;
  asm volatile("ld.global.cg.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_cg_double(const double* p) {
  double v;
  asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// ghost value of side `side` (0 ilo, 1 ihi, 2 jlo, 3 jhi, 4 klo, 5 khi) at the
// ghost cell (a, b, c); `src` is the field the rule reads (u or u_prev)
__device__ __forceinline__ double ghost_value(const Problem& P, const double* __restrict__ src,
                                              int side, int a, int b, int c) {
  const int rule = P.rule[side];
  if (rule == GR_DIRICHLET) return P.val[side];
  const int axis = side >> 1;
  const bool lo = (side & 1) == 0;
  const int n = axis == 0 ? P.ni : (axis == 1 ? P.nj : P.nk);
  int p;  // position along the axis of the cell the rule reads
  if (rule == GR_NONE) p = lo ? -1 : n;
  else if (rule == GR_PERIODIC) p = lo ? n - 1 : 0;
  else p = lo ? 0 : n - 1;  // Neumann, negative symmetry
  int aa = a, bb = b, cc = c;
  if (axis == 0) aa = p;
  else if (axis == 1) bb = p;
  else cc = p;
  const double v = src[fidx(P, aa, bb, cc)];
  return rule == GR_NEGSYM ? -v : v;
}

// classify a ring cell: returns -1 if it is neither a domain cell nor a
// first-layer (non-corner) ghost, else 6 for a domain cell or the side index
__device__ __forceinline__ int classify(const Problem& P, int a, int b, int c) {
  const bool ia = a >= 0 && a < P.ni, ib = b >= 0 && b < P.nj;
  const bool ic = (P.ndim == 2) || (c >= 0 && c < P.nk);
  if (ia && ib && ic) return 6;
  if (ib && ic && (a == -1 || a == P.ni)) return a < 0 ? 0 : 1;
  if (ia && ic && (b == -1 || b == P.nj)) return b < 0 ? 2 : 3;
  if (P.ndim == 3 && ia && ib && (c == -1 || c == P.nk)) return c < 0 ? 4 : 5;
  return -1;
}

}  // namespace cdm
