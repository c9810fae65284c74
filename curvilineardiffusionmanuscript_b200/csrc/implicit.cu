// implicit.cu — the reference's implicit scheme on the GPU: backward Euler in
// the conservative curvilinear form, one linear system per time step, solved by
// a Krylov method (src/implicit/ImplictSolver.jl, init_matrix.jl,
// inner_operators.jl, stencils.jl, src/edge_terms.jl).  It is the comparator of
// the manuscript's pseudo-transient-versus-Krylov study, next to the APT path.
//
// The linear system lives on the diffusion region: the domain plus one halo
// layer (ImplictSolver.jl:77-98), rows column-major over it (n1 = ni + 2 fast).
// Interior rows hold the 9-point stencil of stencils.jl:14-40, stored by
// stencil entry ([entry][row], so the SpMV reads each entry coalesced); boundary
// rows are the constraints of init_matrix.jl (1 on the diagonal, -1 at the
// interior or opposite cell for Neumann and periodic sides, nothing for
// Dirichlet; corners keep the diagonal only) and are applied from the side
// rules, not stored.  The assembly keeps the reference's evaluation order
// (compiled without contracted multiply-adds), so A and b equal the CPU
// restatement's bit for bit.
//
// Solver: BiCGSTAB with the Jacobi (diagonal) preconditioner applied on the
// right, so the residual it tracks is the residual of the system itself; it
// stops at the reference's rule ||b - A x||_2 <= atol + rtol ||b - A x0||_2
// (Krylov.jl's stopping test for GMRES with a right preconditioner, the
// reference's solver), confirmed on the true residual b - A x before it
// returns.  The first solve starts from zero, later ones from the previous
// solution (ImplictSolver.jl:282-303).  The reference's GMRES + ILU(0) and
// this solver reach the same solution to that tolerance; their iteration
// counts differ (a BiCGSTAB iteration applies A twice).
//
// Every Krylov scalar is reduced on the device (per-block partials, the last
// block of a launch sums them in a fixed order, so results do not depend on
// timing) and the stopping rule is evaluated there; kPollIters iterations
// (five kernels each, which return at once after the rule has stopped the
// solve) are replayed from one CUDA graph between host polls.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "cdm_apt.h"
#include "cdm_device.cuh"
#include "engine.h"

namespace cdm {
namespace imp {

constexpr int NT = 256;
constexpr int kPollIters = 16;

// Krylov state on the device
struct KState {
  double rho0, rho1, alpha, omega, rv, ts, tt, rr, r0n, tol;
  double umax, maxrel;  // next_dt reductions
  int iter, done, status, conv, max_iter, pad;
  unsigned int arrive[4];
};

enum { KS_OK = 0, KS_MAX_ITER = 1, KS_NONFINITE = 2 };
enum { CONV_NO = 0, CONV_TOL = 1, CONV_BREAKDOWN = 2 };

struct Geo {
  int nd;                  // 2 or 3
  int ni, nj, nk, nh;      // domain cells (nk = 1 in 2D), halo layers of the mesh arrays
  int nx, ny;              // full row and column lengths of the mesh arrays
  int n1, n2, n3;          // diffusion region (n3 = 1 in 2D)
  long long N;
  int kind[6];             // side kinds (cdm_bc_kind): ilo, ihi, jlo, jhi, klo, khi
  double val[6];           // Dirichlet values
  int rule[6];             // ghost rules of applybcs! (GhostRule, folded per side)
};

__device__ __forceinline__ void row_pos(const Geo& g, int r, int& i2, int& j2, int& k2) {
  const unsigned plane = (unsigned)g.n1 * (unsigned)g.n2;
  k2 = (int)((unsigned)r / plane);
  const int rem = r - k2 * (int)plane;
  j2 = (int)((unsigned)rem / (unsigned)g.n1);
  i2 = rem - j2 * g.n1;
}

__device__ __forceinline__ long long mesh_index(const Geo& g, int i2, int j2, int k2) {
  const long long kz = g.nd == 3 ? (long long)(k2 - 1 + g.nh) : 0;
  return (long long)(i2 - 1 + g.nh) + (long long)g.nx * ((long long)(j2 - 1 + g.nh) + (long long)g.ny * kz);
}

// number of region-2 coordinates on the region's boundary (0: interior row)
__device__ __forceinline__ int on_boundary(const Geo& g, int i2, int j2, int k2) {
  return (i2 == 0 || i2 == g.n1 - 1) + (j2 == 0 || j2 == g.n2 - 1) + (g.nd == 3 && (k2 == 0 || k2 == g.n3 - 1));
}

// the column of the one off-diagonal entry of a boundary row, -1 for none
// (init_matrix.jl:69-167, :252-390: a side's rows over the interior range of
// the other axes; Dirichlet rows, edges and corners have the diagonal only)
__device__ __forceinline__ long long partner(const Geo& g, int i2, int j2, int k2, long long r) {
  if (on_boundary(g, i2, j2, k2) != 1) return -1;
  int side, n;
  long long st;
  if (i2 == 0 || i2 == g.n1 - 1) {
    side = i2 == 0 ? 0 : 1;
    st = 1;
    n = g.n1;
  } else if (j2 == 0 || j2 == g.n2 - 1) {
    side = j2 == 0 ? 2 : 3;
    st = g.n1;
    n = g.n2;
  } else {
    side = k2 == 0 ? 4 : 5;
    st = (long long)g.n1 * g.n2;
    n = g.n3;
  }
  const bool lo = (side & 1) == 0;
  if (g.kind[side] == CDM_BC_NEUMANN) return lo ? r + st : r - st;
  if (g.kind[side] == CDM_BC_PERIODIC) return lo ? r + (long long)(n - 2) * st : r - (long long)(n - 2) * st;
  return -1;
}

// ------------------------------------------------------------ block reductions
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* s_red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) s_red[k * (NT / 32) + warp] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < NT / 32; ++w) s += s_red[k * (NT / 32) + w];
      v[k] = s;
    }
}

// every block stores its K partial sums, the last block to arrive sums all
// blocks' partials in block order into out[0..K) (thread 0) and returns true
template <int K>
__device__ bool grid_sum(double (&v)[K], double* part, unsigned int* arrive, double* s_red, int* s_last,
                         double* out) {
  block_sum<K>(v, s_red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) part[(size_t)blockIdx.x * K + k] = v[k];
    __threadfence();
    *s_last = atomicAdd(arrive, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!*s_last) return false;
  __threadfence();
  double w[K];
#pragma unroll
  for (int k = 0; k < K; ++k) w[k] = 0.0;
  // fixed partition of the partials over the threads, fixed tree: deterministic
  for (unsigned b = threadIdx.x; b < gridDim.x; b += NT)
#pragma unroll
    for (int k = 0; k < K; ++k) w[k] += ((volatile double*)part)[(size_t)b * K + k];
  block_sum<K>(w, s_red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) out[k] = w[k];
    *arrive = 0u;
  }
  return true;
}

// --------------------------------------------------------------- set-up work
// applybcs! (boundary_operators.jl:26-263) on a full mesh array, every side in
// one launch: a side writes only its own ghost slab (the other axes over the
// domain, edges and corners never written) and reads only domain cells, so
// the sides do not depend on one another.  blockIdx.y = side.
__global__ void ghost_fill(Geo g, double* u) {
  const int side = blockIdx.y, axis = side >> 1;
  const bool lo = (side & 1) == 0;
  const int rule = g.rule[side];
  const int nh = g.nh;
  const int dims[3] = {g.ni, g.nj, g.nk};
  const int e0 = axis == 0 ? g.nj : g.ni;                       // first other axis (domain extent)
  const int e1 = axis == 2 ? g.nj : (g.nd == 3 ? g.nk : 1);     // second other axis
  const long long sx = 1, sy = g.nx, sz = (long long)g.nx * g.ny;
  const long long sa = axis == 0 ? sx : axis == 1 ? sy : sz;    // stride along the axis
  const long long s0 = axis == 0 ? sy : sx;
  const long long s1 = axis == 2 ? sy : sz;
  const int k0 = g.nd == 3 ? nh : 0;                            // full offset of the second other axis (2D: z = 0)
  const int dlo = nh, dhi = nh + dims[axis] - 1, nfull = dims[axis] + 2 * nh;
  const long long len = (long long)e0 * e1;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < len; q += (long long)gridDim.x * blockDim.x) {
    const int a0 = (int)(q % e0), a1 = (int)(q / e0);
    const long long base = (long long)(a0 + nh) * s0 + (long long)(a1 + (axis == 2 ? nh : k0)) * s1;
    auto at = [&](int p) { return base + (long long)p * sa; };
    if (rule == GR_NEUMANN) {
      if (lo) u[at(dlo - 1)] = u[at(dlo)];
      else u[at(dhi + 1)] = u[at(dhi)];
    } else if (rule == GR_DIRICHLET) {
      if (g.nd == 2) {  // every halo layer (:137-155)
        if (lo)
          for (int p = 0; p < dlo; ++p) u[at(p)] = g.val[side];
        else
          for (int p = dhi + 1; p < nfull; ++p) u[at(p)] = g.val[side];
      } else {  // one layer (:178-200)
        u[at(lo ? dlo - 1 : dhi + 1)] = g.val[side];
      }
    } else if (rule == GR_PERIODIC) {
      if (lo) u[at(dlo - 1)] = u[at(dhi)];
      else u[at(dhi + 1)] = u[at(dlo)];
    } else if (rule == GR_NEGSYM) {
      if (lo) u[at(dlo - 1)] = -u[at(dlo)];
      else u[at(dhi + 1)] = -u[at(dhi)];
    }
  }
}

// update_conductivity! with scalar cp (conductivity.jl:93-104) over the
// diffusion region; flags a non-finite diffusivity on the domain and its first
// halo layer without edges and corners (validate_scalar, validity_checks.jl:1-43)
__global__ void diffusivity_kernel(Geo g, const double* __restrict__ T, const double* __restrict__ rho,
                                   double cp, double k0, int kmode, int km, int khalf, double kn,
                                   double* __restrict__ alpha, int* bad) {
  const int N = (int)g.N;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    int i2, j2, k2;
    row_pos(g, r, i2, j2, k2);
    const long long m = mesh_index(g, i2, j2, k2);
    const double t = T[m];
    const double kap = isfinite(t) ? k0 * pow_model(fabs(t), kmode, km, khalf, kn) : 0.0;
    const double a = fabs(kap / (rho[m] * cp));
    alpha[r] = a;
    if (on_boundary(g, i2, j2, k2) < 2 && !isfinite(a)) atomicOr(bad, 1);
  }
}

__device__ __forceinline__ double face_mean_ref(int mean, double a, double b) {
  return mean == 0 ? (2.0 * a * b) / (a + b) : (a + b) / 2.0;  // averaging.jl:7-8
}

struct EdgeMetrics {
  const double* J[3];       // edge_metrics.{i+1/2, j+1/2, k+1/2}.J
  const double* hat[3][9];  // {ξ̂, η̂, ζ̂}.{x₁, x₂, x₃} of each face family, [3a + c]
};

// bc_operator (inner_operators.jl:188-236): ilo, ihi, jlo, jhi, klo, khi in that order
__device__ __forceinline__ double bc_rhs(const Geo& g, int i2, int j2, int k2) {
  const int side = i2 == 0 ? 0 : i2 == g.n1 - 1 ? 1 : j2 == 0 ? 2 : j2 == g.n2 - 1 ? 3 : k2 == 0 ? 4 : 5;
  return g.kind[side] == CDM_BC_DIRICHLET ? g.val[side] : 0.0;
}

// _assembly_kernel_2d (inner_operators.jl:62-105): interior rows get the
// stencil of stencils.jl:14-40 built from conservative_edge_terms
// (edge_terms.jl:31-87); every row gets its right-hand side and the inverse of
// its diagonal (the Jacobi preconditioner)
__global__ void assemble_kernel(Geo g, int mean, double dt, const double* __restrict__ alpha,
                                const double* __restrict__ T, const double* __restrict__ S,
                                const double* __restrict__ cellJ, EdgeMetrics em, double* __restrict__ A,
                                double* __restrict__ b, double* __restrict__ dinv) {
  const long long N = g.N;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < (int)N; r += gridDim.x * blockDim.x) {
    int i2, j2, k2;
    row_pos(g, r, i2, j2, k2);
    if (on_boundary(g, i2, j2, k2)) {
      b[r] = bc_rhs(g, i2, j2, k2);
      dinv[r] = 1.0;
      continue;
    }
    const long long m = mesh_index(g, i2, j2, k2);
    const long long mi = m - 1, mj = m - g.nx;  // cells whose +1/2 faces are this cell's -1/2 faces
    const double ac = alpha[r];
    const double a_ip = face_mean_ref(mean, ac, alpha[r + 1]);
    const double a_im = face_mean_ref(mean, ac, alpha[r - 1]);
    const double a_jp = face_mean_ref(mean, ac, alpha[r + g.n1]);
    const double a_jm = face_mean_ref(mean, ac, alpha[r - g.n1]);
    const double Jip = em.J[0][m], Jim = em.J[0][mi], Jjp = em.J[1][m], Jjm = em.J[1][mj];
    // ξ̂.x₁ = [0], ξ̂.x₂ = [1], η̂.x₁ = [3], η̂.x₂ = [4]
    double xx = em.hat[0][0][m], xy = em.hat[0][1][m], ex = em.hat[0][3][m], ey = em.hat[0][4][m];
    const double a_xi2_ip = a_ip * (xx * xx + xy * xy) / Jip;
    const double a_xieta_ip = a_ip * (xx * ex + xy * ey) / (4.0 * Jip);
    xx = em.hat[0][0][mi], xy = em.hat[0][1][mi], ex = em.hat[0][3][mi], ey = em.hat[0][4][mi];
    const double a_xi2_im = a_im * (xx * xx + xy * xy) / Jim;
    const double a_xieta_im = a_im * (xx * ex + xy * ey) / (4.0 * Jim);
    xx = em.hat[1][0][m], xy = em.hat[1][1][m], ex = em.hat[1][3][m], ey = em.hat[1][4][m];
    const double a_eta2_jp = a_jp * (ex * ex + ey * ey) / Jjp;
    const double a_etaxi_jp = a_jp * (xx * ex + xy * ey) / (4.0 * Jjp);
    xx = em.hat[1][0][mj], xy = em.hat[1][1][mj], ex = em.hat[1][3][mj], ey = em.hat[1][4][mj];
    const double a_eta2_jm = a_jm * (ex * ex + ey * ey) / Jjm;
    const double a_etaxi_jm = a_jm * (xx * ex + xy * ey) / (4.0 * Jjm);
    const double Jc = cellJ[m];
    const double diag = Jc + (a_eta2_jp + a_eta2_jm + a_xi2_ip + a_xi2_im) * dt;
    A[0 * N + r] = (-a_etaxi_jm - a_xieta_im) * dt;              // i-1, j-1
    A[1 * N + r] = (-a_eta2_jm + a_xieta_ip - a_xieta_im) * dt;  // i,   j-1
    A[2 * N + r] = (a_etaxi_jm + a_xieta_ip) * dt;               // i+1, j-1
    A[3 * N + r] = (a_etaxi_jp - a_etaxi_jm - a_xi2_im) * dt;    // i-1, j
    A[4 * N + r] = diag;                                         // i,   j
    A[5 * N + r] = (-a_etaxi_jp + a_etaxi_jm - a_xi2_ip) * dt;   // i+1, j
    A[6 * N + r] = (a_etaxi_jp + a_xieta_im) * dt;               // i-1, j+1
    A[7 * N + r] = (-a_eta2_jp - a_xieta_ip + a_xieta_im) * dt;  // i,   j+1
    A[8 * N + r] = (-a_etaxi_jp - a_xieta_ip) * dt;              // i+1, j+1
    b[r] = (S[r] * dt + T[m]) * Jc;
    dinv[r] = 1.0 / diag;
  }
}

// the 18 conservative edge terms of one face (edge_terms.jl:235-257): the
// face's J and J-scaled metric vectors ξ̂, η̂, ζ̂ at full index m of family f
struct Face3 {
  double J, v[3][3];
};
__device__ __forceinline__ Face3 face3(const EdgeMetrics& em, int f, long long m) {
  Face3 F;
  F.J = em.J[f][m];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) F.v[a][c] = em.hat[f][3 * a + c][m];
  return F;
}
__device__ __forceinline__ double dot3(const double* u, const double* v) {
  return u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
}

// _assembly_kernel_3d (inner_operators.jl:107-160): the 19 non-zero entries of
// stencils.jl:42-137 (the eight corner entries are zero), stored in slot order
__global__ void assemble_kernel3(Geo g, int mean, double dt, const double* __restrict__ alpha,
                                 const double* __restrict__ T, const double* __restrict__ S,
                                 const double* __restrict__ cellJ, EdgeMetrics em, double* __restrict__ A,
                                 double* __restrict__ b, double* __restrict__ dinv) {
  const long long N = g.N;
  const int n1 = g.n1, n12 = g.n1 * g.n2;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < (int)N; r += gridDim.x * blockDim.x) {
    int i2, j2, k2;
    row_pos(g, r, i2, j2, k2);
    if (on_boundary(g, i2, j2, k2)) {
      b[r] = bc_rhs(g, i2, j2, k2);
      dinv[r] = 1.0;
      continue;
    }
    const long long m = mesh_index(g, i2, j2, k2);
    const long long sxy = (long long)g.nx * g.ny;
    const double ac = alpha[r];
    const double a_ip = face_mean_ref(mean, ac, alpha[r + 1]);
    const double a_im = face_mean_ref(mean, ac, alpha[r - 1]);
    const double a_jp = face_mean_ref(mean, ac, alpha[r + n1]);
    const double a_jm = face_mean_ref(mean, ac, alpha[r - n1]);
    const double a_kp = face_mean_ref(mean, ac, alpha[r + n12]);
    const double a_km = face_mean_ref(mean, ac, alpha[r - n12]);
    double xi2_ip, xieta_ip, xizeta_ip, xi2_im, xieta_im, xizeta_im;
    double eta2_jp, etaxi_jp, etazeta_jp, eta2_jm, etaxi_jm, etazeta_jm;
    double zeta2_kp, zetaxi_kp, zetaeta_kp, zeta2_km, zetaxi_km, zetaeta_km;
    {
      Face3 F = face3(em, 0, m);
      xi2_ip = a_ip * dot3(F.v[0], F.v[0]) / F.J;
      xieta_ip = a_ip * dot3(F.v[0], F.v[1]) / (4.0 * F.J);
      xizeta_ip = a_ip * dot3(F.v[0], F.v[2]) / (4.0 * F.J);
      F = face3(em, 0, m - 1);
      xi2_im = a_im * dot3(F.v[0], F.v[0]) / F.J;
      xieta_im = a_im * dot3(F.v[0], F.v[1]) / (4.0 * F.J);
      xizeta_im = a_im * dot3(F.v[0], F.v[2]) / (4.0 * F.J);
      F = face3(em, 1, m);
      eta2_jp = a_jp * dot3(F.v[1], F.v[1]) / F.J;
      etaxi_jp = a_jp * dot3(F.v[0], F.v[1]) / (4.0 * F.J);
      etazeta_jp = a_jp * dot3(F.v[1], F.v[2]) / (4.0 * F.J);
      F = face3(em, 1, m - g.nx);
      eta2_jm = a_jm * dot3(F.v[1], F.v[1]) / F.J;
      etaxi_jm = a_jm * dot3(F.v[0], F.v[1]) / (4.0 * F.J);
      etazeta_jm = a_jm * dot3(F.v[1], F.v[2]) / (4.0 * F.J);
      F = face3(em, 2, m);
      zeta2_kp = a_kp * dot3(F.v[2], F.v[2]) / F.J;
      zetaxi_kp = a_kp * dot3(F.v[2], F.v[0]) / (4.0 * F.J);
      zetaeta_kp = a_kp * dot3(F.v[2], F.v[1]) / (4.0 * F.J);
      F = face3(em, 2, m - sxy);
      zeta2_km = a_km * dot3(F.v[2], F.v[2]) / F.J;
      zetaxi_km = a_km * dot3(F.v[2], F.v[0]) / (4.0 * F.J);
      zetaeta_km = a_km * dot3(F.v[2], F.v[1]) / (4.0 * F.J);
    }
    const double Jc = cellJ[m];
    const double diag = Jc + (zeta2_kp + zeta2_km + eta2_jp + eta2_jm + xi2_ip + xi2_im) * dt;
    // compact entries, slot order (slots 1 3 4 5 7 9 10 11 12 13 14 15 16 17 19 21 22 23 25)
    A[0 * N + r] = (-zetaeta_km - etazeta_jm) * dt;                                  // (0,-1,-1)
    A[1 * N + r] = (-zetaxi_km - xizeta_im) * dt;                                    // (-1,0,-1)
    A[2 * N + r] = (-zeta2_km + xizeta_ip - xizeta_im + etazeta_jp - etazeta_jm) * dt;  // (0,0,-1)
    A[3 * N + r] = (zetaxi_km + xizeta_ip) * dt;                                     // (1,0,-1)
    A[4 * N + r] = (zetaeta_km + etazeta_jp) * dt;                                   // (0,1,-1)
    A[5 * N + r] = (-etaxi_jm - xieta_im) * dt;                                      // (-1,-1,0)
    A[6 * N + r] = (-eta2_jm + xieta_ip - xieta_im + zetaeta_kp - zetaeta_km) * dt;  // (0,-1,0)
    A[7 * N + r] = (etaxi_jm + xieta_ip) * dt;                                       // (1,-1,0)
    A[8 * N + r] = (-xi2_im + etaxi_jp - etaxi_jm + zetaxi_kp - zetaxi_km) * dt;     // (-1,0,0)
    A[9 * N + r] = diag;                                                             // (0,0,0)
    A[10 * N + r] = (-xi2_ip - etaxi_jp + etaxi_jm - zetaxi_kp + zetaxi_km) * dt;    // (1,0,0)
    A[11 * N + r] = (etaxi_jp + xieta_im) * dt;                                      // (-1,1,0)
    A[12 * N + r] = (-eta2_jp - xieta_ip + xieta_im - zetaeta_kp + zetaeta_km) * dt; // (0,1,0)
    A[13 * N + r] = (-etaxi_jp - xieta_ip) * dt;                                     // (1,1,0)
    A[14 * N + r] = (zetaeta_kp + etazeta_jm) * dt;                                  // (0,-1,1)
    A[15 * N + r] = (zetaxi_kp + xizeta_im) * dt;                                    // (-1,0,1)
    A[16 * N + r] = (-zeta2_kp - xizeta_ip + xizeta_im - etazeta_jp + etazeta_jm) * dt;  // (0,0,1)
    A[17 * N + r] = (-zetaxi_kp - xizeta_ip) * dt;                                   // (1,0,1)
    A[18 * N + r] = (-zetaeta_kp - etazeta_jp) * dt;                                 // (0,1,1)
    b[r] = (S[r] * dt + T[m]) * Jc;
    dinv[r] = 1.0 / diag;
  }
}

// ------------------------------------------------------------- BiCGSTAB
struct Vecs {
  double *x, *r, *rh, *p, *ph, *v, *s, *sh, *t, *b, *dinv, *part;
  const double* A;
  KState* ks;
};

// The iteration kernels keep several rows' loads in flight per thread: rows
// r0 + k·stride (k < U; the products with A two rows in 2D, one in 3D) are
// loaded first, then combined and stored, with 32-bit row arithmetic (the
// diffusion region has fewer than 2^31 rows).
constexpr int U = 4;  // rows per thread and loop trip, streaming kernels

// one row's product with A: the stored entries of an interior row (9 in 2D,
// the 19 non-corner entries in 3D, slot order), or its constraint row
template <int ND>
struct RowProd {
  static constexpr int NE = ND == 2 ? 9 : 19;
  static constexpr int CENTER = ND == 2 ? 4 : 9;
  double a[NE], x[NE];
  bool inner;
  long long c;
};

template <int ND>
__device__ __forceinline__ void load_row(const Geo& g, const double* __restrict__ A, const double* x, int r,
                                         RowProd<ND>& q) {
  int i2, j2, k2;
  row_pos(g, r, i2, j2, k2);
  q.inner = on_boundary(g, i2, j2, k2) == 0;
  if (q.inner) {
    const long long N = g.N;
    const int n1 = g.n1, n12 = g.n1 * g.n2;
    int e = 0;
#pragma unroll
    for (int dk = (ND == 3 ? -1 : 0); dk <= (ND == 3 ? 1 : 0); ++dk)
#pragma unroll
      for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
        for (int di = -1; di <= 1; ++di) {
          if (ND == 3 && di != 0 && dj != 0 && dk != 0) continue;  // corner entries are zero
          q.a[e] = __ldg(&A[e * N + r]);
          q.x[e] = x[r + di + dj * n1 + dk * n12];
          ++e;
        }
  } else {
    q.c = partner(g, i2, j2, k2, r);
    q.x[RowProd<ND>::CENTER] = x[r];
    q.x[0] = q.c >= 0 ? x[q.c] : 0.0;
  }
}

template <int ND>
__device__ __forceinline__ double row_value(const RowProd<ND>& q) {
  constexpr int C = RowProd<ND>::CENTER;
  if (!q.inner) return q.c >= 0 ? q.x[C] - q.x[0] : q.x[C];
  double y = q.a[C] * q.x[C];
#pragma unroll
  for (int e = 0; e < RowProd<ND>::NE; ++e)
    if (e != C) y = fma(q.a[e], q.x[e], y);
  return y;
}

// r = b - A x; r̂ = r; p = v = 0 and the scalars of a fresh Krylov cycle.
// first = 1: also ||r0||, the stopping tolerance and the iteration count;
// otherwise (restart or the final check) done = (||r|| <= tol)
template <int ND>
__global__ void __launch_bounds__(NT) k_restart(Geo g, Vecs V, int first, double atol, double rtol, int max_iter) {
  __shared__ double s_red[2 * NT / 32];
  __shared__ int s_last;
  double acc[1] = {0.0};
  const int N = (int)g.N;
  for (int r = blockIdx.x * NT + threadIdx.x; r < N; r += gridDim.x * NT) {
    RowProd<ND> q;
    load_row<ND>(g, V.A, V.x, r, q);
    const double rr = V.b[r] - row_value(q);
    V.r[r] = rr;
    V.rh[r] = rr;
    V.p[r] = 0.0;
    V.v[r] = 0.0;
    acc[0] = fma(rr, rr, acc[0]);
  }
  double out[1];
  if (!grid_sum<1>(acc, V.part, &V.ks->arrive[0], s_red, &s_last, out)) return;
  if (threadIdx.x != 0) return;
  KState* K = V.ks;
  const double nrm = sqrt(out[0]);
  K->rho0 = K->alpha = K->omega = 1.0;
  K->rho1 = out[0];
  K->rr = nrm;
  if (first) {
    K->r0n = nrm;
    K->tol = atol + rtol * nrm;
    K->iter = 0;
    K->max_iter = max_iter;
    K->status = KS_OK;
  }
  if (!isfinite(nrm)) {
    K->status = KS_NONFINITE;
    K->done = 1;
    K->conv = CONV_NO;
  } else {
    K->done = nrm <= K->tol ? 1 : 0;
    K->conv = K->done ? CONV_TOL : CONV_NO;
  }
}

// p = r + β(p − ω v), p̂ = D⁻¹ p
__global__ void __launch_bounds__(NT) k_p(Geo g, Vecs V) {
  const KState* K = V.ks;
  if (K->done) return;
  const double beta = (K->rho1 / K->rho0) * (K->alpha / K->omega), om = K->omega;
  const int N = (int)g.N, stride = gridDim.x * NT;
  const double* __restrict__ R = V.r;
  const double* __restrict__ D = V.dinv;
  const double* __restrict__ Vv = V.v;
  double* __restrict__ P = V.p;
  double* __restrict__ Ph = V.ph;
  for (int r0 = blockIdx.x * NT + threadIdx.x; r0 < N; r0 += U * stride) {
    double rr[U], pp[U], vv[U], dd[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        rr[k] = R[r];
        pp[k] = P[r];
        vv[k] = Vv[r];
        dd[k] = __ldg(&D[r]);
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        const double p = rr[k] + beta * (pp[k] - om * vv[k]);
        P[r] = p;
        Ph[r] = dd[k] * p;
      }
    }
  }
}

// v = A p̂; α = ρ / (r̂ · v)
template <int ND>
__global__ void __launch_bounds__(NT) k_v(Geo g, Vecs V) {
  constexpr int US = ND == 2 ? 2 : 1;  // rows in flight per thread (9 or 19 loads each)
  __shared__ double s_red[2 * NT / 32];
  __shared__ int s_last;
  KState* K = V.ks;
  if (K->done) return;
  double acc[1] = {0.0};
  const int N = (int)g.N, stride = gridDim.x * NT;
  for (int r0 = blockIdx.x * NT + threadIdx.x; r0 < N; r0 += US * stride) {
    RowProd<ND> q[US];
    double h[US];
#pragma unroll
    for (int k = 0; k < US; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        load_row<ND>(g, V.A, V.ph, r, q[k]);
        h[k] = V.rh[r];
      }
    }
#pragma unroll
    for (int k = 0; k < US; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        const double v = row_value(q[k]);
        V.v[r] = v;
        acc[0] = fma(h[k], v, acc[0]);
      }
    }
  }
  double out[1];
  if (!grid_sum<1>(acc, V.part, &K->arrive[1], s_red, &s_last, out)) return;
  if (threadIdx.x != 0) return;
  K->rv = out[0];
  if (out[0] == 0.0 || !isfinite(out[0])) {
    K->done = 1;  // breakdown: the host restarts from the true residual
    K->conv = CONV_BREAKDOWN;
  } else {
    K->alpha = K->rho1 / out[0];
  }
}

// s = r − α v, ŝ = D⁻¹ s
__global__ void __launch_bounds__(NT) k_s(Geo g, Vecs V) {
  const KState* K = V.ks;
  if (K->done) return;
  const double al = K->alpha;
  const int N = (int)g.N, stride = gridDim.x * NT;
  const double* __restrict__ R = V.r;
  const double* __restrict__ Vv = V.v;
  const double* __restrict__ D = V.dinv;
  double* __restrict__ S = V.s;
  double* __restrict__ Sh = V.sh;
  for (int r0 = blockIdx.x * NT + threadIdx.x; r0 < N; r0 += U * stride) {
    double rr[U], vv[U], dd[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        rr[k] = R[r];
        vv[k] = Vv[r];
        dd[k] = __ldg(&D[r]);
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        const double sv = rr[k] - al * vv[k];
        S[r] = sv;
        Sh[r] = dd[k] * sv;
      }
    }
  }
}

// t = A ŝ; ω = (t · s) / (t · t)
template <int ND>
__global__ void __launch_bounds__(NT) k_t(Geo g, Vecs V) {
  constexpr int US = ND == 2 ? 2 : 1;
  __shared__ double s_red[2 * NT / 32];
  __shared__ int s_last;
  KState* K = V.ks;
  if (K->done) return;
  double acc[2] = {0.0, 0.0};
  const int N = (int)g.N, stride = gridDim.x * NT;
  for (int r0 = blockIdx.x * NT + threadIdx.x; r0 < N; r0 += US * stride) {
    RowProd<ND> q[US];
    double sv[US];
#pragma unroll
    for (int k = 0; k < US; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        load_row<ND>(g, V.A, V.sh, r, q[k]);
        sv[k] = V.s[r];
      }
    }
#pragma unroll
    for (int k = 0; k < US; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        const double t = row_value(q[k]);
        V.t[r] = t;
        acc[0] = fma(t, sv[k], acc[0]);
        acc[1] = fma(t, t, acc[1]);
      }
    }
  }
  double out[2];
  if (!grid_sum<2>(acc, V.part, &K->arrive[2], s_red, &s_last, out)) return;
  if (threadIdx.x != 0) return;
  K->ts = out[0];
  K->tt = out[1];
  K->omega = out[1] > 0.0 ? out[0] / out[1] : 0.0;
}

// x += α p̂ + ω ŝ; r = s − ω t; the next ρ = r̂ · r and the stopping rule
__global__ void __launch_bounds__(NT) k_x(Geo g, Vecs V) {
  __shared__ double s_red[2 * NT / 32];
  __shared__ int s_last;
  KState* K = V.ks;
  if (K->done) return;
  const double al = K->alpha, om = K->omega;
  double acc[2] = {0.0, 0.0};
  const int N = (int)g.N, stride = gridDim.x * NT;
  double* __restrict__ X = V.x;
  double* __restrict__ R = V.r;
  const double* __restrict__ Ph = V.ph;
  const double* __restrict__ Sh = V.sh;
  const double* __restrict__ S = V.s;
  const double* __restrict__ T = V.t;
  const double* __restrict__ Rh = V.rh;
  for (int r0 = blockIdx.x * NT + threadIdx.x; r0 < N; r0 += U * stride) {
    double xx[U], ph[U], sh[U], ss[U], tt[U], rh[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        xx[k] = X[r];
        ph[k] = Ph[r];
        sh[k] = Sh[r];
        ss[k] = S[r];
        tt[k] = T[r];
        rh[k] = Rh[r];
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        X[r] = xx[k] + al * ph[k] + om * sh[k];
        const double rr = ss[k] - om * tt[k];
        R[r] = rr;
        acc[0] = fma(rh[k], rr, acc[0]);
        acc[1] = fma(rr, rr, acc[1]);
      }
    }
  }
  double out[2];
  if (!grid_sum<2>(acc, V.part, &K->arrive[3], s_red, &s_last, out)) return;
  if (threadIdx.x != 0) return;
  K->iter += 1;
  const double nrm = sqrt(out[1]);
  K->rr = nrm;
  K->rho0 = K->rho1;
  K->rho1 = out[0];
  if (!isfinite(nrm)) {
    K->status = KS_NONFINITE;
    K->done = 1;
  } else if (nrm <= K->tol) {
    K->done = 1;
    K->conv = CONV_TOL;
  } else if (K->iter >= K->max_iter) {
    K->status = KS_MAX_ITER;
    K->done = 1;
  } else if (out[0] == 0.0 || om == 0.0) {
    K->done = 1;  // breakdown: restart from the true residual
    K->conv = CONV_BREAKDOWN;
  }
}

// ------------------------------------------------ after the solve (solve!)
// cutoff (ImplictSolver.jl:384), then the first next_dt reduction: max(uⁿ)
// over the diffusion region (NaN propagates, as Julia's maximum)
__global__ void __launch_bounds__(NT) k_post1(Geo g, double* x, const double* __restrict__ T, int cutoff,
                                              double* part, KState* K) {
  __shared__ double s_red[NT / 32];
  __shared__ int s_last, s_nan;
  if (threadIdx.x == 0) s_nan = 0;
  __syncthreads();
  double m = -INFINITY;
  bool nan = false;
  for (long long r = blockIdx.x * (long long)NT + threadIdx.x; r < g.N; r += (long long)gridDim.x * NT) {
    if (cutoff) {  // (0.5(|a| + a)) * isfinite(a); Julia's false is a strong zero
      const double a = x[r];
      x[r] = isfinite(a) ? 0.5 * (fabs(a) + a) : 0.0;
    }
    int i2, j2, k2;
    row_pos(g, (int)r, i2, j2, k2);
    const double u = T[mesh_index(g, i2, j2, k2)];
    if (u != u) nan = true;
    m = fmax(m, u);
  }
  if (nan) atomicOr(&s_nan, 1);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) s_red[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NT / 32; ++w) m = fmax(m, s_red[w]);
    part[blockIdx.x] = s_nan ? NAN : m;
    __threadfence();
    s_last = atomicAdd(&K->arrive[0], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double all = -INFINITY;
  bool anynan = false;
  for (unsigned b = 0; b < gridDim.x; ++b) {
    const double w = ((volatile double*)part)[b];
    if (w != w) anynan = true;
    all = fmax(all, w);
  }
  K->umax = anynan ? NAN : all;
  K->arrive[0] = 0u;
}

// max relative change (timestep_control.jl:64-71, GPU form) and the copy of
// the solution into T's diffusion region
__global__ void __launch_bounds__(NT) k_post2(Geo g, const double* __restrict__ x, double* T, double ndt_tol,
                                              double* part, KState* K) {
  __shared__ double s_red[NT / 32];
  __shared__ int s_last;
  const double u0 = K->umax * ndt_tol;
  double m = -INFINITY;
  for (long long r = blockIdx.x * (long long)NT + threadIdx.x; r < g.N; r += (long long)gridDim.x * NT) {
    int i2, j2, k2;
    row_pos(g, (int)r, i2, j2, k2);
    const long long mi = mesh_index(g, i2, j2, k2);
    const double a = x[r], b = T[mi];
    const double d = fabs(a - b) / (a + u0);
    m = fmax(m, isfinite(d) ? d : 0.0);  // δ * isfinite(δ), false a strong zero
    T[mi] = a;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) s_red[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < NT / 32; ++w) m = fmax(m, s_red[w]);
    part[blockIdx.x] = m;
    __threadfence();
    s_last = atomicAdd(&K->arrive[1], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double all = -INFINITY;
  for (unsigned b = 0; b < gridDim.x; ++b) all = fmax(all, ((volatile double*)part)[b]);
  K->maxrel = all;
  K->arrive[1] = 0u;
}

}  // namespace imp

// ------------------------------------------------------------------ handle
struct Implicit {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int mean = 0;
  imp::Geo g{};
  int64_t nfull = 0;
  // device arrays: mesh inputs (full mesh layout)
  double* cellJ = nullptr;
  double* edgeJ[3] = {nullptr, nullptr, nullptr};  // face J per family
  double* edgehat[3][9] = {{nullptr}};              // J-scaled face metrics [3a + c] (2D: those read)
  int nent = 9;                                     // stored stencil entries per row (3D: 19)
  double* T = nullptr;               // full mesh layout work copies
  double* rho = nullptr;
  // diffusion region
  double *A = nullptr, *alpha = nullptr, *S = nullptr;
  double *x = nullptr, *r = nullptr, *rh = nullptr, *p = nullptr, *ph = nullptr, *v = nullptr, *s = nullptr,
         *sh = nullptr, *t = nullptr, *b = nullptr, *dinv = nullptr, *part = nullptr;
  imp::KState* ks = nullptr;
  imp::KState* h_ks = nullptr;  // pinned
  int* d_bad = nullptr;
  int* h_bad = nullptr;
  int grid = 1;
  bool warmed_up = false;
  cudaEvent_t ev = nullptr, ev_caller = nullptr;
  double last_solve_ms = 0.0;
  int64_t last_spmv = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaGraphExec_t iters_graph = nullptr;  // kPollIters BiCGSTAB iterations
  ~Implicit();
};

namespace {

template <typename T>
cudaError_t zalloc(T** p, size_t n) {
  *p = nullptr;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) return e;
  return cudaMemset(*p, 0, n * sizeof(T));
}

int wait_event(cudaEvent_t ev, double timeout_s) {
  const auto t0 = std::chrono::steady_clock::now();
  int spins = 0;
  while (true) {
    const cudaError_t e = cudaEventQuery(ev);
    if (e == cudaSuccess) return CDM_OK;
    if (e != cudaErrorNotReady) {
      set_error(std::string("device error: ") + cudaGetErrorString(e));
      return CDM_CUDA_ERROR;
    }
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > timeout_s) {
      set_error("timed out waiting for the device");
      return CDM_TIMEOUT;
    }
    if (++spins > 64) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

cudaError_t stage(double* dst, const double* src, int64_t n, int mem, cudaStream_t s) {
  return cudaMemcpyAsync(dst, src, n * sizeof(double), mem == CDM_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                                             : cudaMemcpyHostToDevice, s);
}

}  // namespace

Implicit::~Implicit() {
  if (device >= 0) cudaSetDevice(device);
  if (stream) cudaStreamSynchronize(stream);
  double* bufs[] = {cellJ, T, rho, A, alpha, S, x, r, rh, p, ph, v, s, sh, t, b, dinv, part};
  for (double* q : bufs)
    if (q) cudaFree(q);
  for (double* q : edgeJ)
    if (q) cudaFree(q);
  for (auto& f : edgehat)
    for (double* q : f)
      if (q) cudaFree(q);
  if (ks) cudaFree(ks);
  if (d_bad) cudaFree(d_bad);
  if (h_ks) cudaFreeHost(h_ks);
  if (h_bad) cudaFreeHost(h_bad);
  if (ev) cudaEventDestroy(ev);
  if (ev_caller) cudaEventDestroy(ev_caller);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (iters_graph) cudaGraphExecDestroy(iters_graph);
  if (own_stream && stream) cudaStreamDestroy(stream);
}

}  // namespace cdm

struct cdm_implicit {
  cdm::Implicit s;
};

using cdm::set_error;

extern "C" void cdm_implicit_opts_default(cdm_implicit_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->atol = 1e-9;  // ImplictSolver.jl:256-257
  o->rtol = 1e-9;
  o->max_iter = 0;  // 0: 2 x the number of rows, Krylov.jl's default itmax
  o->enforce_positivity = 1;  // nonlinear_thermal_conduction.jl:13
  o->apply_density_bc = 1;    // :15
  o->ndt_tol = 1e-3;          // timestep_control.jl:39-41
  o->maximum_u_change = 0.05;
  o->timestep_growth_factor = 1.1;
  o->mem = CDM_MEM_HOST;
}

namespace cdm {
namespace {

int implicit_init(Implicit& s, const cdm_mesh_desc* mesh, const cdm_bc* bcs, const cdm_apt_config& c) {
  s.device = c.device;
  s.mean = c.mean;
  CDM_CK(cudaSetDevice(s.device));
  if (c.stream) {
    s.stream = (cudaStream_t)c.stream;
  } else {
    CDM_CK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
    s.own_stream = true;
  }
  imp::Geo& g = s.g;
  const int nd = mesh->ndim;
  g.nd = nd;
  g.ni = mesh->ni;
  g.nj = mesh->nj;
  g.nk = nd == 3 ? mesh->nk : 1;
  g.nh = mesh->nhalo;
  g.nx = mesh->ni + 2 * mesh->nhalo;
  g.ny = mesh->nj + 2 * mesh->nhalo;
  g.n1 = mesh->ni + 2;
  g.n2 = mesh->nj + 2;
  g.n3 = nd == 3 ? mesh->nk + 2 : 1;
  g.N = (long long)g.n1 * g.n2 * g.n3;
  double gval[6] = {0, 0, 0, 0, 0, 0};
  int grule[6] = {0, 0, 0, 0, 0, 0};
  if (resolve_ghost_rules(nd, bcs, grule, gval) != CDM_OK) {
    set_error("invalid boundary condition kind");
    return CDM_BAD_INPUT;
  }
  for (int l = 0; l < 2 * nd; ++l) {
    g.kind[l] = bcs[l].kind;
    g.rule[l] = grule[l];
    g.val[l] = bcs[l].kind == CDM_BC_DIRICHLET ? bcs[l].value : 0.0;
  }
  s.nent = nd == 3 ? 19 : 9;
  s.nfull = (int64_t)g.nx * g.ny * (nd == 3 ? mesh->nk + 2 * mesh->nhalo : 1);
  const size_t nf = (size_t)s.nfull, N = (size_t)g.N;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s.device);
  const long long need = (g.N + imp::NT - 1) / imp::NT;
  s.grid = (int)std::min<long long>(need, (long long)nsm * 8);
  const cudaMemcpyKind kind = mesh->mem == CDM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  CDM_CK(zalloc(&s.cellJ, nf));
  CDM_CK(cudaMemcpy(s.cellJ, mesh->cell_J, nf * sizeof(double), kind));
  for (int f = 0; f < nd; ++f) {
    CDM_CK(zalloc(&s.edgeJ[f], nf));
    CDM_CK(cudaMemcpy(s.edgeJ[f], mesh->edge_J[f], nf * sizeof(double), kind));
    for (int a = 0; a < nd; ++a)
      for (int c = 0; c < nd; ++c) {
        CDM_CK(zalloc(&s.edgehat[f][3 * a + c], nf));
        CDM_CK(cudaMemcpy(s.edgehat[f][3 * a + c], mesh->edge_hat[f][3 * a + c], nf * sizeof(double), kind));
      }
  }
  CDM_CK(zalloc(&s.T, nf));
  CDM_CK(zalloc(&s.rho, nf));
  CDM_CK(zalloc(&s.A, (size_t)s.nent * N));
  double** vecs[] = {&s.alpha, &s.S, &s.x, &s.r, &s.rh, &s.p, &s.ph, &s.v, &s.s, &s.sh, &s.t, &s.b, &s.dinv};
  for (double** q : vecs) CDM_CK(zalloc(q, N));
  CDM_CK(zalloc(&s.part, (size_t)2 * s.grid));
  CDM_CK(zalloc(&s.ks, (size_t)1));
  CDM_CK(zalloc(&s.d_bad, (size_t)1));
  CDM_CK(cudaMallocHost((void**)&s.h_ks, sizeof(imp::KState)));
  CDM_CK(cudaMallocHost((void**)&s.h_bad, sizeof(int)));
  CDM_CK(cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming));
  CDM_CK(cudaEventCreateWithFlags(&s.ev_caller, cudaEventDisableTiming));
  CDM_CK(cudaEventCreate(&s.e0));
  CDM_CK(cudaEventCreate(&s.e1));
  return CDM_OK;
}

// orders a private stream after the caller's legacy-default-stream work
cudaError_t fence(Implicit& s) {
  if (!s.own_stream) return cudaSuccess;
  cudaError_t e = cudaEventRecord(s.ev_caller, cudaStreamLegacy);
  if (e != cudaSuccess) return e;
  return cudaStreamWaitEvent(s.stream, s.ev_caller, 0);
}

imp::Vecs vecs_of(Implicit& s) {
  imp::Vecs V;
  V.x = s.x;
  V.r = s.r;
  V.rh = s.rh;
  V.p = s.p;
  V.ph = s.ph;
  V.v = s.v;
  V.s = s.s;
  V.sh = s.sh;
  V.t = s.t;
  V.b = s.b;
  V.dinv = s.dinv;
  V.part = s.part;
  V.A = s.A;
  V.ks = s.ks;
  return V;
}

int read_state(Implicit& s, double timeout_s) {
  CDM_CK(cudaMemcpyAsync(s.h_ks, s.ks, sizeof(imp::KState), cudaMemcpyDeviceToHost, s.stream));
  CDM_CK(cudaEventRecord(s.ev, s.stream));
  return wait_event(s.ev, timeout_s);
}

double seconds_now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace cdm

extern "C" int cdm_implicit_create(const cdm_mesh_desc* mesh, const cdm_bc* bcs, const cdm_apt_config* cfg,
                                   cdm_implicit** out) {
  using namespace cdm;
  if (!mesh || !bcs || !out) {
    set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  *out = nullptr;
  const int nd = mesh->ndim;
  if (nd != 2 && nd != 3) {
    set_error("the implicit scheme takes 2D and 3D meshes");
    return CDM_BAD_INPUT;
  }
  if (mesh->ni < 1 || mesh->nj < 1 || (nd == 3 && mesh->nk < 1) || mesh->nhalo < 1) {
    set_error("mesh sizes must be >= 1 and nhalo >= 1");
    return CDM_BAD_INPUT;
  }
  if ((long long)(mesh->ni + 2) * (mesh->nj + 2) * (nd == 3 ? mesh->nk + 2 : 1) >= (1ll << 31)) {
    set_error("the implicit system takes fewer than 2^31 rows");
    return CDM_BAD_INPUT;
  }
  for (int l = 0; l < 2 * nd; ++l)
    if (bcs[l].kind == CDM_BC_NEG_SYMMETRY || bcs[l].kind < CDM_BC_NEUMANN || bcs[l].kind > CDM_BC_NEG_SYMMETRY) {
      set_error("the implicit scheme takes Neumann, Dirichlet and periodic sides (init_matrix.jl)");
      return CDM_BAD_INPUT;
    }
  // init_matrix.jl:7-12 and :184-192 (in 3D the test covers the i and j sides only)
  for (int a = 0; a < 2; ++a)
    if ((bcs[2 * a].kind == CDM_BC_PERIODIC) != (bcs[2 * a + 1].kind == CDM_BC_PERIODIC)) {
      set_error("Inconsistent periodic boundary conditions");
      return CDM_BAD_INPUT;
    }
  if (!mesh->cell_J) {
    set_error("the implicit scheme needs cell_J");
    return CDM_BAD_INPUT;
  }
  for (int f = 0; f < nd; ++f) {
    if (!mesh->edge_J[f]) {
      set_error("the implicit scheme needs the face J of every face family");
      return CDM_BAD_INPUT;
    }
    for (int a = 0; a < nd; ++a)
      for (int c = 0; c < nd; ++c)
        if (!mesh->edge_hat[f][3 * a + c]) {
          set_error("the implicit scheme needs the J-scaled face metrics of every face family");
          return CDM_BAD_INPUT;
        }
  }
  cdm_apt_config c;
  cdm_apt_config_default(&c);
  if (cfg) c = *cfg;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c.device || c.device < 0) {
    set_error("no CUDA device");
    return CDM_NO_DEVICE;
  }
  auto* h = new cdm_implicit();
  const int rc = implicit_init(h->s, mesh, bcs, c);
  if (rc != CDM_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return CDM_OK;
}

extern "C" int cdm_implicit_destroy(cdm_implicit* h) {
  delete h;
  return CDM_OK;
}

extern "C" int cdm_implicit_set_source(cdm_implicit* h, const double* S, int mem) {
  using namespace cdm;
  if (!h || !S) {
    set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  Implicit& s = h->s;
  CDM_CK(cudaSetDevice(s.device));
  // the diffusion region of a full mesh array: n1 values per row, n2 rows per plane, n3 planes
  const imp::Geo& g = s.g;
  if (mem == CDM_MEM_DEVICE) CDM_CK(fence(s));
  const int64_t plane = (int64_t)g.nx * g.ny;
  for (int k2 = 0; k2 < g.n3; ++k2) {
    const int64_t kz = g.nd == 3 ? (int64_t)(k2 - 1 + g.nh) : 0;
    const double* src = S + (g.nh - 1) + (int64_t)g.nx * (g.nh - 1) + kz * plane;
    CDM_CK(cudaMemcpy2DAsync(s.S + (int64_t)k2 * g.n1 * g.n2, (size_t)g.n1 * sizeof(double), src,
                             (size_t)g.nx * sizeof(double), (size_t)g.n1 * sizeof(double), (size_t)g.n2,
                             mem == CDM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s.stream));
  }
  CDM_CK(cudaStreamSynchronize(s.stream));
  return CDM_OK;
}

extern "C" int cdm_implicit_step(cdm_implicit* h, double* T, const double* rho, double cp, cdm_kappa kappa,
                                 double dt, const cdm_implicit_opts* opts, cdm_stats* stats, double* next_dt) {
  using namespace cdm;
  if (!h || !T || !rho || !stats || !next_dt) {
    set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  const double t_start = seconds_now();
  std::memset(stats, 0, sizeof(*stats));
  cdm_implicit_opts o;
  cdm_implicit_opts_default(&o);
  if (opts) o = *opts;
  if (!(dt > 0.0)) {
    set_error("dt must be > 0");
    return stats->status = CDM_BAD_INPUT;
  }
  double timeout_s = 3600.0;
  if (const char* e = std::getenv("CDM_STEP_TIMEOUT_S")) timeout_s = std::atof(e);
  Implicit& s = h->s;
  const imp::Geo& g = s.g;
  CDM_CK(cudaSetDevice(s.device));
  if (o.mem == CDM_MEM_DEVICE) CDM_CK(fence(s));
  // applybcs! on T and, with apply_density_bc, on rho (nonlinear_thermal_conduction.jl:19-23)
  CDM_CK(stage(s.T, T, s.nfull, o.mem, s.stream));
  CDM_CK(stage(s.rho, rho, s.nfull, o.mem, s.stream));
  const long long slab = std::max<long long>({(long long)g.nj * g.nk, (long long)g.ni * g.nk, (long long)g.ni * g.nj});
  const dim3 gg((unsigned)std::max<long long>(1, std::min<long long>(256, (slab + 255) / 256)), 2 * g.nd);
  imp::ghost_fill<<<gg, 256, 0, s.stream>>>(g, s.T);
  if (o.apply_density_bc) imp::ghost_fill<<<gg, 256, 0, s.stream>>>(g, s.rho);
  // update_conductivity! and validate_scalar (:25-33)
  int kmode = 2, km = 0, khalf = 0;
  {
    const double n = kappa.n, twice = 2.0 * n;
    if (n == 0.0) kmode = 0;
    else if (n > 0.0 && n <= 16.0 && twice == std::floor(twice)) {
      kmode = 1;
      km = (int)std::floor(n);
      khalf = (twice != 2.0 * km) ? 1 : 0;
    }
  }
  CDM_CK(cudaMemsetAsync(s.d_bad, 0, sizeof(int), s.stream));
  imp::diffusivity_kernel<<<s.grid, imp::NT, 0, s.stream>>>(g, s.T, s.rho, cp, kappa.k0, kmode, km, khalf,
                                                            kappa.n, s.alpha, s.d_bad);
  imp::EdgeMetrics em;
  for (int f = 0; f < 3; ++f) {
    em.J[f] = s.edgeJ[f];
    for (int q = 0; q < 9; ++q) em.hat[f][q] = s.edgehat[f][q];
  }
  // assemble! (matrix_assembly.jl:5-59)
  if (g.nd == 2)
    imp::assemble_kernel<<<s.grid, imp::NT, 0, s.stream>>>(g, s.mean, dt, s.alpha, s.T, s.S, s.cellJ, em, s.A,
                                                           s.b, s.dinv);
  else
    imp::assemble_kernel3<<<s.grid, imp::NT, 0, s.stream>>>(g, s.mean, dt, s.alpha, s.T, s.S, s.cellJ, em, s.A,
                                                            s.b, s.dinv);
  CDM_CK(cudaGetLastError());
  CDM_CK(cudaMemcpyAsync(s.h_bad, s.d_bad, sizeof(int), cudaMemcpyDeviceToHost, s.stream));
  CDM_CK(cudaEventRecord(s.ev, s.stream));
  int rc = wait_event(s.ev, timeout_s);
  if (rc != CDM_OK) return stats->status = rc;
  if (*s.h_bad) {
    set_error("Invalid diffusivity (non-finite) in the domain or its first halo layer");
    return stats->status = CDM_BAD_INPUT;
  }
  // Krylov solve from zero (first call) or the previous solution (ImplictSolver.jl:282-303)
  if (!s.warmed_up) CDM_CK(cudaMemsetAsync(s.x, 0, (size_t)g.N * sizeof(double), s.stream));
  const int max_iter = o.max_iter > 0 ? o.max_iter : (int)std::min<long long>(2 * g.N, 1 << 30);
  imp::Vecs V = vecs_of(s);
  CDM_CK(cudaEventRecord(s.e0, s.stream));
  auto restart = [&](int first) {
    if (g.nd == 2) imp::k_restart<2><<<s.grid, imp::NT, 0, s.stream>>>(g, V, first, o.atol, o.rtol, max_iter);
    else imp::k_restart<3><<<s.grid, imp::NT, 0, s.stream>>>(g, V, first, o.atol, o.rtol, max_iter);
  };
  restart(1);
  CDM_CK(cudaGetLastError());
  rc = read_state(s, timeout_s - (seconds_now() - t_start));
  bool fresh = true;  // r holds the true residual b - A x (just computed)
  int restarts = 0;
  while (rc == CDM_OK) {
    const imp::KState& K = *s.h_ks;
    if (K.done) {
      if (K.status != imp::KS_OK) break;
      if (fresh && K.conv == imp::CONV_TOL) break;  // the true residual meets the tolerance
      // the recursive residual met the tolerance, or a breakdown: recompute the
      // true residual and, unless it meets the tolerance, start a new cycle from it
      if (++restarts > 1000) {
        set_error("Krylov solve: repeated breakdowns");
        stats->niter = K.iter;
        return stats->status = CDM_NONFINITE;
      }
      restart(0);
      CDM_CK(cudaGetLastError());
      fresh = true;
      rc = read_state(s, timeout_s - (seconds_now() - t_start));
      continue;
    }
    if (!s.iters_graph) {  // the kernels' arguments are fixed for the handle's life
      cudaGraph_t graph;
      CDM_CK(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < imp::kPollIters; ++k) {
        imp::k_p<<<s.grid, imp::NT, 0, s.stream>>>(g, V);
        if (g.nd == 2) imp::k_v<2><<<s.grid, imp::NT, 0, s.stream>>>(g, V);
        else imp::k_v<3><<<s.grid, imp::NT, 0, s.stream>>>(g, V);
        imp::k_s<<<s.grid, imp::NT, 0, s.stream>>>(g, V);
        if (g.nd == 2) imp::k_t<2><<<s.grid, imp::NT, 0, s.stream>>>(g, V);
        else imp::k_t<3><<<s.grid, imp::NT, 0, s.stream>>>(g, V);
        imp::k_x<<<s.grid, imp::NT, 0, s.stream>>>(g, V);
      }
      const cudaError_t le = cudaGetLastError();
      const cudaError_t ce = cudaStreamEndCapture(s.stream, &graph);
      CDM_CK(le);
      CDM_CK(ce);
      const cudaError_t ie = cudaGraphInstantiate(&s.iters_graph, graph, 0);
      cudaGraphDestroy(graph);
      CDM_CK(ie);
    }
    CDM_CK(cudaGraphLaunch(s.iters_graph, s.stream));
    fresh = false;
    rc = read_state(s, timeout_s - (seconds_now() - t_start));
    if (rc == CDM_OK && seconds_now() - t_start > timeout_s) {
      set_error("step exceeded its wall-clock limit");
      rc = CDM_TIMEOUT;
    }
  }
  CDM_CK(cudaEventRecord(s.e1, s.stream));
  if (rc != CDM_OK) return stats->status = rc;
  const imp::KState K = *s.h_ks;
  stats->niter = K.iter;
  stats->abs_err = stats->rel_err = K.rr;
  stats->n_checks = 0;
  if (K.status == imp::KS_NONFINITE) {
    set_error("Krylov solve: non-finite residual");
    stats->time = seconds_now() - t_start;
    return stats->status = CDM_NONFINITE;
  }
  if (K.status == imp::KS_MAX_ITER) {
    set_error("Krylov solve: maximum iteration count reached");
    stats->time = seconds_now() - t_start;
    return stats->status = CDM_MAX_ITER;
  }
  s.warmed_up = true;
  // cutoff, next_dt, copy into T (ImplictSolver.jl:306-317)
  imp::k_post1<<<s.grid, imp::NT, 0, s.stream>>>(g, s.x, s.T, o.enforce_positivity, s.part, s.ks);
  imp::k_post2<<<s.grid, imp::NT, 0, s.stream>>>(g, s.x, s.T, o.ndt_tol, s.part, s.ks);
  CDM_CK(cudaGetLastError());
  CDM_CK(cudaMemcpyAsync(T, s.T, (size_t)s.nfull * sizeof(double),
                         o.mem == CDM_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s.stream));
  rc = read_state(s, timeout_s - (seconds_now() - t_start));
  if (rc != CDM_OK) return stats->status = rc;
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, s.e0, s.e1) == cudaSuccess) s.last_solve_ms = ms;
  s.last_spmv = 2 * (int64_t)K.iter;
  const double mr = s.h_ks->maxrel;
  const double cand = dt * std::sqrt(std::fabs(o.maximum_u_change / mr));
  *next_dt = std::min(cand, o.timestep_growth_factor * dt);
  stats->time = seconds_now() - t_start;
  stats->status = CDM_OK;
  return CDM_OK;
}

extern "C" int cdm_implicit_get_system(cdm_implicit* h, double* A, double* b) {
  using namespace cdm;
  if (!h || !A || !b) {
    set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  Implicit& s = h->s;
  CDM_CK(cudaSetDevice(s.device));
  const size_t N = (size_t)s.g.N;
  if (s.g.nd == 2) {
    CDM_CK(cudaMemcpyAsync(A, s.A, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  } else {  // the 19 stored entries into their slots of 27, the corner slots zero
    int e = 0;
    for (int slot = 0; slot < 27; ++slot) {
      const int di = slot % 3 - 1, dj = (slot / 3) % 3 - 1, dk = slot / 9 - 1;
      if (di != 0 && dj != 0 && dk != 0) {
        std::memset(A + (size_t)slot * N, 0, N * sizeof(double));
        continue;
      }
      CDM_CK(cudaMemcpyAsync(A + (size_t)slot * N, s.A + (size_t)e * N, N * sizeof(double), cudaMemcpyDeviceToHost,
                             s.stream));
      ++e;
    }
  }
  CDM_CK(cudaMemcpyAsync(b, s.b, N * sizeof(double), cudaMemcpyDeviceToHost, s.stream));
  CDM_CK(cudaStreamSynchronize(s.stream));
  return CDM_OK;
}

extern "C" int cdm_implicit_get_profile(const cdm_implicit* h, double* solve_ms, int64_t* spmv, int64_t* rows) {
  using namespace cdm;
  if (!h || !solve_ms || !spmv || !rows) {
    set_error("NULL argument");
    return CDM_BAD_INPUT;
  }
  *solve_ms = h->s.last_solve_ms;
  *spmv = h->s.last_spmv;
  *rows = (int64_t)h->s.g.N;
  return CDM_OK;
}
