// apt_mixed.cu — FP32 correction sweeps with FP64 residual and defect-correction
// restarts (2D).
//
// The pseudo-transient iteration of step! (PseudoTransientSolver.jl:253-319)
// is run in increment form around an FP64 base state u_b:
//
//   u = u_b + δ,   q = q′(u_b) + e,                       δ, e in FP32
//   e ← (e·θ̄ + Δq′)/(1 + θ̄),  Δq′ = q′(u) − q′(u_b) = −(ᾱ·Δδ + Δᾱ·Δu_b)   (fluxes.jl:5-16)
//   δ ← δ + dτΔt/(Δt + dτ)·(R_b − δ/Δt − ∇·e)                              (update.jl:13-15)
//
// with R_b = −(u_b − uⁿ)/Δt − ∇·q′(u_b) + S the FP64 residual of the base
// (residuals.jl:24-47), rounded to FP32.  Every term an FP32 sweep evaluates
// is proportional to the correction, so its rounding error is relative to the
// correction and not to u: the increments of the diffusivity use
// Δα = α_b((1 + δ/u_b)ⁿ − 1) and the exact increment of the harmonic mean,
//   H(a+Δa, b+Δb) − H(a, b) = 2(b²Δa + a²Δb + ΔaΔb(a+b)) / ((a+b)(a+b+Δa+Δb)).
// The pseudo-time parameters (θ, dτ) only set the path of the iteration and
// are computed from u in FP32.
//
// A restart folds δ into u_b in FP64, recomputes R_b and its max-norm on the
// device (the convergence check of :280-318, evaluated in FP64), and clears δ
// and e.  An inner cycle ends when the FP32 correction residual has dropped to
// a fraction of max|R_b| (FP32 resolves about 1e-6 of it) or below the
// stopping tolerance.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cdm_device.cuh"
#include "cdm_finish.cuh"
#include "engine.h"

namespace cdm {

namespace {

__device__ __forceinline__ int off2m(const Problem& P, int a, int b) { return (a + P.nh) + P.nx * (b + P.nh); }

// ghost source (offset) of cell (a, b) for the side rules; -1 constant, -2 inactive
__device__ __forceinline__ int ghost_src(const Problem& P, int a, int b, bool& cst, bool& neg, double& val) {
  cst = false;
  neg = false;
  val = 0.0;
  const bool ca = a >= 0 && a < P.ni, cb = b >= 0 && b < P.nj;
  if (ca && cb) return off2m(P, a, b);
  int side;
  if (cb && (a == -1 || a == P.ni)) side = a < 0 ? 0 : 1;
  else if (ca && (b == -1 || b == P.nj)) side = b < 0 ? 2 : 3;
  else return -2;
  const int rule = P.rule[side];
  const bool lo = (side & 1) == 0;
  const int n = side < 2 ? P.ni : P.nj;
  if (rule == GR_DIRICHLET) {
    cst = true;
    val = P.val[side];
    return -1;
  }
  const int p = rule == GR_NONE ? (lo ? -1 : n) : (rule == GR_PERIODIC ? (lo ? n - 1 : 0) : (lo ? 0 : n - 1));
  neg = rule == GR_NEGSYM;
  return side < 2 ? off2m(P, p, b) : off2m(P, a, p);
}

__device__ __forceinline__ double pow_m64(double x, int mode, int m, int half, double n) {
  if (mode == 0) return 1.0;
  if (mode == 1) {
    double p = 1.0;
    if (m >= 1) {
      p = x;
      for (int e = 1; e < m; ++e) p *= x;
    }
    if (half) p = (m >= 1) ? p * sqrt(x) : sqrt(x);
    return p;
  }
  return pow(x, n);
}

__device__ __forceinline__ float pow_m32(float x, int mode, int m, int half, float n) {
  if (mode == 0) return 1.0f;
  if (mode == 1) {
    float p = 1.0f;
    if (m >= 1) {
      p = x;
      for (int e = 1; e < m; ++e) p *= x;
    }
    if (half) p = (m >= 1) ? p * sqrtf(x) : sqrtf(x);
    return p;
  }
  return powf(x, n);
}

// max-norm reduction of a block, last block of the launch publishes the result
template <int NT>
__device__ void reduce_and_publish(const Problem& P, Ctrl* C, int tile, double local, bool nan, double* s_red,
                                   int* s_flag, bool restart) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int anynan = __syncthreads_or(nan ? 1 : 0);
  double v = local;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  if (tid == 0) {
    double r = s_red[0];
    for (int w = 1; w < NT / 32; ++w) r = fmax(r, s_red[w]);
    if (anynan) r = __longlong_as_double(0x7ff8000000000000ll);
    P.partial[tile] = r;
    __threadfence();
    const unsigned prev = atomicAdd(&C->arrive, 1u);
    *s_flag = (prev == (unsigned)P.ntiles - 1u);
  }
  __syncthreads();
  if (!*s_flag) return;
  __threadfence();
  double m = 0.0;
  bool bad = false;
  for (int t = tid; t < P.ntiles; t += NT) {
    const double w = ld_cg_double(&P.partial[t]);
    if (w != w) bad = true;
    else m = fmax(m, w);
  }
  const int anybad = __syncthreads_or(bad ? 1 : 0);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) s_red[warp] = m;
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < NT / 32; ++w) m = fmax(m, s_red[w]);
    if (anybad) m = __longlong_as_double(0x7ff8000000000000ll);
    C->arrive = 0u;
    if (restart) {
      C->restart_L2 = m;
      C->restart_nan = anybad;
    } else {
      // the cycle ends at the target, on NaN, or when FP32 stops making progress
      // (no 5% improvement of the best max|r| over 12 consecutive checks)
      C->inner_L2 = m;
      if (m < 0.95 * C->inner_best) {
        C->inner_best = m;
        C->inner_stall = 0;
      } else {
        C->inner_stall += 1;
      }
      if (!(m > C->inner_target) || anybad || C->inner_stall >= 12) C->inner_done = 1;
    }
    __threadfence();
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// FP64 restart: u = u_b + δ on the domain, ghosts by the side rules, the FP64
// residual R(u) with the undamped fluxes (residuals.jl:24-47), its max-norm,
// and the FP32 copies the sweeps read.  One block per 32x16 tile.
constexpr int RTX = 32, RTY = 16, RNT = 256;

// The damped flux of the pseudo-time iteration carries over: its total
// q′(u_b) + e is kept, so e ← e + q′(u_old) − q′(u_new) on the faces the tile
// owns.  At the first restart of a step the total is the solver's FP64 flux
// state q (carried across steps as in the reference, PseudoTransientSolver.jl:
// 32): e ← q − q′(u).  Every restart also writes the current total damped flux
// q′(u_old) + e back to the FP64 state.
struct RestartIO {
  const double* ub_in;
  const float* d_in;       // correction to fold in (NULL at the first restart)
  double* ub_out;
  float* ub32;
  float* ab32;             // diffusivity of the new base state, rounded
  float* R32;
  const float* e_in[3];    // flux correction of the last sweep (NULL at the first restart)
  const double* q_in[3];   // FP64 damped-flux state (first restart)
  float* e_out[3];
  double* q_out[3];        // FP64 damped-flux state (written at every restart)
};

__global__ void __launch_bounds__(RNT) mixed_restart2d(const Problem* __restrict__ probs, RestartIO io) {
  const double* __restrict__ ub_in = io.ub_in;
  const float* __restrict__ d_in = io.d_in;
  double* __restrict__ ub_out = io.ub_out;
  float* __restrict__ ub32 = io.ub32;
  float* __restrict__ ab32 = io.ab32;
  float* __restrict__ R32 = io.R32;
  constexpr int RX = RTX + 2, RY = RTY + 2;
  __shared__ double s_u[RY][RX], s_a[RY][RX], s_uo[RY][RX], s_ao[RY][RX];
  __shared__ double s_qx[RY][RTX + 1], s_qy[RTY + 1][RX];
  __shared__ double s_red[RNT / 32];
  __shared__ int s_flag;
  const Problem& P = probs[0];
  Ctrl* C = P.ctrl;
  const int tile = blockIdx.x;
  const int ti = tile % P.tiles_j, tj = tile / P.tiles_j;  // restart tiling: tiles_j columns of RTX
  const int i0 = ti * RTX, j0 = tj * RTY;
  const int tid = threadIdx.x;
  const int ni = P.ni, nj = P.nj;
  const double dt = P.dt;
  for (int r = tid; r < RX * RY; r += RNT) {
    const int rb = r / RX, ra = r - rb * RX;
    const int a = i0 - 1 + ra, b = j0 - 1 + rb;
    bool cst, neg;
    double val;
    const int so = ghost_src(P, a, b, cst, neg, val);
    double u = 0.0, al = 0.0, uo = 0.0, alo = 0.0;
    if (so != -2) {
      if (cst) u = uo = val;
      else {
        uo = ub_in[so];
        u = uo + (d_in ? (double)d_in[so] : 0.0);
        if (neg) {
          u = -u;
          uo = -uo;
        }
      }
      const double rh = P.rho[off2m(P, a, b)];
      const double kap = isfinite(u) ? P.k0 * pow_m64(fabs(u), P.kmode, P.km, P.khalf, P.kn) : 0.0;
      al = kap / (rh * P.cp);
      if (io.e_in[0]) {
        const double ko = isfinite(uo) ? P.k0 * pow_m64(fabs(uo), P.kmode, P.km, P.khalf, P.kn) : 0.0;
        alo = ko / (rh * P.cp);
      }
      // the new base state, ghosts included (copy!(T, u) returns them)
      const bool own = (ra >= 1 && ra <= RTX && rb >= 1 && rb <= RTY) ||
                       ((a == -1 || a == ni) && rb >= 1 && rb <= RTY) || ((b == -1 || b == nj) && ra >= 1 && ra <= RTX);
      if (own) {
        const int o = off2m(P, a, b);
        ub_out[o] = u;
        ub32[o] = (float)u;
        ab32[o] = (float)al;
      }
    }
    s_u[rb][ra] = u;
    s_a[rb][ra] = al;
    s_uo[rb][ra] = uo;
    s_ao[rb][ra] = alo;
  }
  __syncthreads();
  for (int f = tid; f < RY * (RTX + 1); f += RNT) {
    const int fb = f / (RTX + 1), fa = f - fb * (RTX + 1);
    const int a = i0 - 1 + fa, b = j0 - 1 + fb;
    double q = 0.0;
    if (a >= -1 && a <= ni - 1 && b >= 0 && b <= nj - 1) {
      q = -face_mean(P.mean, s_a[fb][fa], s_a[fb][fa + 1]) * (s_u[fb][fa + 1] - s_u[fb][fa]);
      if (fb >= 1 && fb <= RTY && (fa >= 1 || a == -1)) {
        const int o = off2m(P, a, b);
        double total;  // damped flux of the iteration so far
        if (io.e_in[0]) {
          const double qo = -face_mean(P.mean, s_ao[fb][fa], s_ao[fb][fa + 1]) * (s_uo[fb][fa + 1] - s_uo[fb][fa]);
          total = qo + (double)io.e_in[0][o];
        } else {
          total = io.q_in[0][o];
        }
        io.e_out[0][o] = (float)(total - q);
        io.q_out[0][o] = total;
      }
    }
    s_qx[fb][fa] = q;
  }
  for (int f = tid; f < (RTY + 1) * RX; f += RNT) {
    const int fb = f / RX, fa = f - fb * RX;
    const int a = i0 - 1 + fa, b = j0 - 1 + fb;
    double q = 0.0;
    if (a >= 0 && a <= ni - 1 && b >= -1 && b <= nj - 1) {
      q = -face_mean(P.mean, s_a[fb][fa], s_a[fb + 1][fa]) * (s_u[fb + 1][fa] - s_u[fb][fa]);
      if (fa >= 1 && fa <= RTX && (fb >= 1 || b == -1)) {
        const int o = off2m(P, a, b);
        double total;
        if (io.e_in[1]) {
          const double qo = -face_mean(P.mean, s_ao[fb][fa], s_ao[fb + 1][fa]) * (s_uo[fb + 1][fa] - s_uo[fb][fa]);
          total = qo + (double)io.e_in[1][o];
        } else {
          total = io.q_in[1][o];
        }
        io.e_out[1][o] = (float)(total - q);
        io.q_out[1][o] = total;
      }
    }
    s_qy[fb][fa] = q;
  }
  __syncthreads();
  double local = 0.0;
  bool nan = false;
  for (int e = tid; e < RTX * RTY; e += RNT) {
    const int cb = e / RTX, ca = e - cb * RTX;
    const int a = i0 + ca, b = j0 + cb;
    if (a >= ni || b >= nj) continue;
    const int o = off2m(P, a, b);
    const int x = ca + 1, y = cb + 1;
    const double dq = P.coef[0][o] * (s_qx[y][x] - s_qx[y][x - 1]) + P.coef[1][o] * (s_qy[y][x] - s_qy[y - 1][x]) +
                      P.coef[2][o] * ((s_qx[y + 1][x] + s_qx[y + 1][x - 1]) - (s_qx[y - 1][x] + s_qx[y - 1][x - 1])) +
                      P.coef[2][o] * ((s_qy[y][x + 1] + s_qy[y - 1][x + 1]) - (s_qy[y][x - 1] + s_qy[y - 1][x - 1])) +
                      P.coef[3][o] * (0.5 * (s_qx[y][x] + s_qx[y][x - 1])) +
                      P.coef[4][o] * (0.5 * (s_qy[y][x] + s_qy[y - 1][x]));
    const double u = s_u[y][x], up = P.u_prev[o];
    double du = u - up;
    if (isapprox_eps(u, up)) du = 0.0;
    const double r = -du / dt - dq + P.S[o];
    R32[o] = (float)r;
    const double ar = fabs(r);
    if (ar != ar) nan = true;
    else local = fmax(local, ar);
  }
  reduce_and_publish<RNT>(P, C, tile, local, nan, s_red, &s_flag, true);
}

// ---------------------------------------------------------------------------
// Damped flux consistent with a guessed start: at a converged step the damped
// flux equals the plain one (q = q′(u) is the fixed point of fluxes.jl:5-16),
// so a start from u₀ ≠ Tⁿ takes q = q′(u₀) = −ᾱ·Δu₀ on every face the sweeps
// read, with α from u₀ (as at iteration 1) and ghosts by the side rules.
__global__ void flux_init2d(Problem P, const double* __restrict__ u, double* __restrict__ qx,
                            double* __restrict__ qy) {
  const int64_t nfx = (int64_t)(P.ni + 1) * P.nj;  // x faces: a = -1..ni-1, b = 0..nj-1
  const int64_t nfy = (int64_t)P.ni * (P.nj + 1);  // y faces: a = 0..ni-1, b = -1..nj-1
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nfx + nfy;
       e += (int64_t)gridDim.x * blockDim.x) {
    int as[2], bs[2];
    double* out;
    if (e < nfx) {
      as[0] = (int)(e % (P.ni + 1)) - 1;
      bs[0] = (int)(e / (P.ni + 1));
      as[1] = as[0] + 1;
      bs[1] = bs[0];
      out = qx;
    } else {
      const int64_t f = e - nfx;
      as[0] = (int)(f % P.ni);
      bs[0] = (int)(f / P.ni) - 1;
      as[1] = as[0];
      bs[1] = bs[0] + 1;
      out = qy;
    }
    double uu[2], al[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      bool cst, neg;
      double val;
      const int so = ghost_src(P, as[k], bs[k], cst, neg, val);
      double v = so >= 0 ? u[so] : val;
      if (neg) v = -v;
      uu[k] = v;
      const double kap = isfinite(v) ? P.k0 * pow_m64(fabs(v), P.kmode, P.km, P.khalf, P.kn) : 0.0;
      al[k] = kap / (P.rho[off2m(P, as[k], bs[k])] * P.cp);
    }
    out[off2m(P, as[0], bs[0])] = -face_mean(P.mean, al[0], al[1]) * (uu[1] - uu[0]);
  }
}

cudaError_t launch_flux_init2d(const Problem& P, const double* u, double* qx, double* qy, cudaStream_t s) {
  const int64_t n = (int64_t)(P.ni + 1) * P.nj + (int64_t)P.ni * (P.nj + 1);
  const int64_t g = (n + 255) / 256;
  flux_init2d<<<(int)(g < 148 * 16 ? g : 148 * 16), 256, 0, s>>>(P, u, qx, qy);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP32 correction sweep, row-marching (the layout of apt_march2d_fast.cu): a
// block of TX threads owns TX-2 columns of a strip of rows, keeps its own
// column in registers, passes neighbour values through shared memory and
// issues the loads of the row after next before it computes the next row.
// Boundary strips run the general instantiation (ghost rules) in one block per
// strip on a side stream; interior strips run a branch-free instantiation in a
// persistent launch whose blocks claim strips from a ticket counter.
//
// The FP32 arithmetic only moves the correction: reciprocals and square roots
// use the hardware approximations (rcp/sqrt.approx, about one ulp), and the
// restarts evaluate everything the stopping rule sees in FP64.
__device__ __forceinline__ float rcp_a(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ float sqrt_a(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// (|1 + x|)ⁿ − 1, accurate relative to x for small x and defined for every x
// (the reference's κ uses |T|ⁿ): one step r ← r + y(1 + r) per integer power,
// (1 + r)√(1+y) − 1 = r√(1+y) + y/(√(1+y) + 1) for the half of a half-integer
// n, expm1(n·log1p(y)) otherwise
__device__ __forceinline__ float incr_pow32(float x, int mode, int m, int half, float n) {
  if (mode == 0) return 0.f;
  const float y = x >= -1.f ? x : -2.f - x;
  if (mode == 2) return expm1f(n * log1pf(y));
  float r = 0.f;
  for (int k = 0; k < m; ++k) r = fmaf(y, 1.f + r, r);
  if (half) {
    const float sq = sqrt_a(1.f + y);
    r = fmaf(r, sq, y * rcp_a(sq + 1.f));
  }
  return r;
}

template <int TX>
struct MixSmem {
  float D[3][TX], UB[3][TX], AB[3][TX], DA[3][TX], IT[3][TX];
  float EX[3][TX], PX[3][TX], EY[2][TX], PY[2][TX];
  double red[TX / 32];
  int flag;
  int ticket;
};

struct MCell {
  float d, ub, ab, da, it, f;
};

template <int TX, bool EDGE, bool HARM>
__device__ __forceinline__ void mixed_body(const Problem& P, Ctrl* C, int tile, int k, bool check,
                                           MixSmem<TX>& sm) {
  constexpr int OW = TX - 2;
  constexpr float kPiF = 3.14159265358979f;
  const int tid = threadIdx.x;
  const int cbk = tile % P.tiles_i, sj = tile / P.tiles_i;
  const int ni = P.ni, nj = P.nj, nx = P.nx, nh = P.nh;
  const int i0 = cbk * OW, a = i0 - 1 + tid;
  const int j0 = sj * P.strip_h, j1 = min(j0 + P.strip_h, nj);
  const float* __restrict__ din = P.d32[(k - 1) & 1];
  float* __restrict__ dout = P.d32[k & 1];
  const float* __restrict__ exin = P.e32[(k - 1) & 1][0];
  const float* __restrict__ eyin = P.e32[(k - 1) & 1][1];
  float* __restrict__ exout = P.e32[k & 1][0];
  float* __restrict__ eyout = P.e32[k & 1][1];
  const float* __restrict__ ub = P.ub32;
  const float* __restrict__ abv = P.ab32;
  const float* __restrict__ Rb = P.R32;
  const float* __restrict__ rho = P.rho32;
  const float* __restrict__ G11 = P.coef32[0];
  const float* __restrict__ G22 = P.coef32[1];
  const float* __restrict__ C12 = P.coef32[2];
  const float* __restrict__ CA = P.coef32[3];
  const float* __restrict__ CB = P.coef32[4];
  const float dt = (float)P.dt, inv_dt = (float)(1.0 / P.dt), cp = (float)P.cp, k0 = (float)P.k0;
  const float LLdt = (float)(P.LL / P.dt), VpL = (float)P.VpL, VpoL = (float)(P.Vpdtau / P.L);
  const float LoVp = (float)(P.L / P.Vpdtau), VpLdt = (float)(P.VpL * P.dt);
  const float kn = (float)P.kn;
  const int kmode = P.kmode, km = P.km, khalf = P.khalf;
  const bool colIn = EDGE ? (a >= 0 && a < ni) : true;
  const bool owner = tid >= 1 && tid <= OW && colIn;
  const bool qx_col = EDGE ? (a >= -1 && a <= ni - 1 && tid < TX - 1) : (tid < TX - 1);
  const bool qx_own = qx_col && (owner || (EDGE && a == -1));
  const int col = a + nh;

  struct Pre {
    float d, ub, ab, rho, ex, ey;
    bool on;
  };
  // loads of row r: the correction at the ghost source, the base state and
  // diffusivity at the cell itself (the restart writes ghosts), old fluxes
  auto prefetch = [&](int r, Pre& L) {
    const int ro = col + nx * (r + nh);
    if (!EDGE) {
      L.on = true;
      L.d = din[ro];
      L.ub = ub[ro];
      L.ab = abv[ro];
      L.rho = rho[ro];
      L.ex = qx_col ? exin[ro] : 0.f;
      L.ey = eyin[ro - nx];
      return;
    }
    bool cst, neg;
    double val;
    const int so = ghost_src(P, a, r, cst, neg, val);
    L.on = so != -2;
    L.d = 0.f;
    L.ub = 0.f;
    L.ab = 0.f;
    L.rho = 1.f;
    if (L.on) {
      if (!cst) L.d = neg ? -din[so] : din[so];  // Dirichlet ghosts carry no correction
      L.ub = ub[ro];
      L.ab = abv[ro];
      L.rho = rho[ro];
    }
    const bool rIn = r >= 0 && r < nj;
    L.ex = (qx_col && rIn) ? exin[ro] : 0.f;
    L.ey = (colIn && r >= 0 && r <= nj) ? eyin[ro - nx] : 0.f;
  };
  auto stage = [&](const Pre& L) -> MCell {
    MCell c{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (EDGE && !L.on) return c;
    c.d = L.d;
    c.ub = L.ub;
    c.ab = L.ab;
    // Δα = α_b((1 + δ/u_b)ⁿ − 1)
    float da = 0.f;
    if (kmode != 0) {
      const float x = c.d * rcp_a(c.ub);
      if (fabsf(c.ub) > 1e-30f && fabsf(x) < 1e30f) da = c.ab * incr_pow32(x, kmode, km, khalf, kn);
      else da = k0 * pow_m32(fabsf(c.ub + c.d), kmode, km, khalf, kn) * rcp_a(L.rho * cp) - c.ab;
    }
    c.da = da;
    // pseudo-time parameters of α(u) = α_b + Δα (iteration_parameters.jl:2-15):
    // dτΔt/(Δt + dτ) = VpLΔt/(αReΔt + VpL); dτ and θ are 0 where α = 0
    const float al = c.ab + da;
    if (al > 0.f) {
      const float Re = kPiF + sqrt_a(kPiF * kPiF + LLdt * L.rho * rcp_a(al));
      c.f = VpLdt * rcp_a(fmaf(al * Re, dt, VpL));
      c.it = HARM ? VpoL * Re : LoVp * rcp_a(Re);
    } else {
      c.f = 0.f;
      c.it = HARM ? __int_as_float(0x7f800000) : 0.f;
    }
    return c;
  };
  // new flux correction of a face between cells c0 and c1, and its undamped part
  auto face = [&](const MCell& c0, float d1, float ub1, float ab1, float da1, float it1, float eold,
                  float& dqp) -> float {
    float en;
    if (HARM) {
      const float s = c0.ab + ab1;
      const float is = rcp_a(s);
      const float abar = 2.f * c0.ab * ab1 * is;
      const float dabar = 2.f * (ab1 * ab1 * c0.da + c0.ab * c0.ab * da1 + c0.da * da1 * s) * is * rcp_a(s + c0.da + da1);
      const float St = c0.it + it1;
      dqp = -((abar + dabar) * (d1 - c0.d) + dabar * (ub1 - c0.ub));
      en = fabsf(St) < __int_as_float(0x7f800000) ? (2.f * eold + dqp * St) * rcp_a(St + 2.f) : dqp;
    } else {
      const float abar = 0.5f * (c0.ab + ab1);
      const float dabar = 0.5f * (c0.da + da1);
      const float tn = 0.5f * (c0.it + it1);
      dqp = -((abar + dabar) * (d1 - c0.d) + dabar * (ub1 - c0.ub));
      en = (eold * tn + dqp) * rcp_a(1.f + tn);
    }
    return en;
  };
  auto publish = [&](int s, const MCell& c) {
    sm.D[s][tid] = c.d;
    sm.UB[s][tid] = c.ub;
    sm.AB[s][tid] = c.ab;
    sm.DA[s][tid] = c.da;
    sm.IT[s][tid] = c.it;
  };
  auto face_x = [&](int r, int s, const MCell& c, float eold, float& dqp) -> float {
    dqp = 0.f;
    if (!(qx_col && (!EDGE || (r >= 0 && r < nj)))) return 0.f;
    return face(c, sm.D[s][tid + 1], sm.UB[s][tid + 1], sm.AB[s][tid + 1], sm.DA[s][tid + 1], sm.IT[s][tid + 1],
                eold, dqp);
  };
  auto face_y = [&](int r, const MCell& lo, const MCell& hi, float eold, float& dqp) -> float {
    dqp = 0.f;
    if (!(colIn && (!EDGE || (r >= -1 && r <= nj - 1)))) return 0.f;
    return face(lo, hi.d, hi.ub, hi.ab, hi.da, hi.it, eold, dqp);
  };

  int s_m = 0, s_0 = 1, s_p = 2, y_m = 0, y_0 = 1;
  Pre L0, L1, Ln;
  prefetch(j0 - 1, L0);
  prefetch(j0, L1);
  prefetch(j0 + 1, Ln);
  const MCell cm = stage(L0);
  MCell c0 = stage(L1);
  publish(s_m, cm);
  publish(s_0, c0);
  __syncthreads();
  float px_m, px_0, py_m;
  float rqx_m = face_x(j0 - 1, s_m, cm, L0.ex, px_m);
  float rqx_0 = face_x(j0, s_0, c0, L1.ex, px_0);
  float rqy_m = face_y(j0 - 1, cm, c0, L1.ey, py_m);
  sm.EX[s_m][tid] = rqx_m;
  sm.PX[s_m][tid] = px_m;
  sm.EX[s_0][tid] = rqx_0;
  sm.PX[s_0][tid] = px_0;
  sm.EY[y_m][tid] = rqy_m;
  sm.PY[y_m][tid] = py_m;
  if (EDGE && j0 == 0 && owner) eyout[col + nx * (nh - 1)] = rqy_m;
  float rpx_m = px_m, rpx_0 = px_0, rpy_m = py_m;
  float f0 = c0.f;  // update factor of row j; its other values are read from the staged window
  float local = 0.f;
  bool nan = false;
  for (int j = j0; j < j1; ++j) {
    const Pre Lc = Ln;
    if (j + 1 < j1) prefetch(j + 2, Ln);
    const int o = col + nx * (j + nh);
    const MCell cp1 = stage(Lc);
    publish(s_p, cp1);
    __syncthreads();
    // the row's coefficients: their loads overlap the face computations
    float g11 = 0, g22 = 0, c12 = 0, ca = 0, cbv = 0, R = 0;
    if (owner) {
      g11 = G11[o];
      g22 = G22[o];
      c12 = C12[o];
      ca = CA[o];
      cbv = CB[o];
      R = Rb[o];
    }
    float px_p1, py_0n;
    const float qx_p1 = face_x(j + 1, s_p, cp1, Lc.ex, px_p1);
    const MCell lo{sm.D[s_0][tid], sm.UB[s_0][tid], sm.AB[s_0][tid], sm.DA[s_0][tid], sm.IT[s_0][tid], 0.f};
    const float qy_0n = face_y(j, lo, cp1, Lc.ey, py_0n);
    sm.EX[s_p][tid] = qx_p1;
    sm.EY[y_0][tid] = qy_0n;
    if (check) {  // the plain fluxes feed the residual only
      sm.PX[s_p][tid] = px_p1;
      sm.PY[y_0][tid] = py_0n;
    }
    __syncthreads();
    if (owner) {
      const int x = tid;
      const float dq = g11 * (rqx_0 - sm.EX[s_0][x - 1]) + g22 * (qy_0n - rqy_m) +
                       c12 * ((qx_p1 + sm.EX[s_p][x - 1]) - (rqx_m + sm.EX[s_m][x - 1])) +
                       c12 * ((sm.EY[y_0][x + 1] + sm.EY[y_m][x + 1]) - (sm.EY[y_0][x - 1] + sm.EY[y_m][x - 1])) +
                       ca * (0.5f * (rqx_0 + sm.EX[s_0][x - 1])) + cbv * (0.5f * (qy_0n + rqy_m));
      const float d0 = sm.D[s_0][x];
      const float dn = d0 + f0 * (R - d0 * inv_dt - dq);
      dout[o] = dn;
      eyout[o] = qy_0n;
      if (check) {
        const float dqp = g11 * (rpx_0 - sm.PX[s_0][x - 1]) + g22 * (py_0n - rpy_m) +
                          c12 * ((px_p1 + sm.PX[s_p][x - 1]) - (rpx_m + sm.PX[s_m][x - 1])) +
                          c12 * ((sm.PY[y_0][x + 1] + sm.PY[y_m][x + 1]) - (sm.PY[y_0][x - 1] + sm.PY[y_m][x - 1])) +
                          ca * (0.5f * (rpx_0 + sm.PX[s_0][x - 1])) + cbv * (0.5f * (py_0n + rpy_m));
        const float ar = fabsf(R - dn * inv_dt - dqp);
        if (ar != ar) nan = true;
        else local = fmaxf(local, ar);
      }
    }
    if (qx_own) exout[o] = rqx_0;
    f0 = cp1.f;
    rqx_m = rqx_0;
    rqx_0 = qx_p1;
    rpx_m = rpx_0;
    rpx_0 = px_p1;
    rqy_m = qy_0n;
    rpy_m = py_0n;
    const int t = s_m;
    s_m = s_0;
    s_0 = s_p;
    s_p = t;
    const int u2 = y_m;
    y_m = y_0;
    y_0 = u2;
  }
  // arrival; the last block advances the inner counters and, on check
  // iterations, publishes max|r| and the end of the cycle
  if (check) {
    reduce_and_publish<TX>(P, C, tile, (double)local, nan, sm.red, &sm.flag, false);
    if (threadIdx.x == 0 && sm.flag) {
      C->inner_iter = k;
      C->iter += 1;
      __threadfence();
    }
  } else if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&C->arrive, 1u);
    if (prev == (unsigned)P.ntiles - 1u) {
      C->arrive = 0u;
      C->inner_iter = k;
      C->iter += 1;
      __threadfence();
    }
  }
}

// Boundary strips: one block per strip.
template <int TX, bool HARM>
__global__ void __launch_bounds__(TX, 4) mixed_sweep2d_edge(const Problem* __restrict__ probs,
                                                            const int2* __restrict__ items) {
  __shared__ MixSmem<TX> sm;
  const int2 item = items[blockIdx.x];
  const Problem& P = probs[item.x];
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->inner_done) || ld_cg_int(&C->done)) return;
  const int k = ld_cg_int(&C->inner_iter) + 1;  // inner iteration of this cycle
  mixed_body<TX, true, HARM>(P, C, item.y, k, (k % C->inner_check_every) == 0, sm);
}

// Interior strips: persistent blocks claim strips from counters[0] until
// `nitems` are taken; the last block to leave resets the counters.
template <int TX, bool HARM>
__global__ void __launch_bounds__(TX, 7) mixed_sweep2d_inner(const Problem* __restrict__ probs,
                                                             const int2* __restrict__ items, int nitems,
                                                             unsigned int* counters) {
  __shared__ MixSmem<TX> sm;
  while (true) {
    if (threadIdx.x == 0) sm.ticket = (int)atomicAdd(&counters[0], 1u);
    __syncthreads();
    const int t = sm.ticket;
    __syncthreads();
    if (t >= nitems) break;
    const int2 item = items[t];
    const Problem& P = probs[item.x];
    Ctrl* C = P.ctrl;
    if (ld_cg_int(&C->inner_done) || ld_cg_int(&C->done)) continue;
    const int k = ld_cg_int(&C->inner_iter) + 1;
    mixed_body<TX, false, HARM>(P, C, item.y, k, (k % C->inner_check_every) == 0, sm);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&counters[1], 1u);
    if (prev == gridDim.x - 1) {
      counters[0] = 0u;
      counters[1] = 0u;
      __threadfence();
    }
  }
}

template <int TX, bool HARM>
static int mixed_inner_grid(int nitems) {
  static int per_sm = -1, nsm = 0;
  if (per_sm < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mixed_sweep2d_inner<TX, HARM>, TX, 0);
    if (per_sm < 1) per_sm = 1;
  }
  const int g = nsm * per_sm;
  return nitems < g ? nitems : g;
}

// one FP32 sweep: boundary strips on the side stream, interior strips on the
// main stream, joined before the next sweep
template <int TX, bool HARM>
static cudaError_t launch_mixed_pair(const Problem* probs, const int2* items, int n_edge, int n_int,
                                     unsigned int* counters, const SweepStreams& ss) {
  const bool fork = n_edge > 0 && n_int > 0 && ss.side != nullptr;
  cudaError_t e = cudaSuccess;
  if (fork) {
    if ((e = cudaEventRecord(ss.ev_fork, ss.main)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.side, ss.ev_fork, 0)) != cudaSuccess) return e;
  }
  if (n_edge > 0) mixed_sweep2d_edge<TX, HARM><<<n_edge, TX, 0, fork ? ss.side : ss.main>>>(probs, items);
  if (n_int > 0)
    mixed_sweep2d_inner<TX, HARM><<<mixed_inner_grid<TX, HARM>(n_int), TX, 0, ss.main>>>(probs, items + n_edge,
                                                                                          n_int, counters);
  if (fork) {
    if ((e = cudaEventRecord(ss.ev_join, ss.side)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.main, ss.ev_join, 0)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

static cudaError_t launch_mixed_sweep(bool harmonic, const Problem* probs, const int2* items, int n_edge, int n_int,
                                      unsigned int* counters, const SweepStreams& ss) {
  return harmonic ? launch_mixed_pair<128, true>(probs, items, n_edge, n_int, counters, ss)
                  : launch_mixed_pair<128, false>(probs, items, n_edge, n_int, counters, ss);
}

// ---------------------------------------------------------------------------
// 3D.  Ghost source (offset) of cell (a, b, c) for the side rules: -1 for a
// constant (Dirichlet) ghost, -2 for a cell that is neither a domain cell nor
// a first-layer non-corner ghost.
__device__ __forceinline__ int64_t ghost_src3(const Problem& P, int a, int b, int c, bool& cst, bool& neg,
                                              double& val) {
  cst = false;
  neg = false;
  val = 0.0;
  const int cls = classify(P, a, b, c);
  if (cls < 0) return -2;
  if (cls == 6) return fidx(P, a, b, c);
  const int rule = P.rule[cls];
  if (rule == GR_DIRICHLET) {
    cst = true;
    val = P.val[cls];
    return -1;
  }
  const int axis = cls >> 1;
  const bool lo = (cls & 1) == 0;
  const int n = axis == 0 ? P.ni : (axis == 1 ? P.nj : P.nk);
  const int p = rule == GR_NONE ? (lo ? -1 : n) : (rule == GR_PERIODIC ? (lo ? n - 1 : 0) : (lo ? 0 : n - 1));
  neg = rule == GR_NEGSYM;
  int aa = a, bb = b, cc = c;
  if (axis == 0) aa = p;
  else if (axis == 1) bb = p;
  else cc = p;
  return fidx(P, aa, bb, cc);
}

// FP64 restart in 3D (the 2D restart above, on 16 x 8 x 4 tiles with a ring):
// u = u_b + δ, ghosts, the carried damped flux split into q′(u) + e, the FP64
// residual with the undamped fluxes (residuals.jl:105-160) and its max-norm,
// and the FP32 copies the sweeps read.
constexpr int R3X = 16, R3Y = 8, R3Z = 4, R3NT = 256;
struct R3Tile {
  static constexpr int RX = R3X + 2, RY = R3Y + 2, RZ = R3Z + 2, NR = RX * RY * RZ;
  static constexpr int NQI = RZ * RY * (R3X + 1), NQJ = RZ * (R3Y + 1) * RX, NQK = (R3Z + 1) * RY * RX;
  static constexpr size_t bytes = sizeof(double) * (4 * NR + NQI + NQJ + NQK);
};

__global__ void __launch_bounds__(R3NT) mixed_restart3d(const Problem* __restrict__ probs, RestartIO io, int rti,
                                                        int rtj) {
  constexpr int RX = R3Tile::RX, RY = R3Tile::RY, NR = R3Tile::NR;
  extern __shared__ double sm3[];
  double* s_u = sm3;
  double* s_a = s_u + NR;
  double* s_uo = s_a + NR;
  double* s_ao = s_uo + NR;
  double* s_qi = s_ao + NR;
  double* s_qj = s_qi + R3Tile::NQI;
  double* s_qk = s_qj + R3Tile::NQJ;
  __shared__ double s_red[R3NT / 32];
  __shared__ int s_flag;
  auto R = [](int x, int y, int z) { return x + RX * (y + RY * z); };
  auto QI = [](int x, int y, int z) { return x + (R3X + 1) * (y + RY * z); };
  auto QJ = [](int x, int y, int z) { return x + RX * (y + (R3Y + 1) * z); };
  auto QK = [](int x, int y, int z) { return x + RX * (y + RY * z); };
  const Problem& P = probs[0];
  Ctrl* C = P.ctrl;
  const int tile = blockIdx.x;
  const int ti = tile % rti, tj = (tile / rti) % rtj, tk = tile / (rti * rtj);
  const int i0 = ti * R3X, j0 = tj * R3Y, k0 = tk * R3Z;
  const int tid = threadIdx.x;
  const int ni = P.ni, nj = P.nj, nk = P.nk;
  const double dt = P.dt;
  for (int r = tid; r < NR; r += R3NT) {
    const int rz = r / (RX * RY), rem = r - rz * RX * RY, ry = rem / RX, rx = rem - ry * RX;
    const int a = i0 - 1 + rx, b = j0 - 1 + ry, c = k0 - 1 + rz;
    bool cst, neg;
    double val;
    const int64_t so = ghost_src3(P, a, b, c, cst, neg, val);
    double u = 0.0, al = 0.0, uo = 0.0, alo = 0.0;
    if (so != -2) {
      if (cst) {
        u = uo = val;
      } else {
        uo = io.ub_in[so];
        u = uo + (io.d_in ? (double)io.d_in[so] : 0.0);
        if (neg) {
          u = -u;
          uo = -uo;
        }
      }
      const int64_t o = fidx(P, a, b, c);
      const double rh = P.rho[o];
      const double kap = isfinite(u) ? P.k0 * pow_m64(fabs(u), P.kmode, P.km, P.khalf, P.kn) : 0.0;
      al = kap / (rh * P.cp);
      if (io.e_in[0]) {
        const double ko = isfinite(uo) ? P.k0 * pow_m64(fabs(uo), P.kmode, P.km, P.khalf, P.kn) : 0.0;
        alo = ko / (rh * P.cp);
      }
      const bool inx = rx >= 1 && rx <= R3X, iny = ry >= 1 && ry <= R3Y, inz = rz >= 1 && rz <= R3Z;
      const bool own = (inx && iny && inz) || ((a == -1 || a == ni) && iny && inz) ||
                       ((b == -1 || b == nj) && inx && inz) || ((c == -1 || c == nk) && inx && iny);
      if (own) {
        io.ub_out[o] = u;
        io.ub32[o] = (float)u;
        io.ab32[o] = (float)al;
      }
    }
    s_u[r] = u;
    s_a[r] = al;
    s_uo[r] = uo;
    s_ao[r] = alo;
  }
  __syncthreads();
  // faces: the plain flux of the new base, and the split of the carried damped flux
  auto face = [&](int comp, int r0, int r1, int64_t o, bool own) -> double {
    const double q = -face_mean(P.mean, s_a[r0], s_a[r1]) * (s_u[r1] - s_u[r0]);
    if (own) {
      double total;
      if (io.e_in[0]) {
        const double qo = -face_mean(P.mean, s_ao[r0], s_ao[r1]) * (s_uo[r1] - s_uo[r0]);
        total = qo + (double)io.e_in[comp][o];
      } else {
        total = io.q_in[comp][o];
      }
      io.e_out[comp][o] = (float)(total - q);
      io.q_out[comp][o] = total;
    }
    return q;
  };
  for (int f = tid; f < R3Tile::NQI; f += R3NT) {
    const int z = f / ((R3X + 1) * RY), rem = f - z * (R3X + 1) * RY, y = rem / (R3X + 1), x = rem - y * (R3X + 1);
    const int a = i0 - 1 + x, b = j0 - 1 + y, c = k0 - 1 + z;
    double q = 0.0;
    if (a >= -1 && a <= ni - 1 && b >= 0 && b <= nj - 1 && c >= 0 && c <= nk - 1)
      q = face(0, R(x, y, z), R(x + 1, y, z), fidx(P, a, b, c),
               y >= 1 && y <= R3Y && z >= 1 && z <= R3Z && (x >= 1 || a == -1));
    s_qi[f] = q;
  }
  for (int f = tid; f < R3Tile::NQJ; f += R3NT) {
    const int z = f / (RX * (R3Y + 1)), rem = f - z * RX * (R3Y + 1), y = rem / RX, x = rem - y * RX;
    const int a = i0 - 1 + x, b = j0 - 1 + y, c = k0 - 1 + z;
    double q = 0.0;
    if (a >= 0 && a <= ni - 1 && b >= -1 && b <= nj - 1 && c >= 0 && c <= nk - 1)
      q = face(1, R(x, y, z), R(x, y + 1, z), fidx(P, a, b, c),
               x >= 1 && x <= R3X && z >= 1 && z <= R3Z && (y >= 1 || b == -1));
    s_qj[f] = q;
  }
  for (int f = tid; f < R3Tile::NQK; f += R3NT) {
    const int z = f / (RX * RY), rem = f - z * RX * RY, y = rem / RX, x = rem - y * RX;
    const int a = i0 - 1 + x, b = j0 - 1 + y, c = k0 - 1 + z;
    double q = 0.0;
    if (a >= 0 && a <= ni - 1 && b >= 0 && b <= nj - 1 && c >= -1 && c <= nk - 1)
      q = face(2, R(x, y, z), R(x, y, z + 1), fidx(P, a, b, c),
               x >= 1 && x <= R3X && y >= 1 && y <= R3Y && (z >= 1 || c == -1));
    s_qk[f] = q;
  }
  __syncthreads();
  double local = 0.0;
  bool nan = false;
  for (int e = tid; e < R3X * R3Y * R3Z; e += R3NT) {
    const int cz = e / (R3X * R3Y), rem = e - cz * R3X * R3Y, cy = rem / R3X, cx = rem - cy * R3X;
    const int a = i0 + cx, b = j0 + cy, c = k0 + cz;
    if (a >= ni || b >= nj || c >= nk) continue;
    const int64_t o = fidx(P, a, b, c);
    const int x = cx + 1, y = cy + 1, z = cz + 1;
    const double* cf[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) cf[k] = P.coef[k];
    // flux_divergence.jl:119-239
    const double dq =
        cf[0][o] * (s_qi[QI(x, y, z)] - s_qi[QI(x - 1, y, z)]) + cf[1][o] * (s_qj[QJ(x, y, z)] - s_qj[QJ(x, y - 1, z)]) +
        cf[2][o] * (s_qk[QK(x, y, z)] - s_qk[QK(x, y, z - 1)]) +
        cf[3][o] * (0.5 * (s_qi[QI(x, y + 1, z)] + s_qi[QI(x - 1, y + 1, z)]) -
                    0.5 * (s_qi[QI(x, y - 1, z)] + s_qi[QI(x - 1, y - 1, z)])) +
        cf[5][o] * (0.5 * (s_qi[QI(x, y, z + 1)] + s_qi[QI(x - 1, y, z + 1)]) -
                    0.5 * (s_qi[QI(x, y, z - 1)] + s_qi[QI(x - 1, y, z - 1)])) +
        cf[3][o] * (0.5 * (s_qj[QJ(x + 1, y, z)] + s_qj[QJ(x + 1, y - 1, z)]) -
                    0.5 * (s_qj[QJ(x - 1, y, z)] + s_qj[QJ(x - 1, y - 1, z)])) +
        cf[4][o] * (0.5 * (s_qj[QJ(x, y, z + 1)] + s_qj[QJ(x, y - 1, z + 1)]) -
                    0.5 * (s_qj[QJ(x, y, z - 1)] + s_qj[QJ(x, y - 1, z - 1)])) +
        cf[4][o] * (0.5 * (s_qk[QK(x, y + 1, z)] + s_qk[QK(x, y + 1, z - 1)]) -
                    0.5 * (s_qk[QK(x, y - 1, z)] + s_qk[QK(x, y - 1, z - 1)])) +
        cf[5][o] * (0.5 * (s_qk[QK(x + 1, y, z)] + s_qk[QK(x + 1, y, z - 1)]) -
                    0.5 * (s_qk[QK(x - 1, y, z)] + s_qk[QK(x - 1, y, z - 1)])) +
        cf[6][o] * (0.5 * (s_qi[QI(x, y, z)] + s_qi[QI(x - 1, y, z)])) +
        cf[7][o] * (0.5 * (s_qj[QJ(x, y, z)] + s_qj[QJ(x, y - 1, z)])) +
        cf[8][o] * (0.5 * (s_qk[QK(x, y, z)] + s_qk[QK(x, y, z - 1)]));
    const double u = s_u[R(x, y, z)], up = P.u_prev[o];
    double du = u - up;
    if (isapprox_eps(u, up)) du = 0.0;
    const double r = -du / dt - dq + P.S[o];
    io.R32[o] = (float)r;
    const double ar = fabs(r);
    if (ar != ar) nan = true;
    else local = fmax(local, ar);
  }
  reduce_and_publish<R3NT>(P, C, tile, local, nan, s_red, &s_flag, true);
}

// FP32 correction sweep in 3D: the plane-marching layout of apt_march3d.cu
// (32 x 8 column, two staged planes, three i/j face planes, two k face planes,
// the loads that stage plane z + 2 issued while plane z is updated, column
// ghost rules resolved once per strip and the k rule once per plane) with the
// cells and faces of the 2D increment form above.
constexpr int X3 = 32, Y3 = 8, NT3 = X3 * Y3, RX3 = X3 + 2, RY3 = Y3 + 2;
constexpr int NRING3 = RX3 * RY3 - NT3;

struct MixSmem3 {
  float D[2][RY3][RX3], UB[2][RY3][RX3], AB[2][RY3][RX3], DA[2][RY3][RX3], IT[2][RY3][RX3];
  float EI[3][RY3][X3 + 1], EJ[3][Y3 + 1][RX3], EK[2][RY3][RX3];
  float PI[3][RY3][X3 + 1], PJ[3][Y3 + 1][RX3], PK[2][RY3][RX3];
  double red[NT3 / 32];
  int flag;
};

template <bool HARM>
__global__ void __launch_bounds__(NT3, 3) mixed_sweep3d(const Problem* __restrict__ probs,
                                                        const int2* __restrict__ items) {
  __shared__ MixSmem3 sm;
  const int2 item = items[blockIdx.x];
  // one descriptor copy serves the whole strip (see stage_problem)
  __shared__ __align__(16) Problem sP;
  stage_problem<NT3>(sP, probs + item.x);
  const Problem& P = sP;
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->inner_done) || ld_cg_int(&C->done)) return;
  const int kk = ld_cg_int(&C->inner_iter) + 1;  // inner iteration of this cycle
  const bool check = (kk % C->inner_check_every) == 0;
  const int tid = threadIdx.x;
  const int tile = item.y;
  const int ti = tile % P.tiles_i, tj = (tile / P.tiles_i) % P.tiles_j, sk = tile / (P.tiles_i * P.tiles_j);
  const int ni = P.ni, nj = P.nj, nk = P.nk;
  const int i0 = ti * X3, j0 = tj * Y3;
  const int k0 = sk * P.strip_h, k1 = min(k0 + P.strip_h, nk);
  const float* __restrict__ din = P.d32[(kk - 1) & 1];
  float* __restrict__ dout = P.d32[kk & 1];
  const float* __restrict__ ein[3] = {P.e32[(kk - 1) & 1][0], P.e32[(kk - 1) & 1][1], P.e32[(kk - 1) & 1][2]};
  float* __restrict__ eout[3] = {P.e32[kk & 1][0], P.e32[kk & 1][1], P.e32[kk & 1][2]};
  const float* __restrict__ ub = P.ub32;
  const float* __restrict__ abv = P.ab32;
  const float* __restrict__ Rb = P.R32;
  const float* __restrict__ rho = P.rho32;
  const float inv_dt = (float)(1.0 / P.dt), dt = (float)P.dt, cp = (float)P.cp, k0c = (float)P.k0;
  const float LLdt = (float)(P.LL / P.dt), VpL = (float)P.VpL, VpoL = (float)(P.Vpdtau / P.L);
  const float LoVp = (float)(P.L / P.Vpdtau), VpLdt = (float)(P.VpL * P.dt);
  const float kn = (float)P.kn;
  const int kmode = P.kmode, km = P.km, khalf = P.khalf;
  constexpr float kPiF = 3.14159265358979f;

  const int ox = tid % X3 + 1, oy = tid / X3 + 1;
  const int oa = i0 + ox - 1, ob = j0 + oy - 1;
  const bool own_in = oa < ni && ob < nj;
  int rx = -1, ry = -1;
  if (tid < NRING3) {
    if (tid < RX3) {
      rx = tid;
      ry = 0;
    } else if (tid < 2 * RX3) {
      rx = tid - RX3;
      ry = RY3 - 1;
    } else {
      const int t = tid - 2 * RX3;
      rx = (t & 1) ? RX3 - 1 : 0;
      ry = 1 + (t >> 1);
    }
  }
  const int ra = i0 + rx - 1, rb = j0 + ry - 1;

  // Raw loads of a cell of plane c — the correction from the cell its ghost
  // rules read, base state, base diffusivity and ρ at the cell itself (the
  // restart writes first-layer ghosts) — issued a plane ahead of stage_pre.
  // mode: 0 copy, 1 negate, 2 constant ghost (zero correction), 3 no cell (a
  // corner ghost or a position outside the ghost layer: staged as zeros).
  struct PreM {
    float d, ub, ab, rh;
    int mode;
  };
  const int64_t plane_sz = (int64_t)P.nx * P.ny;
  const int64_t own_col = fidx(P, oa, ob, 0);
  const int64_t ring_col = rx >= 0 ? fidx(P, ra, rb, 0) : own_col;
  // (i, j) source of a cell's column, fixed for the strip: kind 0 a domain
  // column (the k-ghost rule of each plane applies), 1 / 2 / 3 a first-layer
  // i- or j-ghost column whose side's rule copies / negates the column at `off`
  // or is a constant, 4 neither (boundary_operators.jl)
  struct ColSrc {
    int64_t off;
    int kind;
  };
  auto col_src = [&](int a, int b) -> ColSrc {
    ColSrc r{0, 0};
    const bool ia = a >= 0 && a < ni, ib = b >= 0 && b < nj;
    if (ia && ib) return r;
    int side = -1;
    if (ib && (a == -1 || a == ni)) side = a < 0 ? 0 : 1;
    else if (ia && (b == -1 || b == nj)) side = b < 0 ? 2 : 3;
    r.kind = 4;
    if (side < 0) return r;
    const int rule = P.rule[side];
    if (rule == GR_DIRICHLET) {
      r.kind = 3;
      return r;
    }
    const bool lo = (side & 1) == 0;
    const int n = side < 2 ? ni : nj;
    const int pos = rule == GR_NONE ? (lo ? -1 : n) : rule == GR_PERIODIC ? (lo ? n - 1 : 0) : (lo ? 0 : n - 1);
    r.off = side < 2 ? fidx(P, pos, b, 0) : fidx(P, a, pos, 0);
    r.kind = rule == GR_NEGSYM ? 2 : 1;
    return r;
  };
  const ColSrc own_src = col_src(oa, ob);
  const ColSrc ring_src = rx >= 0 ? col_src(ra, rb) : ColSrc{0, 4};
  // k-ghost rule of plane c (block-uniform): source plane, mode 1 negate, 2 constant
  auto kplane = [&](int c, int& cs, int& mode) {
    cs = c;
    mode = 0;
    if (c >= 0 && c < nk) return;
    const int side = c < 0 ? 4 : 5;
    const int rule = P.rule[side];
    const bool lo = side == 4;
    if (rule == GR_DIRICHLET) mode = 2;
    else if (rule == GR_PERIODIC) cs = lo ? nk - 1 : 0;
    else if (rule != GR_NONE) {
      cs = lo ? 0 : nk - 1;
      mode = rule == GR_NEGSYM ? 1 : 0;
    }
  };
  auto load_cell = [&](const ColSrc& cd, int64_t col, int c, int cs, int kmode, PreM& L) {
    if (cd.kind == 4 || (cd.kind != 0 && (c < 0 || c >= nk))) {
      L.mode = 3;
      return;
    }
    const int64_t o = col + plane_sz * c;
    L.ub = ub[o];
    L.ab = abv[o];
    L.rh = rho[o];
    if (cd.kind == 0) {
      L.mode = kmode;
      L.d = kmode == 2 ? 0.f : din[col + plane_sz * cs];
    } else {
      L.mode = cd.kind == 3 ? 2 : cd.kind - 1;
      L.d = L.mode == 2 ? 0.f : din[cd.off + plane_sz * c];
    }
  };
  auto prefetch = [&](int c, PreM& own, PreM& rg) {
    int cs, mode;
    kplane(c, cs, mode);
    load_cell(own_src, own_col, c, cs, mode, own);
    if (rx >= 0) load_cell(ring_src, ring_col, c, cs, mode, rg);
  };
  // the cell's increments from its raw loads
  auto stage_pre = [&](const PreM& L) -> MCell {
    MCell r{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (L.mode == 3) return r;
    r.d = L.mode == 1 ? -L.d : L.d;
    r.ub = L.ub;
    r.ab = L.ab;
    const float rh = L.rh;
    float da = 0.f;
    if (kmode != 0) {
      const float x = r.d * rcp_a(r.ub);
      if (fabsf(r.ub) > 1e-30f && fabsf(x) < 1e30f) da = r.ab * incr_pow32(x, kmode, km, khalf, kn);
      else da = k0c * pow_m32(fabsf(r.ub + r.d), kmode, km, khalf, kn) * rcp_a(rh * cp) - r.ab;
    }
    r.da = da;
    const float al = r.ab + da;
    if (al > 0.f) {
      const float Re = kPiF + sqrt_a(kPiF * kPiF + LLdt * rh * rcp_a(al));
      r.f = VpLdt * rcp_a(fmaf(al * Re, dt, VpL));
      r.it = HARM ? VpoL * Re : LoVp * rcp_a(Re);
    } else {
      r.f = 0.f;
      r.it = HARM ? __int_as_float(0x7f800000) : 0.f;
    }
    return r;
  };
  // stage plane c into cell slot s from its loads: the own cell (returned) and the ring cell
  auto stage_plane_pre = [&](int s, const PreM& own_l, const PreM& rg_l) -> MCell {
    const MCell own = stage_pre(own_l);
    sm.D[s][oy][ox] = own.d;
    sm.UB[s][oy][ox] = own.ub;
    sm.AB[s][oy][ox] = own.ab;
    sm.DA[s][oy][ox] = own.da;
    sm.IT[s][oy][ox] = own.it;
    if (rx >= 0) {
      const MCell rg = stage_pre(rg_l);
      sm.D[s][ry][rx] = rg.d;
      sm.UB[s][ry][rx] = rg.ub;
      sm.AB[s][ry][rx] = rg.ab;
      sm.DA[s][ry][rx] = rg.da;
      sm.IT[s][ry][rx] = rg.it;
    }
    return own;
  };
  auto stage_plane = [&](int c, int s) -> MCell {
    PreM lo{0.f, 0.f, 0.f, 0.f, 3}, lr{0.f, 0.f, 0.f, 0.f, 3};
    prefetch(c, lo, lr);
    return stage_plane_pre(s, lo, lr);
  };
  // new flux correction between cells (s0, y0, x0) and (s1, y1, x1), and its undamped part
  auto face = [&](int s0, int y0, int x0, int s1, int y1, int x1, float eold, float& dqp) -> float {
    const float ab0 = sm.AB[s0][y0][x0], ab1 = sm.AB[s1][y1][x1];
    const float da0 = sm.DA[s0][y0][x0], da1 = sm.DA[s1][y1][x1];
    const float d0 = sm.D[s0][y0][x0], d1 = sm.D[s1][y1][x1];
    const float ub0 = sm.UB[s0][y0][x0], ub1 = sm.UB[s1][y1][x1];
    const float it0 = sm.IT[s0][y0][x0], it1 = sm.IT[s1][y1][x1];
    float en;
    if (HARM) {
      const float s = ab0 + ab1;
      const float is = rcp_a(s);
      const float abar = 2.f * ab0 * ab1 * is;
      const float dabar = 2.f * (ab1 * ab1 * da0 + ab0 * ab0 * da1 + da0 * da1 * s) * is * rcp_a(s + da0 + da1);
      const float St = it0 + it1;
      dqp = -((abar + dabar) * (d1 - d0) + dabar * (ub1 - ub0));
      en = fabsf(St) < __int_as_float(0x7f800000) ? (2.f * eold + dqp * St) * rcp_a(St + 2.f) : dqp;
    } else {
      const float abar = 0.5f * (ab0 + ab1);
      const float dabar = 0.5f * (da0 + da1);
      const float tn = 0.5f * (it0 + it1);
      dqp = -((abar + dabar) * (d1 - d0) + dabar * (ub1 - ub0));
      en = (eold * tn + dqp) * rcp_a(1.f + tn);
    }
    return en;
  };
  // Face assignment, fixed for the whole strip (as in the FP64 plane march):
  // every thread computes the three faces on the high side of its own cell;
  // NRI + NRJ + NRK threads, each kind starting on a warp boundary, compute one
  // ring face each (i-faces of column 0 and rows 0, RY3-1; j-faces of row 0
  // and columns 0, RX3-1; k-faces of the ring cells).
  constexpr int NRI = RY3 + 2 * X3, NRJ = RX3 + 2 * Y3, NRK = 2 * RX3 + 2 * Y3;
  constexpr int BJ = (NRI + 31) / 32 * 32, BK = BJ + (NRJ + 31) / 32 * 32;
  static_assert(BK + NRK <= NT3, "ring faces fit the block");
  int fk = -1, fx = 0, fy = 0;
  if (tid < NRI) {
    fk = 0;
    if (tid < RY3) {
      fy = tid;
    } else {
      const int t = tid - RY3;
      fy = t < X3 ? 0 : RY3 - 1;
      fx = 1 + (t < X3 ? t : t - X3);
    }
  } else if (tid >= BJ && tid < BJ + NRJ) {
    fk = 1;
    const int t = tid - BJ;
    if (t < RX3) {
      fx = t;
    } else {
      const int u = t - RX3;
      fx = (u & 1) ? RX3 - 1 : 0;
      fy = 1 + (u >> 1);
    }
  } else if (tid >= BK && tid < BK + NRK) {
    fk = 2;
    const int t = tid - BK;
    if (t < 2 * RX3) {
      fy = t < RX3 ? 0 : RY3 - 1;
      fx = t < RX3 ? t : t - RX3;
    } else {
      const int u = t - 2 * RX3;
      fx = (u & 1) ? RX3 - 1 : 0;
      fy = 1 + (u >> 1);
    }
  }
  const int fa = i0 - 1 + fx, fb = j0 - 1 + fy;
  const bool f_ab = fk == 0   ? (fa >= -1 && fa <= ni - 1 && fb >= 0 && fb <= nj - 1)
                    : fk == 1 ? (fa >= 0 && fa <= ni - 1 && fb >= -1 && fb <= nj - 1)
                              : (fa >= 0 && fa <= ni - 1 && fb >= 0 && fb <= nj - 1);
  const bool f_wr = (fk == 0 && fx == 0 && i0 == 0 && fy >= 1 && fy <= Y3) ||
                    (fk == 1 && fy == 0 && j0 == 0 && fx >= 1 && fx <= X3);
  const float* f_in = fk == 0 ? ein[0] : (fk == 1 ? ein[1] : ein[2]);
  float* f_out = fk == 0 ? eout[0] : eout[1];
  const int64_t plane = (int64_t)P.nx * P.ny;
  const int64_t o_col = fidx(P, oa, ob, 0), f_col = fidx(P, fa, fb, 0);
  // old flux corrections at plane c (i, j) and above plane ck (k): {own i, own j, own k, ring}
  auto load_faces = [&](int c, int ck, bool do_k, float* ev) {
    const bool cin = c >= 0 && c < nk, kin = do_k && ck >= -1 && ck <= nk - 1;
    const int64_t oc = o_col + plane * c;
    ev[0] = (own_in && cin) ? ein[0][oc] : 0.f;
    ev[1] = (own_in && cin) ? ein[1][oc] : 0.f;
    ev[2] = (own_in && kin) ? ein[2][o_col + plane * ck] : 0.f;
    ev[3] = 0.f;
    if (f_ab && (fk == 2 ? kin : (fk >= 0 && cin))) ev[3] = f_in[f_col + plane * (fk == 2 ? ck : c)];
  };
  auto faces = [&](int c, int s, int fs, int ck, int sl, int sh, int kf, bool do_k, const float* ev) {
    const bool inz = c >= k0 && c < k1;
    const bool kown = (ck >= k0 && ck < k1) || ck == -1;
    const bool cin = c >= 0 && c < nk, kin = ck >= -1 && ck <= nk - 1;
    const int x = ox, y = oy;
    const int64_t oc = o_col + plane * c;
    {  // own i-face
      float en = 0.f, dqp = 0.f;
      if (own_in && cin) {
        en = face(s, y, x, s, y, x + 1, ev[0], dqp);
        if (inz) eout[0][oc] = en;
      }
      sm.EI[fs][y][x] = en;
      if (check) sm.PI[fs][y][x] = dqp;
    }
    {  // own j-face
      float en = 0.f, dqp = 0.f;
      if (own_in && cin) {
        en = face(s, y, x, s, y + 1, x, ev[1], dqp);
        if (inz) eout[1][oc] = en;
      }
      sm.EJ[fs][y][x] = en;
      if (check) sm.PJ[fs][y][x] = dqp;
    }
    if (do_k) {  // own k-face
      float en = 0.f, dqp = 0.f;
      if (own_in && kin) {
        en = face(sl, y, x, sh, y, x, ev[2], dqp);
        if (kown) eout[2][o_col + plane * ck] = en;
      }
      sm.EK[kf][y][x] = en;
      if (check) sm.PK[kf][y][x] = dqp;
    }
    if (fk == 0) {
      float en = 0.f, dqp = 0.f;
      if (f_ab && cin) {
        en = face(s, fy, fx, s, fy, fx + 1, ev[3], dqp);
        if (inz && f_wr) f_out[f_col + plane * c] = en;
      }
      sm.EI[fs][fy][fx] = en;
      if (check) sm.PI[fs][fy][fx] = dqp;
    } else if (fk == 1) {
      float en = 0.f, dqp = 0.f;
      if (f_ab && cin) {
        en = face(s, fy, fx, s, fy + 1, fx, ev[3], dqp);
        if (inz && f_wr) f_out[f_col + plane * c] = en;
      }
      sm.EJ[fs][fy][fx] = en;
      if (check) sm.PJ[fs][fy][fx] = dqp;
    } else if (fk == 2 && do_k) {
      float en = 0.f, dqp = 0.f;
      if (f_ab && kin) en = face(sl, fy, fx, sh, fy, fx, ev[3], dqp);
      sm.EK[kf][fy][fx] = en;
      if (check) sm.PK[kf][fy][fx] = dqp;
    }
  };
  auto divergence = [&](const float (*QI)[RY3][X3 + 1], const float (*QJ)[Y3 + 1][RX3], const float (*QK)[RY3][RX3],
                        int zm, int z0, int zp, int kmn, int kpl, const float* cf) -> float {
    const int x = ox, y = oy;
    return cf[0] * (QI[z0][y][x] - QI[z0][y][x - 1]) + cf[1] * (QJ[z0][y][x] - QJ[z0][y - 1][x]) +
           cf[2] * (QK[kpl][y][x] - QK[kmn][y][x]) +
           cf[3] * (0.5f * (QI[z0][y + 1][x] + QI[z0][y + 1][x - 1]) - 0.5f * (QI[z0][y - 1][x] + QI[z0][y - 1][x - 1])) +
           cf[5] * (0.5f * (QI[zp][y][x] + QI[zp][y][x - 1]) - 0.5f * (QI[zm][y][x] + QI[zm][y][x - 1])) +
           cf[3] * (0.5f * (QJ[z0][y][x + 1] + QJ[z0][y - 1][x + 1]) - 0.5f * (QJ[z0][y][x - 1] + QJ[z0][y - 1][x - 1])) +
           cf[4] * (0.5f * (QJ[zp][y][x] + QJ[zp][y - 1][x]) - 0.5f * (QJ[zm][y][x] + QJ[zm][y - 1][x])) +
           cf[4] * (0.5f * (QK[kpl][y + 1][x] + QK[kmn][y + 1][x]) - 0.5f * (QK[kpl][y - 1][x] + QK[kmn][y - 1][x])) +
           cf[5] * (0.5f * (QK[kpl][y][x + 1] + QK[kmn][y][x + 1]) - 0.5f * (QK[kpl][y][x - 1] + QK[kmn][y][x - 1])) +
           cf[6] * (0.5f * (QI[z0][y][x] + QI[z0][y][x - 1])) + cf[7] * (0.5f * (QJ[z0][y][x] + QJ[z0][y - 1][x])) +
           cf[8] * (0.5f * (QK[kpl][y][x] + QK[kmn][y][x]));
  };

  int s_0 = 1, s_p = 0;
  int f_m = 0, f_0 = 1, f_p = 2, k_m = 0, k_p = 1;
  float ea[4], eb[4];
  load_faces(k0 - 1, k0 - 1, true, ea);
  load_faces(k0, 0, false, eb);
  stage_plane(k0 - 1, 0);
  MCell cur = stage_plane(k0, 1);
  __syncthreads();
  faces(k0 - 1, 0, f_m, k0 - 1, 0, 1, k_m, true, ea);
  faces(k0, 1, f_0, 0, 0, 0, 0, false, eb);
  load_faces(k0 + 1, k0, true, ea);
  __syncthreads();
  // the stage loads of plane k0 + 1, for the first loop iteration
  PreM p_own{0.f, 0.f, 0.f, 0.f, 3}, p_rg{0.f, 0.f, 0.f, 0.f, 3};
  prefetch(k0 + 1, p_own, p_rg);
  float local = 0.f;
  bool nan = false;
  for (int z = k0; z < k1; ++z) {
    if (z + 1 < k1) load_faces(z + 2, z + 1, true, eb);
    // stage plane z + 1 from its loads, then issue those of plane z + 2
    const MCell nxt = stage_plane_pre(s_p, p_own, p_rg);
    if (z + 1 < k1) prefetch(z + 2, p_own, p_rg);
    __syncthreads();
    float cf[9], R = 0.f;
    const int64_t id = fidx(P, oa, ob, z);
    if (own_in) {
#pragma unroll
      for (int q = 0; q < 9; ++q) cf[q] = P.coef32[q][id];
      R = Rb[id];
    }
    faces(z + 1, s_p, f_p, z, s_0, s_p, k_p, true, ea);
    __syncthreads();
    if (own_in) {
      const float dq = divergence(sm.EI, sm.EJ, sm.EK, f_m, f_0, f_p, k_m, k_p, cf);
      const float dn = cur.d + cur.f * (R - cur.d * inv_dt - dq);
      dout[id] = dn;
      if (check) {
        const float dqp = divergence(sm.PI, sm.PJ, sm.PK, f_m, f_0, f_p, k_m, k_p, cf);
        const float ar = fabsf(R - dn * inv_dt - dqp);
        if (ar != ar) nan = true;
        else local = fmaxf(local, ar);
      }
    }
    cur = nxt;
    const int ts = s_0;
    s_0 = s_p;
    s_p = ts;
    const int tf = f_m;
    f_m = f_0;
    f_0 = f_p;
    f_p = tf;
    const int tk = k_m;
    k_m = k_p;
    k_p = tk;
#pragma unroll
    for (int r = 0; r < 4; ++r) ea[r] = eb[r];
  }
  if (check) {
    reduce_and_publish<NT3>(P, C, tile, (double)local, nan, sm.red, &sm.flag, false);
    if (threadIdx.x == 0 && sm.flag) {
      C->inner_iter = kk;
      C->iter += 1;
      __threadfence();
    }
  } else if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&C->arrive, 1u);
    if (prev == (unsigned)P.ntiles - 1u) {
      C->arrive = 0u;
      C->inner_iter = kk;
      C->iter += 1;
      __threadfence();
    }
  }
}

static cudaError_t launch_mixed_sweep3d(bool harmonic, const Problem* probs, const int2* items, int nitems,
                                        cudaStream_t s) {
  if (harmonic) mixed_sweep3d<true><<<nitems, NT3, 0, s>>>(probs, items);
  else mixed_sweep3d<false><<<nitems, NT3, 0, s>>>(probs, items);
  return cudaGetLastError();
}

// FP32 copies of the metric coefficients and of rho
__global__ void to_f32(const double* __restrict__ src, float* __restrict__ dst, int64_t n) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    dst[e] = (float)src[e];
}

// ---------------------------------------------------------------------------
// host side
int Engine::mixed_alloc() {
  if (ps.size() != 1) {
    set_error("mixed precision is available for single problems (2D or 3D)");
    return CDM_BAD_INPUT;
  }
  ProbState& s = ps[0];
  const size_t N = (size_t)s.nfull;
  auto fa = [&](float** p) -> cudaError_t {
    cudaError_t e = cudaMalloc((void**)p, N * sizeof(float));
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(*p, 0, N * sizeof(float), stream);
  };
  for (int b = 0; b < 2; ++b) {
    CDM_CK(fa(&s.d32[b]));
    for (int d = 0; d < ndim; ++d) CDM_CK(fa(&s.e32[b][d]));
    CDM_CK(cudaMalloc((void**)&s.ub64[b], N * sizeof(double)));
  }
  CDM_CK(fa(&s.ub32));
  CDM_CK(fa(&s.ab32));
  CDM_CK(fa(&s.R32));
  CDM_CK(fa(&s.rho32));
  for (int k = 0; k < (ndim == 2 ? 5 : 9); ++k) {
    CDM_CK(fa(&s.coef32[k]));
    to_f32<<<1184, 256, 0, stream>>>(s.coef[k], s.coef32[k], (int64_t)N);
    CDM_CK(cudaGetLastError());
  }
  return CDM_OK;
}

int Engine::step_mixed(const cdm_step_opts* o, double t_start, double timeout_s) {
  ProbState& s = ps[0];
  Problem& P = hp[0];
  const size_t N = (size_t)s.nfull;
  // restart tiling: 2D rti x rtj tiles of RTX x RTY, 3D rti x rtj x rtk tiles of R3X x R3Y x R3Z
  const int rti = ndim == 2 ? (s.ni + RTX - 1) / RTX : (s.ni + R3X - 1) / R3X;
  const int rtj = ndim == 2 ? (s.nj + RTY - 1) / RTY : (s.nj + R3Y - 1) / R3Y;
  const int rtk = ndim == 2 ? 1 : (s.nk + R3Z - 1) / R3Z;
  if (ndim == 3) {
    static bool attr = false;
    if (!attr) {
      CDM_CK(cudaFuncSetAttribute(mixed_restart3d, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)R3Tile::bytes));
      attr = true;
    }
  }
  // the FP32 sweep uses the strips of the 2D row-marching layout (variant 0)
  to_f32<<<1184, 256, 0, stream>>>(P.rho, s.rho32, (int64_t)N);
  CDM_CK(cudaGetLastError());
  // the bases start as T everywhere (corners and outer halo layers are never rewritten)
  for (int b = 0; b < 2; ++b)
    CDM_CK(cudaMemcpyAsync(s.ub64[b], s.u[0], N * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  Ctrl& Ch = h_ctrl[0];
  const bool debug = std::getenv("CDM_DEBUG_MIXED") != nullptr;
  const double tolmax_abs = o->atol * Ch.sqrtN;  // abs tolerance in max|R| units
  int restarts = 0, iters = 0;
  double init_L2 = INFINITY, rel = 2 * o->rtol, ab = 2 * o->atol;
  auto upload = [&]() -> int {
    CDM_CK(cudaMemcpyAsync(d_probs, hp.data(), sizeof(Problem), cudaMemcpyHostToDevice, stream));
    CDM_CK(cudaMemcpyAsync(d_ctrl, &Ch, sizeof(Ctrl), cudaMemcpyHostToDevice, stream));
    return CDM_OK;
  };
  auto poll = [&]() -> int {
    CDM_CK(cudaMemcpyAsync(&Ch, d_ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream));
    return wait_stream(timeout_s - (now_seconds() - t_start));
  };
  // restart r: u_b(r) = u_b(r-1) + δ (δ absent for r = 0), R_b, max|R_b|
  // ecur: parity of the flux-correction buffer the last sweep wrote (-1: none)
  auto restart = [&](const float* d, int ecur) -> int {
    const double* in = restarts == 0 ? s.u[0] : s.ub64[(restarts - 1) & 1];
    double* out = s.ub64[restarts & 1];
    const int saved_tj = P.tiles_j;
    if (ndim == 2) P.tiles_j = rti;
    P.ntiles = rti * rtj * rtk;
    int rc = upload();
    if (rc != CDM_OK) return rc;
    // the carried flux correction lands in buffer 0, read by the next cycle's
    // first sweep; when the last sweep wrote buffer 1 it is read from there
    RestartIO io;
    io.ub_in = in;
    io.d_in = d;
    io.ub_out = out;
    io.ub32 = s.ub32;
    io.ab32 = s.ab32;
    io.R32 = s.R32;
    for (int c = 0; c < 3; ++c) {
      const bool has = c < ndim;
      io.e_in[c] = has && ecur >= 0 ? s.e32[ecur][c] : nullptr;
      io.q_in[c] = has ? s.q[s.qpar][c] : nullptr;
      io.e_out[c] = has ? s.e32[0][c] : nullptr;
      io.q_out[c] = has ? s.q[s.qpar][c] : nullptr;
    }
    if (ndim == 2) mixed_restart2d<<<rti * rtj, RNT, 0, stream>>>(d_probs, io);
    else mixed_restart3d<<<rti * rtj * rtk, R3NT, R3Tile::bytes, stream>>>(d_probs, io, rti, rtj);
    CDM_CK(cudaGetLastError());
    prof.other_launches += 1;
    prof.fp64_cell_evals += s.ndomain;
    rc = poll();
    if (rc != CDM_OK) return rc;
    P.tiles_j = saved_tj;
    P.ntiles = s.ntiles;
    ++restarts;
    // clear the correction for the next cycle (the flux correction carries over)
    for (int b = 0; b < 2; ++b) CDM_CK(cudaMemsetAsync(s.d32[b], 0, N * sizeof(float), stream));
    return CDM_OK;
  };
  // a convergence check on the FP64 residual of the current base (:284-318)
  auto check = [&](bool first) -> int {
    const double L2 = Ch.restart_nan ? NAN : Ch.restart_L2 / Ch.sqrtN;
    Ch.n_checks += 1;
    if (first) init_L2 = Ch.init_fixed ? Ch.init_L2 : L2;
    rel = L2 / init_L2;
    ab = L2;
    if (!std::isfinite(rel) || !std::isfinite(ab)) return ST_NONFINITE;
    if (iters > o->max_iter) return ST_MAX_ITER;
    if (rel <= o->rtol || ab <= o->atol) return 0;
    return -1;  // continue
  };
  // inner sweeps in blocks of 16 replayed from a captured graph; a sweep after
  // the end of the cycle returns at once
  auto sweeps = [&](int n) -> int {
    int rc = upload();
    if (rc != CDM_OK) return rc;
    const int K = 16;
    if (!mixed_graph) {
      cudaGraph_t g;
      CDM_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t le = cudaSuccess;
      for (int k = 0; k < K && le == cudaSuccess; ++k)
        le = ndim == 2 ? launch_mixed_sweep(mean == CDM_MEAN_HARMONIC, d_probs, d_items, n_edge, nitems - n_edge,
                                            d_counters, sweep_streams())
                       : launch_mixed_sweep3d(mean == CDM_MEAN_HARMONIC, d_probs, d_items, nitems, stream);
      cudaError_t ce = cudaStreamEndCapture(stream, &g);
      CDM_CK(le);
      CDM_CK(ce);
      CDM_CK(cudaGraphInstantiate(&mixed_graph, g, 0));
      cudaGraphDestroy(g);
    }
    int done = 0;
    while (done < n) {
      const int pe = record_pair();
      if (pe >= 0) CDM_CK(cudaEventRecord(ev_pool[pe], stream));
      if (n - done >= K) {
        CDM_CK(cudaGraphLaunch(mixed_graph, stream));
        done += K;
        prof.sweep_launches += K;
      } else {
        for (int k = 0; k < n - done; ++k)
          CDM_CK(ndim == 2 ? launch_mixed_sweep(mean == CDM_MEAN_HARMONIC, d_probs, d_items, n_edge, nitems - n_edge,
                                                d_counters, sweep_streams())
                           : launch_mixed_sweep3d(mean == CDM_MEAN_HARMONIC, d_probs, d_items, nitems, stream));
        prof.sweep_launches += n - done;
        done = n;
      }
      if (pe >= 0) CDM_CK(cudaEventRecord(ev_pool[pe + 1], stream));
      rc = poll();
      if (rc != CDM_OK) return rc;
      if (debug)
        std::fprintf(stderr, "   [mixed] k=%d inner max|r| %.3e best %.3e stall %d\n", Ch.inner_iter, Ch.inner_L2,
                     Ch.inner_best, Ch.inner_stall);
      if (Ch.inner_done) break;
    }
    return CDM_OK;
  };

  Ch.iter = 0;
  Ch.inner_iter = 0;
  Ch.inner_done = 0;
  Ch.inner_check_every = 4;
  Ch.n_checks = 0;
  int rc = restart(nullptr, -1);
  if (rc != CDM_OK) return rc;
  if (Ch.restart_nan) {
    Ch.status = ST_NONFINITE;
    Ch.done = 1;
    return CDM_OK;
  }
  int st = -1;
  bool first = true;
  const int cap_inner = std::max(64, std::min(o->max_iter, 4096));
  while (st < 0) {
    // first cycle: one sweep, so that the first check is at iteration 1 as in the reference
    const double Rmax = Ch.restart_L2;
    // either stopping criterion suffices (rel <= rtol || abs <= atol), so the
    // cycle need not go below the larger of the two thresholds (in max|R| units)
    double target = 1e-3 * Rmax;
    double floor_t = tolmax_abs;
    if (Ch.init_fixed && first) init_L2 = Ch.init_L2;
    if ((!first || Ch.init_fixed) && std::isfinite(init_L2))
      floor_t = std::max(floor_t, o->rtol * init_L2 * Ch.sqrtN);
    target = std::max(target, 0.5 * floor_t);
    Ch.inner_target = target;
    Ch.inner_done = 0;
    Ch.inner_iter = 0;
    Ch.inner_stall = 0;
    Ch.inner_best = INFINITY;
    const int n = first ? 1 : cap_inner;
    rc = sweeps(n);
    if (rc != CDM_OK) return rc;
    iters = Ch.iter;
    const int cur = Ch.inner_iter;
    rc = restart(s.d32[cur & 1], cur & 1);
    if (rc != CDM_OK) return rc;
    st = check(first);
    if (debug)
      std::fprintf(stderr, "[mixed] cycle %d: inner %d (target %.3e, last inner %.3e) restart max|R| %.3e rel %.3e st %d\n",
                   restarts - 1, cur, target, Ch.inner_L2, Ch.restart_L2, rel, st);
    first = false;
    if (Ch.inner_iter >= cap_inner && st < 0 && iters > o->max_iter) st = ST_MAX_ITER;
  }
  Ch.rel = rel;
  Ch.abs = ab;
  Ch.status = st;
  Ch.done = 1;
  Ch.n_restarts = restarts;
  Ch.iter = iters;
  prof.fp32_cell_iters += s.ndomain * (int64_t)iters;
  return CDM_OK;
}

}  // namespace cdm
