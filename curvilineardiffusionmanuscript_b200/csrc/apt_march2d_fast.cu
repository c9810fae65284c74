// apt_march2d_fast.cu — row-marching FP64 APT pseudo-iteration, reciprocal form.
//
// The same discrete iteration as apt_march2d.cu (and the reference's step!,
// PseudoTransientSolver.jl:253-319), with the divisions of the reference's
// expressions rewritten algebraically so that a cell needs three reciprocals
// and a square root and a face two reciprocals, instead of 4 + 3 per face + 3
// IEEE divisions:
//
//   α⁻¹ = ρcₚ/κ,  Re = π + √(π² + (L²/Δt)·ρ·α⁻¹)            (iteration_parameters.jl:2-15)
//   dτ = Vp·L/(αRe),  θ = L/(Vp·Re),  θ⁻¹ = (Vp/L)·Re
//   D = Δt·κ·Re + Vp·L·ρcₚ:   Δt/(Δt + dτ) = Δt·κ·Re/D,  dτΔt/(Δt + dτ) = Vp·L·Δt·ρcₚ/D
//   harmonic face means  ᾱ = 2/(α⁻¹ₐ + α⁻¹_b),  θ̄ = 2/S_θ with S_θ = θ⁻¹ₐ + θ⁻¹_b
//   q ← (qθ̄ − ᾱΔu)/(1 + θ̄) = (2q − ᾱΔu·S_θ)/(S_θ + 2)                  (fluxes.jl:5-16)
//   u ← (u + dτ(uⁿ/Δt − ∇·q + S))/(1 + dτ/Δt)
//     = u·Δt/(Δt + dτ) + dτΔt/(Δt + dτ)·(uⁿ·Δt⁻¹ − ∇·q + S)              (update.jl:13-15)
//
// Reciprocals come from the hardware approximation refined by two Newton–
// Raphson steps (y ← y + y(1 − b·y)), accurate to about one ulp, and
// multiply-adds are contracted, so results differ from the operation-for-
// operation path in the last bits only (checked against the CPU oracle at a
// relative L2 of 1e-10 with equal iteration counts).
//
// Organisation: a block of TX threads owns TX-2 columns of a strip of rows and
// marches up it (see apt_march2d.cu); each thread keeps its own column's values
// in registers and publishes only what its neighbours read.  Ghost cells are
// handled by per-thread and per-row source offsets, so every tile runs the same
// code.  Blocks are persistent: the grid fills the GPU once and each block
// claims strips from a ticket counter until the launch's strips are exhausted,
// so the last wave is at most one strip long.  The row loop is unrolled by four
// with four shared-memory row slots, which makes every slot index a constant.
#include <type_traits>

#include "cdm_device.cuh"
#include "cdm_finish.cuh"
#include "cdm_kernels.h"

namespace cdm {

namespace {

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

__device__ __forceinline__ double pow_fast(double x, int mode, int m, int half, double n) {
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

template <int TX>
struct FastSmem {
  double U[4][TX], IA[4][TX], IT[4][TX];  // u, α⁻¹ (or α), θ⁻¹ (or θ): read by the i-1 neighbour
  double QX[4][TX], PX[4][TX];           // new damped / undamped i+1/2 fluxes
  double QY[2][TX], PY[2][TX];           // new damped / undamped j+1/2 fluxes
  double red[TX / 32];
  int flag;
  int ticket;
};

struct Cell {
  double u, ia, it, g, f;
};

struct Pre {
  double u, ua, rho, qx, qy;
  bool act;
};

// ghost source of one boundary side: the row/column the rule reads, or a constant
struct SideSrc {
  int pos;   // position along the axis read by the rule
  bool cst;  // Dirichlet
  bool neg;  // negative symmetry
  double val;
};

__device__ __forceinline__ SideSrc side_src(const Problem& P, int side, int n) {
  SideSrc s;
  const int rule = P.rule[side];
  const bool lo = (side & 1) == 0;
  s.cst = rule == GR_DIRICHLET;
  s.neg = rule == GR_NEGSYM;
  s.val = P.val[side];
  s.pos = rule == GR_NONE ? (lo ? -1 : n) : (rule == GR_PERIODIC ? (lo ? n - 1 : 0) : (lo ? 0 : n - 1));
  return s;
}

}  // namespace

template <int TX, bool HARM>
__device__ __forceinline__ void strip(const Problem& P, Ctrl* C, int tile, int iter, bool check, FastSmem<TX>& sm) {
  constexpr int OW = TX - 2;
  const int tid = threadIdx.x;
  const int cb = tile % P.tiles_i, sj = tile / P.tiles_i;
  const int ni = P.ni, nj = P.nj, nx = P.nx, nh = P.nh;
  const int i0 = cb * OW;
  const int a = i0 - 1 + tid;
  const int j0 = sj * P.strip_h, j1 = min(j0 + P.strip_h, nj);
  const int pin = (iter - 1) & 1;
  const double* __restrict__ uin = P.u[pin];
  double* __restrict__ uout = P.u[pin ^ 1];
  const int qin = (P.qpar + iter - 1) & 1;
  const double* __restrict__ qxin = P.q[qin][0];
  const double* __restrict__ qyin = P.q[qin][1];
  double* __restrict__ qxout = P.q[qin ^ 1][0];
  double* __restrict__ qyout = P.q[qin ^ 1][1];
  const double* __restrict__ uprev = P.u_prev;
  const double* __restrict__ rho = P.rho;
  const double* __restrict__ Sg = P.S;
  const double* __restrict__ G11 = P.coef[0];
  const double* __restrict__ G22 = P.coef[1];
  const double* __restrict__ C12 = P.coef[2];
  const double* __restrict__ CA = P.coef[3];
  const double* __restrict__ CB = P.coef[4];
  const bool alpha_from_u = P.subcycle || iter == 1;
  const bool rms = C->norm_kind == 1;
  const double dt = P.dt, cp = P.cp, k0 = P.k0;
  const double inv_dt = 1.0 / dt;
  const double LLdt = P.LL / dt, VpL = P.VpL, LoVp = P.L / P.Vpdtau, VpoL = P.Vpdtau / P.L;
  const double VpLdt = VpL * dt;
  const int kmode = P.kmode, km = P.km, khalf = P.khalf;
  const double kn = P.kn;

  // column of this thread: domain, ghost (i side) or outside
  const bool colIn = a >= 0 && a < ni;
  const bool colGhost = a == -1 || a == ni;
  const bool owner = tid >= 1 && tid <= OW && colIn;
  const bool qx_col = a >= -1 && a <= ni - 1 && tid < TX - 1;
  const bool qx_own = qx_col && (owner || a == -1);
  const int col = a + nh;
  int src_col = col;  // column the u value is read from
  bool col_cst = false, col_neg = false;
  double col_val = 0.0;
  if (colGhost) {
    const SideSrc s = side_src(P, a < 0 ? 0 : 1, ni);
    src_col = s.pos + nh;
    col_cst = s.cst;
    col_neg = s.neg;
    col_val = s.val;
  }
  // ghost rows (j sides)
  const SideSrc rlo = side_src(P, 2, nj), rhi = side_src(P, 3, nj);

  auto prefetch = [&](int r, Pre& L) {
    const int ro = col + nx * (r + nh);
    const bool rowIn = r >= 0 && r < nj;
    const bool rowGhost = r == -1 || r == nj;
    L.act = (colIn && (rowIn || rowGhost)) || (colGhost && rowIn);
    int srow = r;
    bool cst = col_cst, neg = col_neg;
    double cv = col_val;
    if (rowGhost) {
      const SideSrc& s = r < 0 ? rlo : rhi;
      srow = s.pos;
      cst = s.cst;
      neg = s.neg;
      cv = s.val;
    }
    const int so = src_col + nx * (srow + nh);
    double u = cv, ua = cv;
    if (L.act && !cst) {
      u = uin[so];
      ua = alpha_from_u ? u : uprev[so];
      if (neg) {
        u = -u;
        ua = -ua;
      }
    }
    L.u = u;
    L.ua = ua;
    L.rho = L.act ? rho[ro] : 1.0;
    L.qx = (qx_col && rowIn) ? qxin[ro] : 0.0;
    L.qy = (colIn && r >= 0 && r <= nj) ? qyin[ro - nx] : 0.0;
  };

  int bad = 0;
  // diffusivity, pseudo-time parameters and update factors of cell (a, r)
  auto stage = [&](int r, const Pre& L) -> Cell {
    Cell c{0.0, 0.0, 0.0, 0.0, 0.0};
    if (!L.act) return c;
    const double src = alpha_from_u ? L.u : L.ua;
    const double kap = isfinite(src) ? k0 * pow_fast(fabs(src), kmode, km, khalf, kn) : 0.0;
    const double rc = L.rho * cp;
    const double inva = rc * rcp_nr(kap);
    const double Re = kPi + sqrt(kPi * kPi + LLdt * L.rho * inva);
    const double kRe = dt * kap * Re;
    const double iD = rcp_nr(kRe + VpL * rc);
    c.u = L.u;
    // dτ = Vp·L/(α·Re); where dτ is not finite the reference masks it to 0
    const bool dt_ok = isfinite(VpL * inva * rcp_nr(Re));
    c.g = dt_ok ? kRe * iD : 1.0;
    c.f = dt_ok ? VpLdt * rc * iD : 0.0;
    if (HARM) {
      c.ia = inva;
      c.it = VpoL * Re;
    } else {
      const double th = LoVp * rcp_nr(Re);
      c.ia = kap * rcp_nr(rc);
      c.it = isfinite(th) ? th : 0.0;
    }
    // validity of α = κ/(ρcₚ) on owned cells and first-layer ghosts
    const bool track = (tid >= 1 && tid <= OW) || colGhost;
    if (track && r >= j0 - (j0 == 0) && r < j1 + (j1 == nj)) {
      if (!(isfinite(kap) && isfinite(rc) && rc != 0.0)) bad |= 1;
      if (kap != 0.0 && ((kap < 0.0) != (rc < 0.0))) bad |= 2;
    }
    return c;
  };

  auto flux = [&](double ia0, double ia1, double it0, double it1, double du, double qold, double& qp) -> double {
    double an, qn;
    if (HARM) {
      an = 2.0 * rcp_nr(ia0 + ia1);
      const double St = it0 + it1;
      // θ̄ = 0 when a cell has θ = 0 (θ⁻¹ infinite): q ← −ᾱΔu
      qn = isfinite(St) ? (2.0 * qold - an * du * St) * rcp_nr(St + 2.0) : -an * du;
    } else {
      an = 0.5 * (ia0 + ia1);
      const double tn = 0.5 * (it0 + it1);
      qn = (qold * tn - an * du) * rcp_nr(1.0 + tn);
    }
    qp = -an * du;
    return qn;
  };

  double local = 0.0;
  bool local_nan = false;

  // prologue: rows j0-1 and j0 (slots 3 and 0), x faces of both, y face j0-1 (slot 1)
  Pre Lm, L0, Ln;
  prefetch(j0 - 1, Lm);
  prefetch(j0, L0);
  prefetch(j0 + 1, Ln);
  const Cell cm = stage(j0 - 1, Lm);
  Cell c0 = stage(j0, L0);
  sm.U[3][tid] = cm.u;
  sm.IA[3][tid] = cm.ia;
  sm.IT[3][tid] = cm.it;
  sm.U[0][tid] = c0.u;
  sm.IA[0][tid] = c0.ia;
  sm.IT[0][tid] = c0.it;
  __syncthreads();
  double rqx_m = 0.0, rpx_m = 0.0, rqx_0 = 0.0, rpx_0 = 0.0, rqy_m = 0.0, rpy_m = 0.0;
  if (qx_col && j0 - 1 >= 0)
    rqx_m = flux(cm.ia, sm.IA[3][tid + 1], cm.it, sm.IT[3][tid + 1], sm.U[3][tid + 1] - cm.u, Lm.qx, rpx_m);
  if (qx_col)
    rqx_0 = flux(c0.ia, sm.IA[0][tid + 1], c0.it, sm.IT[0][tid + 1], sm.U[0][tid + 1] - c0.u, L0.qx, rpx_0);
  if (colIn) rqy_m = flux(cm.ia, c0.ia, cm.it, c0.it, c0.u - cm.u, L0.qy, rpy_m);
  sm.QX[3][tid] = rqx_m;
  sm.PX[3][tid] = rpx_m;
  sm.QX[0][tid] = rqx_0;
  sm.PX[0][tid] = rpx_0;
  sm.QY[1][tid] = rqy_m;
  sm.PY[1][tid] = rpy_m;
  if (j0 == 0 && owner) {
    qyout[col + nx * (nh - 1)] = rqy_m;
    uout[col + nx * (nh - 1)] = cm.u;  // row -1 ghost after applybcs!
  }

  // one output row j with constant slots: SM, S0, SP rows j-1, j, j+1; YM, Y0 face rows j-1, j
  auto row = [&](int j, auto SMc, auto S0c, auto SPc, auto YMc, auto Y0c) {
    constexpr int SMi = decltype(SMc)::value, S0i = decltype(S0c)::value, SPi = decltype(SPc)::value;
    constexpr int YMi = decltype(YMc)::value, Y0i = decltype(Y0c)::value;
    const Pre Lc = Ln;
    if (j + 1 < j1) prefetch(j + 2, Ln);
    const int o = col + nx * (j + nh);
    double g11 = 0, g22 = 0, c12 = 0, ca = 0, cbv = 0, up = 0, S = 0;
    if (owner) {
      g11 = G11[o];
      g22 = G22[o];
      c12 = C12[o];
      ca = CA[o];
      cbv = CB[o];
      up = uprev[o];
      S = Sg[o];
    }
    const Cell cp1 = stage(j + 1, Lc);
    sm.U[SPi][tid] = cp1.u;
    sm.IA[SPi][tid] = cp1.ia;
    sm.IT[SPi][tid] = cp1.it;
    __syncthreads();
    double px_p1 = 0.0, py_0n = 0.0, qx_p1 = 0.0, qy_0n = 0.0;
    if (qx_col && j + 1 < nj)
      qx_p1 = flux(cp1.ia, sm.IA[SPi][tid + 1], cp1.it, sm.IT[SPi][tid + 1], sm.U[SPi][tid + 1] - cp1.u, Lc.qx,
                   px_p1);
    if (colIn) qy_0n = flux(c0.ia, cp1.ia, c0.it, cp1.it, cp1.u - c0.u, Lc.qy, py_0n);
    sm.QX[SPi][tid] = qx_p1;
    sm.PX[SPi][tid] = px_p1;
    sm.QY[Y0i][tid] = qy_0n;
    sm.PY[Y0i][tid] = py_0n;
    __syncthreads();
    if (owner) {
      const int x = tid;
      const double dq = g11 * (rqx_0 - sm.QX[S0i][x - 1]) + g22 * (qy_0n - rqy_m) +
                        c12 * ((qx_p1 + sm.QX[SPi][x - 1]) - (rqx_m + sm.QX[SMi][x - 1])) +
                        c12 * ((sm.QY[Y0i][x + 1] + sm.QY[YMi][x + 1]) - (sm.QY[Y0i][x - 1] + sm.QY[YMi][x - 1])) +
                        ca * (0.5 * (rqx_0 + sm.QX[S0i][x - 1])) + cbv * (0.5 * (qy_0n + rqy_m));
      const double un = c0.g * c0.u + c0.f * (up * inv_dt - dq + S);
      uout[o] = un;
      qyout[o] = qy_0n;
      if (check) {
        const double dqp = g11 * (rpx_0 - sm.PX[S0i][x - 1]) + g22 * (py_0n - rpy_m) +
                           c12 * ((px_p1 + sm.PX[SPi][x - 1]) - (rpx_m + sm.PX[SMi][x - 1])) +
                           c12 * ((sm.PY[Y0i][x + 1] + sm.PY[YMi][x + 1]) - (sm.PY[Y0i][x - 1] + sm.PY[YMi][x - 1])) +
                           ca * (0.5 * (rpx_0 + sm.PX[S0i][x - 1])) + cbv * (0.5 * (py_0n + rpy_m));
        double du = un - up;
        if (isapprox_eps(un, up)) du = 0.0;
        const double r = -du * inv_dt - dqp + S;
        if (rms) local += r * r;
        else {
          const double ar = fabs(r);
          if (ar != ar) local_nan = true;
          else local = fmax(local, ar);
        }
      }
      if (j == nj - 1) uout[o + nx] = cp1.u;
    }
    if (qx_own) qxout[o] = rqx_0;
    if (colGhost) uout[o] = c0.u;
    c0 = cp1;
    rqx_m = rqx_0;
    rqx_0 = qx_p1;
    rpx_m = rpx_0;
    rpx_0 = px_p1;
    rqy_m = qy_0n;
    rpy_m = py_0n;
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  using I3 = std::integral_constant<int, 3>;
  // row j0 + k uses slots ((k+3)&3, k&3, (k+1)&3) and face slots ((k+1)&1, k&1)
  int j = j0;
  for (; j + 4 <= j1; j += 4) {
    row(j, I3{}, I0{}, I1{}, I1{}, I0{});
    row(j + 1, I0{}, I1{}, I2{}, I0{}, I1{});
    row(j + 2, I1{}, I2{}, I3{}, I1{}, I0{});
    row(j + 3, I2{}, I3{}, I0{}, I0{}, I1{});
  }
  const int rem = j1 - j;
  if (rem > 0) row(j, I3{}, I0{}, I1{}, I1{}, I0{});
  if (rem > 1) row(j + 1, I0{}, I1{}, I2{}, I0{}, I1{});
  if (rem > 2) row(j + 2, I1{}, I2{}, I3{}, I1{}, I0{});
  finish_iteration<TX>(P, C, tile, iter, check, local, local_nan, bad, sm.red, &sm.flag);
}

// Persistent launch: blocks claim items from counters[0] until `nitems` are
// taken; the last block to leave resets the counters for the next launch.
template <int TX, bool HARM>
__global__ void __launch_bounds__(TX, 4) march2d_fast(const Problem* __restrict__ probs,
                                                      const int2* __restrict__ items, int nitems,
                                                      unsigned int* counters) {
  __shared__ FastSmem<TX> sm;
  while (true) {
    if (threadIdx.x == 0) sm.ticket = (int)atomicAdd(&counters[0], 1u);
    __syncthreads();
    const int t = sm.ticket;
    __syncthreads();
    if (t >= nitems) break;
    const int2 item = items[t];
    const Problem& P = probs[item.x];
    Ctrl* C = P.ctrl;
    if (ld_cg_int(&C->done)) continue;
    const int iter = ld_cg_int(&C->iter) + 1;
    const bool check = is_check_iter(C, iter);
    strip<TX, HARM>(P, C, item.y, iter, check, sm);
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

template <int TX>
static int fast_grid(int nitems) {
  static int per_sm = -1;
  static int nsm = 0;
  if (per_sm < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, march2d_fast<TX, true>, TX, 0);
    if (per_sm < 1) per_sm = 1;
  }
  const int g = nsm * per_sm;
  return nitems < g ? nitems : g;
}

cudaError_t launch_march2d_fast(int variant, int harmonic, const Problem* probs, const int2* items, int nitems,
                                unsigned int* counters, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  if (variant == 0) {
    const int g = fast_grid<128>(nitems);
    if (harmonic) march2d_fast<128, true><<<g, 128, 0, s>>>(probs, items, nitems, counters);
    else march2d_fast<128, false><<<g, 128, 0, s>>>(probs, items, nitems, counters);
  } else {
    const int g = fast_grid<64>(nitems);
    if (harmonic) march2d_fast<64, true><<<g, 64, 0, s>>>(probs, items, nitems, counters);
    else march2d_fast<64, false><<<g, 64, 0, s>>>(probs, items, nitems, counters);
  }
  return cudaGetLastError();
}

}  // namespace cdm
