// apt_march2d_fast.cu — row-marching FP64 APT pseudo-iteration, reciprocal form.
//
// The same discrete iteration as apt_march2d.cu (and the reference's step!,
// PseudoTransientSolver.jl:253-319), with the divisions of the reference's
// expressions rewritten algebraically so that, with harmonic face means, a cell
// needs two reciprocals and a face one, instead of 4 + 3 per face + 3 IEEE
// divisions (arithmetic means: four per cell, one per face):
//
//   α⁻¹ = ρcₚ/κ,  Re = π + √(π² + (L²/Δt)·ρ·α⁻¹),  dτ = Vp·L·α⁻¹·Re⁻¹,
//   θ = (L/Vp)·Re⁻¹,  θ⁻¹ = (Vp/L)·Re,           (iteration_parameters.jl:2-15)
//   harmonic face means  ᾱ = 2/A, A = α⁻¹ₐ + α⁻¹_b,  θ̄ = 2/S_θ, S_θ = θ⁻¹ₐ + θ⁻¹_b,
//   q ← (qθ̄ − ᾱΔu)/(1 + θ̄) = (2qA − 2Δu·S_θ)/(A(S_θ + 2))        (fluxes.jl:5-16)
//   u ← (u + dτ(uⁿ/Δt − ∇·q + S))/(1 + dτ/Δt)
//     = u·Δt/(Δt + dτ) + dτΔt/(Δt + dτ)·(uⁿ·Δt⁻¹ − ∇·q + S)      (update.jl:13-15)
//   with Δt/(Δt + dτ) = Δt·Re/D, dτΔt/(Δt + dτ) = Vp·L·α⁻¹·Δt/D,
//   D = Δt·Re + Vp·L·α⁻¹
//
// Reciprocals come from the hardware approximation refined by two Newton–
// Raphson steps (y ← y + y(1 − b·y)), accurate to about one ulp, and
// multiply-adds are contracted, so results differ from the operation-for-
// operation path in the last bits only (checked against the CPU oracle at a
// relative L2 of 1e-10 with equal iteration counts).
//
// Organisation (see apt_march2d.cu): a block of TX threads owns TX-2 columns
// and marches up a strip of rows.  Each thread keeps the values of its own
// column (u, update factors, the fluxes of its faces) in registers; only the
// values its neighbours need go through shared memory.  Strips that touch no
// domain boundary run a branch-free instantiation without ghost logic, in a
// persistent launch whose blocks claim strips from a ticket counter (the last
// wave is one strip long); boundary strips run the general instantiation in a
// concurrent launch on a side stream.  Strips whose ring rows are domain rows
// run the branch-free body even when they hold a ghost column: that column's
// rule (source column, negation or constant) is resolved per thread once per
// strip, so only the first and last strip of each column of strips take the
// general body.
#include "cdm_device.cuh"
#include "cdm_finish.cuh"
#include "cdm_fast.cuh"
#include "cdm_kernels.h"

namespace cdm {

namespace {

using fastmath::pow_fast;
using fastmath::rcp_nr;
using fastmath::rcp_pos;

// the row's divergence coefficients, uⁿ and the source, copied into shared
// memory a row ahead by asynchronous copies (each thread its own column): their
// loads then overlap a whole row instead of the row's face computations, and
// hold no registers while in flight.  The wavefront kernel (CO = true) does
// this; the per-iteration kernels keep plain loads: their 6 blocks of 128
// threads per SM would not fit the buffer's shared memory
constexpr int kCoVals = 7;
constexpr int kCoBuf = 2;  // rows in flight + 1: the copies of row j + kCoBuf - 1 are issued at row j

template <int TX, bool CO = false>
struct FastSmem {
  double U[3][TX], IA[3][TX], IT[3][TX];  // u, α⁻¹ (or α), θ⁻¹ (or θ) for the i-1 neighbour
  double QX[3][TX], PX[3][TX];           // new damped / undamped i+1/2 fluxes
  double QY[2][TX], PY[2][TX];           // new damped / undamped j+1/2 fluxes
  double CO_[CO ? kCoBuf : 1][kCoVals][CO ? TX : 1];  // g11, g22, c12, α, β, uⁿ, S of the next rows
  double red[TX / 32];
  int flag;
  int ticket;
  int wok;
  int item;
};

struct Cell {
  double u, ia, it, g, f;
};



}  // namespace

// WAVE: the wavefront schedule, in which other blocks of the same launch write
// u and q between this block's iterations; those arrays are then read through
// L2 only (no read-only-path or L1 copies of another block's writes).
template <int TX, bool EDGE, bool HARM, bool WAVE = false>
__device__ __forceinline__ void fast_body(const Problem& P, Ctrl* C, int tile, int iter, bool check,
                                          FastSmem<TX, WAVE>& sm, int* wave_count = nullptr) {
  constexpr bool kCoAsync = WAVE;
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
  const int kmode = P.kmode, km = P.km, khalf = P.khalf;
  const double kn = P.kn;
  // EDGE = false: the strip's rows and its two ring rows are domain rows, but its
  // columns may include a ghost column (a = -1 or ni), whose rule is resolved
  // below once per strip, and inactive threads past it (a < -1 or a > ni)
  const bool colIn = a >= 0 && a < ni;
  const bool active = a >= -1 && a <= ni;
  const bool owner = tid >= 1 && tid <= OW && colIn;
  const bool qx_col = a >= -1 && a <= ni - 1 && tid < TX - 1;
  const bool qx_own = qx_col && (owner || a == -1);
  // inactive threads read a domain column (their values are never used)
  const int col = active ? a + nh : nh;

  // ghost rule of this thread's column (i sides), resolved once
  int cside = -1, csrc_col = col;
  bool cneg = false, cconst = false;
  double cval = 0.0;
  {
    if (a == -1) cside = 0;
    else if (a == ni) cside = 1;
    if (cside >= 0) {
      const int rule = P.rule[cside];
      const bool lo = cside == 0;
      if (rule == GR_DIRICHLET) {
        cconst = true;
        cval = P.val[cside];
      } else {
        const int p = rule == GR_NONE ? (lo ? -1 : ni) : (rule == GR_PERIODIC ? (lo ? ni - 1 : 0) : (lo ? 0 : ni - 1));
        csrc_col = p + nh;
        cneg = rule == GR_NEGSYM;
      }
    }
  }

  struct Pre {
    double u, ua, rho, qx, qy;
    int off;  // >= 0 source offset, -1 constant (value in u), -2 inactive
    bool neg;
  };
  // issue the loads of row r (u with its ghost source, rho, old fluxes)
  auto prefetch = [&](int r, Pre& L) {
    const int ro = col + nx * (r + nh);
    L.neg = false;
    L.ua = 0.0;
    if (!EDGE) {
      // u of the cell the column rule reads (the cell itself off the ghost column)
      const int so = csrc_col + nx * (r + nh);
      L.off = ro;
      L.neg = cneg;
      L.u = cconst ? cval : (WAVE ? __ldcg(uin + so) : uin[so]);
      if (!alpha_from_u) L.ua = cconst ? cval : uprev[so];
      L.rho = rho[ro];
      L.qx = qx_col ? (WAVE ? __ldcg(qxin + ro) : qxin[ro]) : 0.0;
      L.qy = colIn ? (WAVE ? __ldcg(qyin + ro - nx) : qyin[ro - nx]) : 0.0;
      return;
    }
    int off = -2;
    double cv = 0.0;
    const bool rIn = r >= 0 && r < nj;
    if (rIn) {
      if (colIn) off = ro;
      else if (cside >= 0) {
        if (cconst) {
          off = -1;
          cv = cval;
        } else {
          off = csrc_col + nx * (r + nh);
          L.neg = cneg;
        }
      }
    } else if (colIn && (r == -1 || r == nj)) {
      const int side = r < 0 ? 2 : 3;
      const int rule = P.rule[side];
      const bool lo = side == 2;
      if (rule == GR_DIRICHLET) {
        off = -1;
        cv = P.val[side];
      } else {
        const int p = rule == GR_NONE ? (lo ? -1 : nj) : (rule == GR_PERIODIC ? (lo ? nj - 1 : 0) : (lo ? 0 : nj - 1));
        off = col + nx * (p + nh);
        L.neg = rule == GR_NEGSYM;
      }
    }
    L.off = off;
    L.u = cv;
    L.rho = 1.0;
    if (off >= 0) {
      L.u = WAVE ? __ldcg(uin + off) : uin[off];
      if (!alpha_from_u) L.ua = uprev[off];
    } else if (off == -1) {
      L.ua = cv;
    }
    if (off != -2) L.rho = rho[ro];
    L.qx = (qx_col && rIn) ? (WAVE ? __ldcg(qxin + ro) : qxin[ro]) : 0.0;
    L.qy = (colIn && r >= 0 && r <= nj) ? (WAVE ? __ldcg(qyin + ro - nx) : qyin[ro - nx]) : 0.0;
  };

  int bad = 0;
  // the validity bits of α are read for a step's last iteration only, which is a
  // check iteration or the one past max_iter: other iterations skip the tests
  const bool track_iter = check || iter > C->max_iter;
  // diffusivity, pseudo-time parameters and update factors of cell (a, r)
  auto stage = [&](int r, const Pre& L) -> Cell {
    Cell c{0.0, 0.0, 0.0, 0.0, 0.0};
    if (EDGE ? L.off == -2 : !active) return c;
    const double us = L.neg ? -L.u : L.u;
    const double src = alpha_from_u ? us : (L.neg ? -L.ua : L.ua);
    const double kap = isfinite(src) ? k0 * pow_fast(fabs(src), kmode, km, khalf, kn) : 0.0;
    const double rc = L.rho * cp;
    const double inva = rc * rcp_nr(kap);
    const double Re = kPi + sqrt(kPi * kPi + LLdt * L.rho * inva);
    c.u = us;
    if (HARM) {
      // g = Δt/(Δt + dτ) = Δt·Re/D and f = dτ·g = Vp·L·α⁻¹·Δt/D with
      // D = Δt·Re + Vp·L·α⁻¹: one reciprocal.  A cell whose dτ is not finite
      // (κ = 0) keeps its value: g = 1, f = 0, as dτ = 0 gives.
      const double VA = VpL * inva;
      const double dRe = dt * Re;
      const double D = dRe + VA;
      const bool fin = isfinite(D);
      const double iD = rcp_pos(fin ? D : 1.0);
      c.g = fin ? dRe * iD : 1.0;
      c.f = fin ? VA * dt * iD : 0.0;
      c.ia = inva;
      c.it = VpoL * Re;
    } else {
      const double iRe = rcp_nr(Re);
      double dtau = VpL * inva * iRe;
      double th = LoVp * iRe;
      dtau = isfinite(dtau) ? dtau : 0.0;
      th = isfinite(th) ? th : 0.0;
      const double id = rcp_nr(dt + dtau);
      c.g = dt * id;
      c.f = dtau * dt * id;
      c.ia = kap * rcp_nr(rc);
      c.it = th;
    }
    // validity of α = κ/(ρcₚ) on owned cells and first-layer ghosts
    const bool track = ((tid >= 1 && tid <= OW) || cside >= 0) && track_iter;
    if (track && r >= j0 - (EDGE && j0 == 0) && r < j1 + (EDGE && j1 == nj)) {
      if (!(isfinite(kap) && isfinite(rc) && rc != 0.0)) bad |= 1;
      if (kap != 0.0 && ((kap < 0.0) != (rc < 0.0))) bad |= 2;
    }
    return c;
  };

  auto flux = [&](double ia0, double ia1, double it0, double it1, double du, double qold, double& qp) -> double {
    if (HARM) {
      // ᾱ = 2/A with A = α⁻¹ₐ + α⁻¹_b: q ← (2q − ᾱΔu·S_θ)/(S_θ + 2)
      // = (2qA − 2Δu·S_θ)/(A(S_θ + 2)) and the plain flux −ᾱΔu = −2Δu(S_θ + 2)/(A(S_θ + 2)),
      // over one reciprocal.  θ̄ = 0 when a cell has θ = 0 (θ⁻¹ infinite): q ← −ᾱΔu.
      const double A = ia0 + ia1, St = it0 + it1;
      const bool fin = isfinite(St);
      const double S2 = fin ? St + 2.0 : 1.0;
      const double R = rcp_nr(A * S2);
      const double du2 = 2.0 * du;
      qp = -du2 * S2 * R;
      return fin ? (2.0 * qold * A - du2 * St) * R : qp;
    }
    const double an = 0.5 * (ia0 + ia1);
    const double tn = 0.5 * (it0 + it1);
    qp = -an * du;
    return (qold * tn - an * du) * rcp_nr(1.0 + tn);
  };
  // i+1/2 face of row r between this column and the next (neighbour from shared memory)
  auto face_x = [&](int r, int s, const Cell& c, double qold, double& qp) -> double {
    double qn = 0.0;
    qp = 0.0;
    if (qx_col && (!EDGE || (r >= 0 && r < nj)))
      qn = flux(c.ia, sm.IA[s][tid + 1], c.it, sm.IT[s][tid + 1], sm.U[s][tid + 1] - c.u, qold, qp);
    return qn;
  };
  // j+1/2 face between rows r and r+1 of this column (registers only)
  auto face_y = [&](int r, const Cell& lo, const Cell& hi, double qold, double& qp) -> double {
    double qn = 0.0;
    qp = 0.0;
    if (colIn && (!EDGE || (r >= -1 && r <= nj - 1))) qn = flux(lo.ia, hi.ia, lo.it, hi.it, hi.u - lo.u, qold, qp);
    return qn;
  };
  auto publish = [&](int s, const Cell& c) {
    sm.U[s][tid] = c.u;
    sm.IA[s][tid] = c.ia;
    sm.IT[s][tid] = c.it;
  };

  int s_m = 0, s_0 = 1, s_p = 2;  // slots of rows j-1, j, j+1
  int y_m = 0, y_0 = 1;           // slots of face rows j-1, j
  Pre L0, L1, Ln;
  prefetch(j0 - 1, L0);
  prefetch(j0, L1);
  prefetch(j0 + 1, Ln);
  Cell cm = stage(j0 - 1, L0);
  Cell c0 = stage(j0, L1);
  publish(s_m, cm);
  publish(s_0, c0);
  __syncthreads();
  double px_m, px_0, py_m;
  const double qx_m = face_x(j0 - 1, s_m, cm, L0.qx, px_m);
  const double qx_0 = face_x(j0, s_0, c0, L1.qx, px_0);
  const double qy_m = face_y(j0 - 1, cm, c0, L1.qy, py_m);
  sm.QX[s_m][tid] = qx_m;
  sm.QX[s_0][tid] = qx_0;
  sm.QY[y_m][tid] = qy_m;
  if (check) {  // the plain fluxes feed the residual only
    sm.PX[s_m][tid] = px_m;
    sm.PX[s_0][tid] = px_0;
    sm.PY[y_m][tid] = py_m;
  }
  if (EDGE && j0 == 0 && owner) {
    qyout[col + nx * (nh - 1)] = qy_m;
    uout[col + nx * (nh - 1)] = cm.u;  // row -1 ghost after applybcs!
  }
  // own-column fluxes in registers: x faces of rows j-1 and j, y face of row j-1
  double rqx_m = qx_m, rqx_0 = qx_0, rpx_m = px_m, rpx_0 = px_0, rqy_m = qy_m, rpy_m = py_m;
  double g0 = c0.g, f0 = c0.f;  // update factors of row j; its u, α⁻¹, θ⁻¹ are read from shared memory

  // coefficients of row r into buffer r mod kCoBuf (owners only; every thread commits a group)
  auto fetch_co = [&](int r) {
    if (owner && r < j1) {
      const int o = col + nx * (r + nh);
      const int b = r % kCoBuf;
      cp_async8(&sm.CO_[b][0][tid], G11 + o);
      cp_async8(&sm.CO_[b][1][tid], G22 + o);
      cp_async8(&sm.CO_[b][2][tid], C12 + o);
      cp_async8(&sm.CO_[b][3][tid], CA + o);
      cp_async8(&sm.CO_[b][4][tid], CB + o);
      cp_async8(&sm.CO_[b][5][tid], uprev + o);
      cp_async8(&sm.CO_[b][6][tid], Sg + o);
    }
    cp_async_commit();
  };
  if (kCoAsync)
    for (int r = j0; r < j0 + kCoBuf - 1; ++r) fetch_co(r);

  double local = 0.0;
  bool local_nan = false;
  for (int j = j0; j < j1; ++j) {
    const int o = col + nx * (j + nh);
    if (kCoAsync) fetch_co(j + kCoBuf - 1);  // past the strip: an empty group, so the wait below covers row j
    const Cell cp1 = stage(j + 1, Ln);
    const double lqx = Ln.qx, lqy = Ln.qy;  // old fluxes of row j + 1, used below
    if (j + 1 < j1) prefetch(j + 2, Ln);
    publish(s_p, cp1);
    __syncthreads();
    // the row's coefficients: their loads overlap the face computations
    double g11 = 0, g22 = 0, c12 = 0, ca = 0, cbv = 0, up = 0, S = 0;
    if (!kCoAsync && owner) {
      g11 = G11[o];
      g22 = G22[o];
      c12 = C12[o];
      ca = CA[o];
      cbv = CB[o];
      up = uprev[o];
      S = Sg[o];
    }
    double px_p1, py_0n;
    const double qx_p1 = face_x(j + 1, s_p, cp1, lqx, px_p1);
    const Cell lo{sm.U[s_0][tid], sm.IA[s_0][tid], sm.IT[s_0][tid], 0.0, 0.0};
    const double qy_0n = face_y(j, lo, cp1, lqy, py_0n);
    sm.QX[s_p][tid] = qx_p1;
    sm.QY[y_0][tid] = qy_0n;
    if (check) {
      sm.PX[s_p][tid] = px_p1;
      sm.PY[y_0][tid] = py_0n;
    }
    __syncthreads();
    if (kCoAsync) {
      cp_async_wait<kCoBuf - 1>();  // this thread's copies of row j have landed
      if (owner) {
        const int b = j % kCoBuf;
        g11 = sm.CO_[b][0][tid];
        g22 = sm.CO_[b][1][tid];
        c12 = sm.CO_[b][2][tid];
        ca = sm.CO_[b][3][tid];
        cbv = sm.CO_[b][4][tid];
        up = sm.CO_[b][5][tid];
        S = sm.CO_[b][6][tid];
      }
    }
    if (owner) {
      const int x = tid;
      const double dq = g11 * (rqx_0 - sm.QX[s_0][x - 1]) + g22 * (qy_0n - rqy_m) +
                        c12 * ((qx_p1 + sm.QX[s_p][x - 1]) - (rqx_m + sm.QX[s_m][x - 1])) +
                        c12 * ((sm.QY[y_0][x + 1] + sm.QY[y_m][x + 1]) - (sm.QY[y_0][x - 1] + sm.QY[y_m][x - 1])) +
                        ca * (0.5 * (rqx_0 + sm.QX[s_0][x - 1])) + cbv * (0.5 * (qy_0n + rqy_m));
      const double un = g0 * sm.U[s_0][tid] + f0 * (up * inv_dt - dq + S);
      uout[o] = un;
      qyout[o] = qy_0n;
      if (check) {
        const double dqp = g11 * (rpx_0 - sm.PX[s_0][x - 1]) + g22 * (py_0n - rpy_m) +
                           c12 * ((px_p1 + sm.PX[s_p][x - 1]) - (rpx_m + sm.PX[s_m][x - 1])) +
                           c12 * ((sm.PY[y_0][x + 1] + sm.PY[y_m][x + 1]) - (sm.PY[y_0][x - 1] + sm.PY[y_m][x - 1])) +
                           ca * (0.5 * (rpx_0 + sm.PX[s_0][x - 1])) + cbv * (0.5 * (py_0n + rpy_m));
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
      if (EDGE && j == nj - 1) uout[o + nx] = cp1.u;
    }
    if (qx_own) qxout[o] = rqx_0;
    if (cside >= 0) uout[o] = sm.U[s_0][tid];
    // rotate: rows (j, j+1) become (j-1, j)
    g0 = cp1.g;
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
  // wavefront: every thread's stores are ordered before the arrival that can
  // release the problem's next iteration to other blocks
  if (WAVE) __threadfence();
  finish_iteration<TX>(P, C, tile, iter, check, local, local_nan, bad, sm.red, &sm.flag, wave_count);
}

// Boundary strips: one block per strip.
template <int TX, bool HARM>
__global__ void __launch_bounds__(TX, 5) march2d_fast_edge(const Problem* __restrict__ probs,
                                                           const int2* __restrict__ items) {
  __shared__ FastSmem<TX> sm;
  const int2 item = items[blockIdx.x];
  const Problem& P = probs[item.x];
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->done)) return;
  const int iter = ld_cg_int(&C->iter) + 1;
  const bool check = is_check_iter(C, iter);
  fast_body<TX, true, HARM>(P, C, item.y, iter, check, sm);
}

// Interior strips: persistent blocks claim strips from counters[0] until
// `nitems` are taken; the last block to leave resets the counters.
template <int TX, bool HARM>
__global__ void __launch_bounds__(TX, 6) march2d_fast_inner(const Problem* __restrict__ probs,
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
    fast_body<TX, false, HARM>(P, C, item.y, iter, check, sm);
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

// Wavefront schedule: one persistent launch runs up to K pseudo-iterations of
// every problem.  The launch is K rounds; in each round a problem takes part
// or not, and a problem that takes part contributes one ticket per strip (a
// problem's strips together; bit 30 of the tile index marks a boundary strip).
// Tickets are numbered round by round, problems in order within a round: a
// job is (problem, its j-th iteration of the launch) and covers that
// problem's strips.  A block holding a ticket of job (p, j) with j > 0 waits
// until p has finished j iterations of the launch (wave_count[p] >= j); only
// the blocks holding p's tickets of earlier rounds, all below this ticket, can
// bring that about.  Tickets are taken in order by running blocks, so the
// lowest unfinished ticket never waits and the schedule cannot deadlock.  A
// problem starts its next iteration as soon as its own strips are done.
//
// Pacing: the iteration counts of a batch's problems differ by an order of
// magnitude, and with every problem in every round the fast problems finish
// first and leave the slow ones to run their last iterations on a GPU they no
// longer fill.  The plan kernel gives problem p
//   K_p = ceil(K · rem_p / max_q rem_q)   (1 <= K_p <= K)
// rounds of the launch, rem_p being the iterations left to its expected count
// (the previous step's, Ctrl::est_iter), spread evenly over the K rounds
// (round floor((j + ½)·K/K_p) for its j-th iteration), so that every round
// mixes all problems and they converge together.  A problem without an
// estimate, or past it, takes every round; so does every problem when no
// problem has one (the first step), which is the unpaced schedule.  Pacing
// reorders iterations of independent problems only: every problem runs the
// same iterations on the same data as without it.
//
// Every wait is bounded (about 2 s); a wait that runs out sets counters[3],
// after which every block of the launch leaves without work and the host
// reports the step as failed.
__device__ __forceinline__ int ld_acquire_int(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// thread 0: true once *count >= target; false when the launch's error flag is
// set or the wait runs out after limit_ns (then it sets the flag)
__device__ bool wave_wait(const int* count, int target, unsigned int* err,
                          unsigned long long limit_ns = 2000000000ull) {
  const unsigned long long t0 = global_ns();
  unsigned ns = 32;
  for (int n = 0; n < (1 << 22); ++n) {
    if (ld_acquire_int(count) >= target) return true;
    if (ld_cg_int((const int*)err)) return false;
    if (global_ns() - t0 > limit_ns) break;
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
  atomicExch(err, 1u);
  return false;
}

// self-test of the bounded wait: thread 0 of one block waits for a count that
// nothing raises, gives up after limit_ns and sets *err
__global__ void wave_wait_probe(const int* count, unsigned int* err, unsigned long long limit_ns) {
  if (threadIdx.x == 0) wave_wait(count, 1, err, limit_ns);
}

cudaError_t launch_wave_wait_probe(const int* count, unsigned int* err, double limit_s, cudaStream_t s) {
  wave_wait_probe<<<1, 32, 0, s>>>(count, err, (unsigned long long)(limit_s * 1e9));
  return cudaGetLastError();
}

constexpr int kPlanThreads = 256;

// block-wide inclusive sum of v (kPlanThreads threads); returns the block total in *tot
__device__ __forceinline__ long long plan_scan(long long v, long long* s_w, long long* tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long w = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += w;
  }
  if (lane == 31) s_w[warp] = v;
  __syncthreads();
  long long base = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kPlanThreads / 32; ++w) {
    const long long x = s_w[w];
    if (w < warp) base += x;
    all += x;
  }
  __syncthreads();
  *tot = all;
  return v + base;
}

// Launch prologue (one block): wave counts (problems already done pass every
// wait), the launch's jobs in ticket order and the ticket counter's restart.
__global__ void __launch_bounds__(kPlanThreads) march2d_wave_plan(const Problem* __restrict__ probs, int nprob,
                                                                  int K, int pace, int* wave_count,
                                                                  unsigned int* counters, WavePlan W) {
  __shared__ long long s_w[kPlanThreads / 32];
  __shared__ int s_max[kPlanThreads / 32];
  const int tid = threadIdx.x;
  // the largest number of iterations a problem is expected to have left
  int rmax = 0;
  for (int p = tid; p < nprob; p += kPlanThreads) {
    const Ctrl* C = probs[p].ctrl;
    const int done = ld_cg_int(&C->done);
    wave_count[p] = done ? kWaveDone : 0;
    if (!done && pace) rmax = max(rmax, ld_cg_int(&C->est_iter) - ld_cg_int(&C->iter));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
  if ((tid & 31) == 0) s_max[tid >> 5] = rmax;
  __syncthreads();
  rmax = 0;
  for (int w = 0; w < kPlanThreads / 32; ++w) rmax = max(rmax, s_max[w]);
  // each problem's rounds
  for (int p = tid; p < nprob; p += kPlanThreads) {
    const Ctrl* C = probs[p].ctrl;
    unsigned long long m = 0ull;
    if (!ld_cg_int(&C->done) && probs[p].item0 >= 0) {
      const int rem = ld_cg_int(&C->est_iter) - ld_cg_int(&C->iter);
      int kp = K;
      if (pace && rmax > 0 && rem > 0) kp = min(K, max(1, (int)(((long long)K * rem + rmax - 1) / rmax)));
      for (int j = 0; j < kp; ++j) m |= 1ull << ((2 * j + 1) * K / (2 * kp));
    }
    W.mask[p] = m;
  }
  __syncthreads();
  // jobs round by round, problems in order within a round: the (round,
  // problem) pairs q = r·nprob + p in ticket order, each thread a contiguous
  // run of them, one block scan for every thread's first job and ticket
  const int total = K * nprob;
  const int per = (total + kPlanThreads - 1) / kPlanThreads;
  const int q0 = min(total, tid * per), q1 = min(total, q0 + per);
  long long mine = 0;
  for (int q = q0; q < q1; ++q) {
    const int r = q / nprob, p = q - r * nprob;
    if ((W.mask[p] >> r) & 1ull) mine += (1ll << 40) | (long long)probs[p].ntiles;
  }
  long long tot;
  const long long ex = plan_scan(mine, s_w, &tot) - mine;
  int J = (int)(ex >> 40), tk = (int)(ex & ((1ll << 40) - 1));
  for (int q = q0; q < q1; ++q) {
    const int r = q / nprob, p = q - r * nprob;
    const unsigned long long m = W.mask[p];
    if ((m >> r) & 1ull) {
      W.tb[J] = tk;
      W.pj[J] = make_int2(p, __popcll(m & ((1ull << r) - 1ull)));
      ++J;
      tk += probs[p].ntiles;
    }
  }
  if (tid == 0) {
    const int jobs = (int)(tot >> 40), tickets = (int)(tot & ((1ll << 40) - 1));
    W.tb[jobs] = tickets;
    W.head[0] = jobs;
    W.head[1] = tickets;
    counters[2] = 0u;
  }
}

// 640 threads per SM at the register budget of 5 blocks of 128 (96 registers)
template <int TX, bool HARM>
__global__ void __launch_bounds__(TX, 640 / TX) march2d_fast_wave(const Problem* __restrict__ probs,
                                                           const int2* __restrict__ items, WavePlan W,
                                                           unsigned int* counters, int* wave_count) {
  __shared__ FastSmem<TX, true> sm;
  const int total = W.head[1], njobs = W.head[0];
  while (true) {
    // thread 0 takes the ticket, finds its job and waits for the problem's
    // previous iteration of the launch
    if (threadIdx.x == 0) {
      const int t = ld_cg_int((const int*)&counters[3]) ? total : (int)atomicAdd(&counters[2], 1u);
      int ok = 1, item = 0;
      if (t < total) {
        int lo = 0, hi = njobs - 1;  // the last job starting at or before t
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (__ldg(&W.tb[mid]) <= t) lo = mid;
          else hi = mid - 1;
        }
        const int2 pj = __ldg(&W.pj[lo]);
        item = probs[pj.x].item0 + (t - __ldg(&W.tb[lo]));
        if (pj.y > 0) ok = wave_wait(&wave_count[pj.x], pj.y, &counters[3]);
      }
      sm.ticket = t;
      sm.wok = ok;
      sm.item = item;
    }
    __syncthreads();
    const int t = sm.ticket, ok = sm.wok;
    const int2 item = items[sm.item];
    __syncthreads();
    if (t >= total) break;
    if (!ok) continue;
    const Problem& P = probs[item.x];
    Ctrl* C = P.ctrl;
    if (ld_cg_int(&C->done)) continue;
    const int iter = ld_cg_int(&C->iter) + 1;
    const bool check = is_check_iter(C, iter);
    const int tile = item.y & ((1 << 30) - 1);
    if (item.y >> 30) fast_body<TX, true, HARM, true>(P, C, tile, iter, check, sm, &wave_count[item.x]);
    else fast_body<TX, false, HARM, true>(P, C, tile, iter, check, sm, &wave_count[item.x]);
    __syncthreads();
  }
}

template <int TX, bool HARM>
static int wave_slots() {
  static int per_sm = -1, nsm = 0;
  if (per_sm < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, march2d_fast_wave<TX, HARM>, TX, 0);
    if (per_sm < 1) per_sm = 1;
  }
  return nsm * per_sm;
}

int march2d_wave_slots(int tx, int harmonic) {
  if (tx == 64) return harmonic ? wave_slots<64, true>() : wave_slots<64, false>();
  return harmonic ? wave_slots<128, true>() : wave_slots<128, false>();
}

template <int TX, bool HARM>
static cudaError_t launch_wave(const Problem* probs, int nprob, const int2* items, int nitems, int K, int pace,
                               unsigned int* counters, int* wave_count, const WavePlan& W, cudaStream_t s) {
  const long long slots = wave_slots<TX, HARM>();
  const long long total = (long long)K * nitems;
  const int grid = (int)(total < slots ? total : slots);
  march2d_wave_plan<<<1, kPlanThreads, 0, s>>>(probs, nprob, K, pace, wave_count, counters, W);
  march2d_fast_wave<TX, HARM><<<grid, TX, 0, s>>>(probs, items, W, counters, wave_count);
  return cudaGetLastError();
}

cudaError_t launch_march2d_wave(int tx, int harmonic, const Problem* probs, int nprob, const int2* items,
                                int nitems, int K, int pace, unsigned int* counters, int* wave_count,
                                const WavePlan& W, cudaStream_t s) {
  if (nitems <= 0 || K <= 0) return cudaSuccess;
  if (K > kWaveMaxRounds || (long long)K * nitems >= (1ll << 31) || (long long)K * nprob > W.cap)
    return cudaErrorInvalidValue;
  if (tx == 64)
    return harmonic ? launch_wave<64, true>(probs, nprob, items, nitems, K, pace, counters, wave_count, W, s)
                    : launch_wave<64, false>(probs, nprob, items, nitems, K, pace, counters, wave_count, W, s);
  return harmonic ? launch_wave<128, true>(probs, nprob, items, nitems, K, pace, counters, wave_count, W, s)
                  : launch_wave<128, false>(probs, nprob, items, nitems, K, pace, counters, wave_count, W, s);
}

// Is tile `tile` of a problem free of domain-boundary logic (no ghost column,
// no ghost row in its staged rows)?  The FP32 correction sweep's split.
bool march_tile_interior(int ni, int nj, int tiles_i, int strip_h, int tx, int tile) {
  const int ow = tx - 2;
  const int cb = tile % tiles_i, sj = tile / tiles_i;
  const int i0 = cb * ow, j0 = sj * strip_h, j1 = (j0 + strip_h < nj) ? j0 + strip_h : nj;
  return cb > 0 && i0 + tx - 2 < ni && j0 > 0 && j1 < nj;
}

// Does tile `tile` run the FP64 kernels' branch-free body: no ghost row among its
// staged rows (its columns may include a ghost column, resolved per thread)?
bool march_tile_no_ghost_rows(int nj, int tiles_i, int strip_h, int tile) {
  const int sj = tile / tiles_i;
  const int j0 = sj * strip_h, j1 = (j0 + strip_h < nj) ? j0 + strip_h : nj;
  return j0 > 0 && j1 < nj;
}

template <int TX, bool HARM>
static int inner_grid(int nitems) {
  static int per_sm = -1, nsm = 0;
  if (per_sm < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, march2d_fast_inner<TX, HARM>, TX, 0);
    if (per_sm < 1) per_sm = 1;
  }
  const int g = nsm * per_sm;
  return nitems < g ? nitems : g;
}

template <int TX, bool HARM>
static cudaError_t launch_pair(const Problem* probs, const int2* items, int n_edge, int n_int,
                               unsigned int* counters, const SweepStreams& ss) {
  const bool fork = n_edge > 0 && n_int > 0 && ss.side != nullptr;
  cudaError_t e = cudaSuccess;
  if (fork) {
    if ((e = cudaEventRecord(ss.ev_fork, ss.main)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.side, ss.ev_fork, 0)) != cudaSuccess) return e;
  }
  if (n_edge > 0) march2d_fast_edge<TX, HARM><<<n_edge, TX, 0, fork ? ss.side : ss.main>>>(probs, items);
  if (n_int > 0)
    march2d_fast_inner<TX, HARM><<<inner_grid<TX, HARM>(n_int), TX, 0, ss.main>>>(probs, items + n_edge, n_int,
                                                                                   counters);
  if (fork) {
    if ((e = cudaEventRecord(ss.ev_join, ss.side)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.main, ss.ev_join, 0)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

cudaError_t launch_march2d_fast(int variant, int harmonic, const Problem* probs, const int2* items, int n_edge,
                                int n_int, unsigned int* counters, const SweepStreams& ss) {
  if (variant == 0)
    return harmonic ? launch_pair<128, true>(probs, items, n_edge, n_int, counters, ss)
                    : launch_pair<128, false>(probs, items, n_edge, n_int, counters, ss);
  return harmonic ? launch_pair<64, true>(probs, items, n_edge, n_int, counters, ss)
                  : launch_pair<64, false>(probs, items, n_edge, n_int, counters, ss);
}

}  // namespace cdm
