// apt_march2d_fast.cu — row-marching FP64 APT pseudo-iteration, reciprocal form.
//
// The same discrete iteration as apt_march2d.cu (and the reference's step!,
// PseudoTransientSolver.jl:253-319), with the divisions of the reference's
// expressions rewritten algebraically so that a cell needs four reciprocals
// and a face two, instead of 4 + 3 per face + 3 IEEE divisions:
//
//   α⁻¹ = ρcₚ/κ,  Re = π + √(π² + (L²/Δt)·ρ·α⁻¹),  dτ = Vp·L·α⁻¹·Re⁻¹,
//   θ = (L/Vp)·Re⁻¹,  θ⁻¹ = (Vp/L)·Re,           (iteration_parameters.jl:2-15)
//   harmonic face means  ᾱ = 2/(α⁻¹ₐ + α⁻¹_b),  θ̄ = 2/S_θ with S_θ = θ⁻¹ₐ + θ⁻¹_b,
//   q ← (qθ̄ − ᾱΔu)/(1 + θ̄) = (2q − ᾱΔu·S_θ)/(S_θ + 2)          (fluxes.jl:5-16)
//   u ← (u + dτ(uⁿ/Δt − ∇·q + S))/(1 + dτ/Δt)
//     = u·Δt/(Δt + dτ) + dτΔt/(Δt + dτ)·(uⁿ·Δt⁻¹ − ∇·q + S)      (update.jl:13-15)
//
// Reciprocals come from the hardware approximation refined by two Newton–
// Raphson steps (y ← y + y(1 − b·y)), accurate to about one ulp, and
// multiply-adds are contracted.  Results therefore differ from the
// operation-for-operation path in the last bits only (checked against the
// CPU oracle at a relative L2 of 1e-10 with equal iteration counts).
#include "cdm_device.cuh"
#include "cdm_finish.cuh"
#include "cdm_kernels.h"

namespace cdm {

namespace {

// Newton–Raphson refinement of the hardware reciprocal approximation
// (each step doubles the number of correct bits); exact IEEE division is
// used for zero, subnormal, huge and non-finite arguments.
__device__ __forceinline__ double rcp_nr(double b) {
  const double ab = fabs(b);
  if (!(ab > 1e-290 && ab < 1e290)) return 1.0 / b;
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  e = fma(-b, y, 1.0);
  y = fma(y, e, y);
  return y;
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

}  // namespace

template <int TX>
__global__ void __launch_bounds__(TX, 5) march2d_fast(const Problem* __restrict__ probs,
                                                      const int2* __restrict__ items) {
  constexpr int OW = TX - 2;
  __shared__ double sU[3][TX], sA[3][TX], sT[3][TX], sG[3][TX], sF[3][TX];
  __shared__ double sQX[3][TX], sQY[2][TX], sPX[3][TX], sPY[2][TX];
  __shared__ double s_red[TX / 32];
  __shared__ int s_flag;

  const int2 item = items[blockIdx.x];
  const Problem& P = probs[item.x];
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->done)) return;
  const int iter = ld_cg_int(&C->iter) + 1;
  const bool check = is_check_iter(C, iter);
  const int tid = threadIdx.x;
  const int tile = item.y;
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
  const bool alpha_from_u = P.subcycle || iter == 1;
  const bool harmonic = P.mean == 0;
  const bool rms = C->norm_kind == 1;
  const double dt = P.dt, cp = P.cp, k0 = P.k0;
  const double inv_dt = 1.0 / dt;
  const double LLdt = P.LL / dt, VpL = P.VpL, LoVp = P.L / P.Vpdtau, VpoL = P.Vpdtau / P.L;
  const int kmode = P.kmode, km = P.km, khalf = P.khalf;
  const double kn = P.kn;
  const bool colIn = a >= 0 && a < ni;
  const bool owner = tid >= 1 && tid <= OW && colIn;
  const bool qx_col = a >= -1 && a <= ni - 1 && tid < TX - 1;
  const bool qx_own = qx_col && (owner || a == -1);
  const int col = a + nh;  // full-array column of this thread

  // ghost rule of this thread's column (i sides) resolved once
  int cside = -1;
  if (a == -1) cside = 0;
  else if (a == ni) cside = 1;
  int csrc_col = col;
  bool cneg = false, cconst = false;
  double cval = 0.0;
  if (cside >= 0) {
    const int rule = P.rule[cside];
    const bool lo = cside == 0;
    if (rule == GR_DIRICHLET) {
      cconst = true;
      cval = P.val[cside];
    } else {
      int p = rule == GR_NONE ? (lo ? -1 : ni) : (rule == GR_PERIODIC ? (lo ? ni - 1 : 0) : (lo ? 0 : ni - 1));
      csrc_col = p + nh;
      cneg = rule == GR_NEGSYM;
    }
  }

  // u-source of cell (a, r): offset, constant or inactive
  struct Src {
    int off;  // >= 0 offset; -1 constant; -2 inactive
    bool neg;
    double cv;
  };
  auto src_of = [&](int r) -> Src {
    Src s{-2, false, 0.0};
    const bool rIn = r >= 0 && r < nj;
    if (rIn) {
      if (colIn) s.off = col + nx * (r + nh);
      else if (cside >= 0) {
        if (cconst) {
          s.off = -1;
          s.cv = cval;
        } else {
          s.off = csrc_col + nx * (r + nh);
          s.neg = cneg;
        }
      }
    } else if (colIn && (r == -1 || r == nj)) {
      const int side = r < 0 ? 2 : 3;
      const int rule = P.rule[side];
      const bool lo = side == 2;
      if (rule == GR_DIRICHLET) {
        s.off = -1;
        s.cv = P.val[side];
      } else {
        const int p = rule == GR_NONE ? (lo ? -1 : nj) : (rule == GR_PERIODIC ? (lo ? nj - 1 : 0) : (lo ? 0 : nj - 1));
        s.off = col + nx * (p + nh);
        s.neg = rule == GR_NEGSYM;
      }
    }
    return s;
  };

  struct Pre {
    double u, ua, rho, qx, qy;
    Src s;
  };
  auto prefetch = [&](int r, Pre& L) {
    L.s = src_of(r);
    L.u = 0.0;
    L.ua = 0.0;
    L.rho = 1.0;
    const int ro = col + nx * (r + nh);
    if (L.s.off >= 0) {
      L.u = uin[L.s.off];
      if (!alpha_from_u) L.ua = uprev[L.s.off];
    }
    if (L.s.off != -2) L.rho = rho[ro];
    L.qx = (qx_col && r >= 0 && r < nj) ? qxin[ro] : 0.0;
    L.qy = (colIn && r >= 0 && r <= nj) ? qyin[ro - nx] : 0.0;
  };

  int bad = 0;
  auto stage = [&](int r, int s, const Pre& L) {
    double us = 0.0, ia = 0.0, it = 0.0, g = 0.0, f = 0.0;
    if (L.s.off != -2) {
      us = L.s.off == -1 ? L.s.cv : (L.s.neg ? -L.u : L.u);
      double src = us;
      if (!alpha_from_u) src = L.s.off == -1 ? L.s.cv : (L.s.neg ? -L.ua : L.ua);
      const double kap = isfinite(src) ? k0 * pow_fast(fabs(src), kmode, km, khalf, kn) : 0.0;
      const double rc = L.rho * cp;
      const double inva = rc * rcp_nr(kap);    // α⁻¹
      const double al = harmonic ? 0.0 : kap * rcp_nr(rc);  // α for the arithmetic mean
      const double Re = kPi + sqrt(kPi * kPi + LLdt * L.rho * inva);
      const double iRe = rcp_nr(Re);
      double dtau = VpL * inva * iRe;
      double th = LoVp * iRe;
      dtau = isfinite(dtau) ? dtau : 0.0;
      th = isfinite(th) ? th : 0.0;
      const double id = rcp_nr(dt + dtau);
      g = dt * id;
      f = dtau * dt * id;
      if (harmonic) {
        ia = inva;
        it = VpoL * Re;
      } else {
        ia = al;
        it = th;
      }
      const bool track = (tid >= 1 && tid <= OW) || cside >= 0;
      if (track && r >= j0 - (j0 == 0) && r < j1 + (j1 == nj)) {
        // α = κ/(ρcₚ) is finite iff κ and ρcₚ are finite and ρcₚ ≠ 0; negative iff signs differ
        if (!(isfinite(kap) && isfinite(rc) && rc != 0.0)) bad |= 1;
        if (kap != 0.0 && ((kap < 0.0) != (rc < 0.0))) bad |= 2;
      }
    }
    sU[s][tid] = us;
    sA[s][tid] = ia;
    sT[s][tid] = it;
    sG[s][tid] = g;
    sF[s][tid] = f;
  };

  auto flux = [&](double ia0, double ia1, double it0, double it1, double du, double qold, double& qp) {
    double an, qn;
    if (harmonic) {
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
  auto face_x = [&](int r, int s, double qold) {
    double qn = 0.0, qp = 0.0;
    if (qx_col && r >= 0 && r < nj)
      qn = flux(sA[s][tid], sA[s][tid + 1], sT[s][tid], sT[s][tid + 1], sU[s][tid + 1] - sU[s][tid], qold, qp);
    sQX[s][tid] = qn;
    sPX[s][tid] = qp;
  };
  auto face_y = [&](int r, int s0, int s1, int sy, double qold) {
    double qn = 0.0, qp = 0.0;
    if (colIn && r >= -1 && r <= nj - 1)
      qn = flux(sA[s0][tid], sA[s1][tid], sT[s0][tid], sT[s1][tid], sU[s1][tid] - sU[s0][tid], qold, qp);
    sQY[sy][tid] = qn;
    sPY[sy][tid] = qp;
    return qn;
  };

  // rotating slots: row r lives in slot sl[(r - j0 + 1) % 3]; handled by rotation
  int sm = 0, s0 = 1, sp = 2;  // slots of rows j-1, j, j+1 when processing row j
  int ym = 0, y0 = 1;          // slots of face rows j-1 and j
  Pre L0, L1, Ln;
  prefetch(j0 - 1, L0);
  prefetch(j0, L1);
  stage(j0 - 1, sm, L0);
  stage(j0, s0, L1);
  __syncthreads();
  face_x(j0 - 1, sm, L0.qx);
  face_x(j0, s0, L1.qx);
  {
    const double qn = face_y(j0 - 1, sm, s0, ym, L1.qy);
    if (j0 == 0 && owner) {
      qyout[col + nx * (nh - 1)] = qn;
      uout[col + nx * (nh - 1)] = sU[sm][tid];
    }
  }
  prefetch(j0 + 1, Ln);

  double local = 0.0;
  bool local_nan = false;
  for (int j = j0; j < j1; ++j) {
    const Pre Lc = Ln;
    if (j + 1 < j1) prefetch(j + 2, Ln);
    const int o = col + nx * (j + nh);
    double G11 = 0, G22 = 0, C12 = 0, CA = 0, CB = 0, UP = 0, SS = 0;
    if (owner) {
      G11 = P.coef[0][o];
      G22 = P.coef[1][o];
      C12 = P.coef[2][o];
      CA = P.coef[3][o];
      CB = P.coef[4][o];
      UP = uprev[o];
      SS = P.S[o];
    }
    stage(j + 1, sp, Lc);
    __syncthreads();
    face_x(j + 1, sp, Lc.qx);
    const double qyn = face_y(j, s0, sp, y0, Lc.qy);
    __syncthreads();
    if (owner) {
      const int x = tid;
      const double dq = G11 * (sQX[s0][x] - sQX[s0][x - 1]) + G22 * (sQY[y0][x] - sQY[ym][x]) +
                        C12 * ((sQX[sp][x] + sQX[sp][x - 1]) - (sQX[sm][x] + sQX[sm][x - 1])) +
                        C12 * ((sQY[y0][x + 1] + sQY[ym][x + 1]) - (sQY[y0][x - 1] + sQY[ym][x - 1])) +
                        CA * (0.5 * (sQX[s0][x] + sQX[s0][x - 1])) + CB * (0.5 * (sQY[y0][x] + sQY[ym][x]));
      const double un = sG[s0][x] * sU[s0][x] + sF[s0][x] * (UP * inv_dt - dq + SS);
      uout[o] = un;
      qyout[o] = qyn;
      if (check) {
        const double dqp = G11 * (sPX[s0][x] - sPX[s0][x - 1]) + G22 * (sPY[y0][x] - sPY[ym][x]) +
                           C12 * ((sPX[sp][x] + sPX[sp][x - 1]) - (sPX[sm][x] + sPX[sm][x - 1])) +
                           C12 * ((sPY[y0][x + 1] + sPY[ym][x + 1]) - (sPY[y0][x - 1] + sPY[ym][x - 1])) +
                           CA * (0.5 * (sPX[s0][x] + sPX[s0][x - 1])) + CB * (0.5 * (sPY[y0][x] + sPY[ym][x]));
        double du = un - UP;
        if (isapprox_eps(un, UP)) du = 0.0;
        const double r = -du * inv_dt - dqp + SS;
        if (rms) local += r * r;
        else {
          const double ar = fabs(r);
          if (ar != ar) local_nan = true;
          else local = fmax(local, ar);
        }
      }
      if (j == nj - 1) uout[o + nx] = sU[sp][x];
    }
    if (qx_own) qxout[o] = sQX[s0][tid];
    if (cside >= 0) uout[o] = sU[s0][tid];
    // rotate the windows: rows (j, j+1, j+2) -> slots (s0, sp, sm)
    const int t = sm;
    sm = s0;
    s0 = sp;
    sp = t;
    const int u = ym;
    ym = y0;
    y0 = u;
  }
  finish_iteration<TX>(P, C, tile, iter, check, local, local_nan, bad, s_red, &s_flag);
}

cudaError_t launch_march2d_fast(int variant, const Problem* probs, const int2* items, int nitems, cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  if (variant == 0) march2d_fast<128><<<nitems, 128, 0, s>>>(probs, items);
  else march2d_fast<64><<<nitems, 64, 0, s>>>(probs, items);
  return cudaGetLastError();
}

}  // namespace cdm
