// apt_march2d.cu — row-marching fused FP64 APT pseudo-iteration (2D).
//
// Same arithmetic as apt_sweep_fp64.cu (one pseudo-iteration of step!,
// PseudoTransientSolver.jl:253-319, with the stages of conductivity.jl:15-23,
// iteration_parameters.jl:2-15, fluxes.jl:5-26, flux_divergence.jl:7-42,
// update.jl:2-21 and residuals.jl:24-47), organised for bandwidth:
//
//  * a block of TX threads owns TX-2 consecutive columns; thread t works on
//    column i0-1+t for the whole strip, so the one-cell column ring is part of
//    the block (neighbouring blocks overlap by two columns) and every thread
//    executes the same instructions;
//  * the block marches up a strip of rows.  For output row j it stages
//    row j+1 (u with ghost rules, diffusivity, pseudo-time parameters), then
//    the new damped fluxes of face row j+1 (i+1/2) and j+1/2, then updates
//    row j.  Three-row rolling windows in shared memory hold what the
//    divergence of row j reads, so each face is computed once per strip;
//  * the global loads of the next row are issued one row ahead into
//    registers, so memory latency overlaps the FP64 work of the current row;
//  * all offsets are 32-bit (the engine rejects 2D meshes with nx*ny >= 2^31);
//  * TZ: the twilight-zone forcing (update.jl:23-71, residuals.jl:49-99) is
//    added to the update and the residual, from the step's precomputed terms
//    and the row's diffusivity (cdm_tz.cuh).
#include "cdm_device.cuh"
#include "cdm_kernels.h"
#include "cdm_finish.cuh"
#include "cdm_tz.cuh"

namespace cdm {

namespace {

// full-array offset of domain cell (a, b) in 2D
__device__ __forceinline__ int off2(const Problem& P, int a, int b) { return (a + P.nh) + P.nx * (b + P.nh); }

// Source of u at cell (a, r) for the ghost rules: returns the offset to read
// (or -1 for a constant, written to *cval, or -2 for an inactive corner).
// `neg` is set for the negative-symmetry rule.
__device__ __forceinline__ int u_source(const Problem& P, int a, int r, double* cval, bool* neg) {
  *neg = false;
  const bool ca = a >= 0 && a < P.ni, cr = r >= 0 && r < P.nj;
  if (ca && cr) return off2(P, a, r);
  int side, pos_a = a, pos_r = r;
  if (cr && (a == -1 || a == P.ni)) side = a < 0 ? 0 : 1;
  else if (ca && (r == -1 || r == P.nj)) side = r < 0 ? 2 : 3;
  else return -2;
  const int rule = P.rule[side];
  if (rule == GR_DIRICHLET) {
    *cval = P.val[side];
    return -1;
  }
  const bool lo = (side & 1) == 0;
  const int n = side < 2 ? P.ni : P.nj;
  int p;
  if (rule == GR_NONE) p = lo ? -1 : n;
  else if (rule == GR_PERIODIC) p = lo ? n - 1 : 0;
  else p = lo ? 0 : n - 1;
  if (side < 2) pos_a = p;
  else pos_r = p;
  *neg = rule == GR_NEGSYM;
  return off2(P, pos_a, pos_r);
}

// Per-row loads of one thread, issued a row ahead.
struct RowLoads {
  double u, up_bc, rho;   // stage of cell (a, r): u_in (rule applied later), u_prev (rule), rho
  double qx, qy;          // old fluxes at faces (a, r) i+1/2 and (a, r-1) j+1/2
  double g11, g22, c12, ca, cb, up, S;  // update of cell (a, r-1)
  tz::Terms tzt;          // its twilight-zone terms (TZ only)
  int usrc;               // -1 const, -2 inactive, else offset
  bool neg;
  double cval;
};

}  // namespace

template <int TX, bool TZ>
__global__ void __launch_bounds__(TX) march2d_fp64(const Problem* __restrict__ probs, const int2* __restrict__ items) {
  constexpr int OW = TX - 2;
  __shared__ double sU[3][TX], sA[3][TX], sT[3][TX], sD[3][TX];
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
  const int ni = P.ni, nj = P.nj;
  const int H = P.strip_h;  // strip height (rows)
  const int i0 = cb * OW;
  const int a = i0 - 1 + tid;
  const int j0 = sj * H, j1 = min(j0 + H, nj);
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
  const int mean = P.mean;
  const double dt = P.dt;
  const bool rms = C->norm_kind == 1;
  const bool colIn = a >= 0 && a < ni;
  const bool owner = tid >= 1 && tid <= OW && colIn;                 // updates cells of column a
  const bool qx_act_col = a >= -1 && a <= ni - 1 && tid < TX - 1;    // i+1/2 face of column a exists
  const bool qx_own = qx_act_col && (owner || (a == -1));           // writes that face
  const bool qy_act_col = colIn;

  // issue the loads that row r needs (stage of row r, fluxes, update of row r-1)
  auto load_row = [&](int r, RowLoads& L) {
    L.usrc = u_source(P, a, r, &L.cval, &L.neg);
    L.u = 0.0;
    L.up_bc = 0.0;
    L.rho = 1.0;
    if (L.usrc >= 0) {
      L.u = uin[L.usrc];
      if (!alpha_from_u) L.up_bc = uprev[L.usrc];
    }
    if (L.usrc != -2) L.rho = rho[off2(P, a, r)];
    L.qx = (qx_act_col && r >= 0 && r < nj) ? qxin[off2(P, a, r)] : 0.0;
    L.qy = (qy_act_col && r - 1 >= -1 && r - 1 <= nj - 1) ? qyin[off2(P, a, r - 1)] : 0.0;
    const int ru = r - 1;
    if (owner && ru >= j0 && ru < j1) {
      const int o = off2(P, a, ru);
      L.g11 = G11[o];
      L.g22 = G22[o];
      L.c12 = C12[o];
      L.ca = CA[o];
      L.cb = CB[o];
      L.up = uprev[o];
      L.S = Sg[o];
      if (TZ) {
        const double* tzp = P.tz + o;
        const int64_t st = (int64_t)P.nx * P.ny;
        L.tzt.ut = tzp[0];
        L.tzt.p1 = tzp[st];
        L.tzt.uxx = tzp[2 * st];
        L.tzt.p2 = tzp[3 * st];
        L.tzt.uee = tzp[4 * st];
        L.tzt.uxe = tzp[5 * st];
        L.tzt.p3 = tzp[6 * st];
        L.tzt.p4 = tzp[7 * st];
        L.tzt.ux = tzp[8 * st];
        L.tzt.ue = tzp[9 * st];
      }
    }
  };

  int bad = 0;
  // stage of row r into buffer slot (r+3)%3 from loads L
  auto stage = [&](int r, const RowLoads& L) {
    const int s = (r + 3) % 3;
    double us = 0.0, al = 0.0, th = 0.0, dtau = 0.0;
    if (L.usrc != -2) {
      us = L.usrc == -1 ? L.cval : (L.neg ? -L.u : L.u);
      double src = us;
      if (!alpha_from_u) src = L.usrc == -1 ? L.cval : (L.neg ? -L.up_bc : L.up_bc);
      al = diffusivity(P, src, L.rho);
      iter_params(P, al, L.rho, dtau, th);
      // validity of the diffusivity on owned cells and first-layer ghosts
      const bool track = (tid >= 1 && tid <= OW) || a == -1 || a == ni;
      if (track && r >= j0 - (j0 == 0) && r < j1 + (j1 == nj)) {
        if (!isfinite(al)) bad |= 1;
        if (al < 0.0) bad |= 2;
      }
    }
    sU[s][tid] = us;
    sA[s][tid] = al;
    sT[s][tid] = th;
    sD[s][tid] = dtau;
  };

  // new damped (and undamped) i+1/2 flux of face row r
  auto face_x = [&](int r, double qold) {
    const int s = (r + 3) % 3;
    double qn = 0.0, qp = 0.0;
    if (qx_act_col && r >= 0 && r < nj) {
      const double af = face_mean(mean, sA[s][tid], sA[s][tid + 1]);
      const double tf = face_mean(mean, sT[s][tid], sT[s][tid + 1]);
      const double du = sU[s][tid + 1] - sU[s][tid];
      qn = (qold * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
    }
    sQX[s][tid] = qn;
    sPX[s][tid] = qp;
  };
  // new j+1/2 flux of face row r (between rows r and r+1)
  auto face_y = [&](int r, double qold) {
    const int s0 = (r + 3) % 3, s1 = (r + 4) % 3, sy = (r + 2) % 2;
    double qn = 0.0, qp = 0.0;
    if (qy_act_col && r >= -1 && r <= nj - 1) {
      const double af = face_mean(mean, sA[s0][tid], sA[s1][tid]);
      const double tf = face_mean(mean, sT[s0][tid], sT[s1][tid]);
      const double du = sU[s1][tid] - sU[s0][tid];
      qn = (qold * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
    }
    sQY[sy][tid] = qn;
    sPY[sy][tid] = qp;
    return qn;
  };

  // prologue: rows j0-1 and j0 staged, face row j0-1 (x and y) computed
  RowLoads L0, L1;
  load_row(j0 - 1, L0);
  load_row(j0, L1);
  stage(j0 - 1, L0);
  stage(j0, L1);
  const double qx_j0 = L1.qx;  // old flux of face row j0, used in iteration j0-1's role below
  __syncthreads();
  face_x(j0 - 1, L0.qx);
  face_x(j0, qx_j0);
  {
    const double qn = face_y(j0 - 1, L1.qy);
    if (j0 == 0 && owner) {
      qyout[off2(P, a, -1)] = qn;
      uout[off2(P, a, -1)] = sU[2][tid];  // row -1 ghost after applybcs!
    }
  }
  // the update loads of row j0 come with load_row(j0 + 1)
  RowLoads Ln;
  load_row(j0 + 1, Ln);

  double local = 0.0;
  bool local_nan = false;
  for (int j = j0; j < j1; ++j) {
    RowLoads Lc = Ln;                    // loads for row j+1 (stage) / row j (update)
    if (j + 1 < j1) load_row(j + 2, Ln);  // prefetch the next row
    stage(j + 1, Lc);
    __syncthreads();
    face_x(j + 1, Lc.qx);
    const double qyn = face_y(j, Lc.qy);
    __syncthreads();
    const int sm = (j + 2) % 3, s0 = (j + 3) % 3, sp = (j + 4) % 3;
    const int ym = (j + 1) % 2, y0 = (j + 2) % 2;
    if (owner) {
      const int x = tid;
      const int o = off2(P, a, j);
      const double dq = Lc.g11 * (sQX[s0][x] - sQX[s0][x - 1]) + Lc.g22 * (sQY[y0][x] - sQY[ym][x]) +
                        Lc.c12 * ((sQX[sp][x] + sQX[sp][x - 1]) - (sQX[sm][x] + sQX[sm][x - 1])) +
                        Lc.c12 * ((sQY[y0][x + 1] + sQY[ym][x + 1]) - (sQY[y0][x - 1] + sQY[ym][x - 1])) +
                        Lc.ca * (0.5 * (sQX[s0][x] + sQX[s0][x - 1])) + Lc.cb * (0.5 * (sQY[y0][x] + sQY[ym][x]));
      const double dtau = sD[s0][x];
      // forcing of this cell with the iteration's diffusivity; g12 = 4·c12 exactly
      const double f = TZ ? tz::combine(Lc.tzt, sA[s0][x], Lc.g11, Lc.g22, 4.0 * Lc.c12, Lc.ca, Lc.cb, Lc.S) : 0.0;
      const double un = TZ ? (sU[s0][x] + dtau * (Lc.up / dt - dq + Lc.S + f)) / (1.0 + dtau / dt)
                           : (sU[s0][x] + dtau * (Lc.up / dt - dq + Lc.S)) / (1.0 + dtau / dt);
      uout[o] = un;
      qyout[o] = qyn;
      if (check) {
        const double dqp = Lc.g11 * (sPX[s0][x] - sPX[s0][x - 1]) + Lc.g22 * (sPY[y0][x] - sPY[ym][x]) +
                           Lc.c12 * ((sPX[sp][x] + sPX[sp][x - 1]) - (sPX[sm][x] + sPX[sm][x - 1])) +
                           Lc.c12 * ((sPY[y0][x + 1] + sPY[ym][x + 1]) - (sPY[y0][x - 1] + sPY[ym][x - 1])) +
                           Lc.ca * (0.5 * (sPX[s0][x] + sPX[s0][x - 1])) +
                           Lc.cb * (0.5 * (sPY[y0][x] + sPY[ym][x]));
        double du = un - Lc.up;
        if (isapprox_eps(un, Lc.up)) du = 0.0;
        const double r = TZ ? -du / dt - dqp + Lc.S + f : -du / dt - dqp + Lc.S;
        if (rms) local += r * r;
        else {
          const double ar = fabs(r);
          if (ar != ar) local_nan = true;
          else local = fmax(local, ar);
        }
      }
      // ghost of u after this iteration's applybcs! (copy!(T, u) returns it);
      // the row -1 ghost is written in the prologue
      if (j == nj - 1) uout[off2(P, a, nj)] = sU[sp][x];
    }
    if (qx_own) qxout[off2(P, a, j)] = sQX[s0][tid];
    if (a == -1 || a == ni) uout[off2(P, a, j)] = sU[s0][tid];
  }
  finish_iteration<TX>(P, C, tile, iter, check, local, local_nan, bad, s_red, &s_flag);
}

cudaError_t launch_march2d_fp64(int variant, int tz, const Problem* probs, const int2* items, int nitems,
                                cudaStream_t s) {
  if (nitems <= 0) return cudaSuccess;
  if (tz) {
    if (variant == 0) march2d_fp64<128, true><<<nitems, 128, 0, s>>>(probs, items);
    else march2d_fp64<64, true><<<nitems, 64, 0, s>>>(probs, items);
  } else {
    if (variant == 0) march2d_fp64<128, false><<<nitems, 128, 0, s>>>(probs, items);
    else march2d_fp64<64, false><<<nitems, 64, 0, s>>>(probs, items);
  }
  return cudaGetLastError();
}

}  // namespace cdm
