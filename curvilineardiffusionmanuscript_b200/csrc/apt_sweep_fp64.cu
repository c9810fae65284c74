// apt_sweep_fp64.cu — fused FP64 APT pseudo-iteration for sm_100a.
//
// One launch performs one pseudo-iteration of step! (PseudoTransientSolver.jl:
// 253-319) for every tile of every active problem of a batch:
//
//   applybcs!            boundary_operators.jl:26-263   ghosts filled on the fly
//   update_conductivity! pseudo_transient/conductivity.jl:15-23
//   update_iteration_params! iteration_parameters.jl:2-34
//   compute_flux!        flux/fluxes.jl:5-26, flux/fluxes_gpu.jl:34-129
//   compute_update!      update.jl:2-21 with flux_divergence.jl:7-42 / :119-239
//   update_residual!     residuals.jl:24-47 (check iterations only)
//   L2_norm              residuals.jl:1-22 (block partials + last-block finish)
//
// Each block owns a tile of cells.  It stages the tile plus a one-cell ring of
// u (ghosts from the boundary rules), the diffusivity and the pseudo-time
// parameters in shared memory, computes the new damped fluxes on every face
// the tile's divergence reads (ring faces redundantly, so no other block's
// output is needed), updates u into the other ping-pong buffer and, on check
// iterations, evaluates the residual with the undamped fluxes and reduces
// max|r| (or sum r^2).  The last block of a problem to finish reduces the
// partials and runs the stopping rule of :289-318 on the device.
//
// Reads per cell and iteration: u, q (ndim), u_prev, S, rho and the packed
// metric coefficients; writes u and q.  Diffusivity, pseudo-time parameters,
// q' and r are never stored.
#include "cdm_device.cuh"
#include "cdm_kernels.h"
#include "cdm_finish.cuh"

namespace cdm {

// stage one ring cell: u (with ghost rule), diffusivity and parameters
__device__ __forceinline__ void stage_cell(const Problem& P, const double* __restrict__ uin, int iter,
                                           int a, int b, int c, double& us, double& as, double& ts,
                                           double& ds, int& bad) {
  const int cls = classify(P, a, b, c);
  if (cls < 0) {
    us = 0.0; as = 0.0; ts = 0.0; ds = 0.0;
    return;
  }
  const int64_t id = fidx(P, a, b, c);
  double uval, asrc;
  if (cls == 6) {
    uval = uin[id];
    asrc = (P.subcycle || iter == 1) ? uval : P.u_prev[id];
  } else {
    uval = ghost_value(P, uin, cls, a, b, c);
    asrc = (P.subcycle || iter == 1) ? uval : ghost_value(P, P.u_prev, cls, a, b, c);
  }
  const double rh = P.rho[id];
  const double al = diffusivity(P, asrc, rh);
  double d, t;
  iter_params(P, al, rh, d, t);
  us = uval; as = al; ts = t; ds = d;
  if (!isfinite(al)) bad |= 1;
  if (al < 0.0) bad |= 2;
}

// ---------------------------------------------------------------------------
// 2D: tile TX x TY cells
template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) sweep2d_fp64(const Problem* __restrict__ probs,
                                                   const int2* __restrict__ items) {
  constexpr int RX = TX + 2, RY = TY + 2;
  __shared__ double s_u[RY][RX], s_a[RY][RX], s_t[RY][RX], s_d[RY][RX];
  __shared__ double s_qx[RY][TX + 1], s_qy[TY + 1][RX];
  __shared__ double s_px[RY][TX + 1], s_py[TY + 1][RX];
  __shared__ double s_red[NT / 32];
  __shared__ int s_flag;

  const int2 item = items[blockIdx.x];
  const Problem& P = probs[item.x];
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->done)) return;
  const int iter = ld_cg_int(&C->iter) + 1;
  const bool check = is_check_iter(C, iter);
  const int tid = threadIdx.x;
  const int tile = item.y;
  const int i0 = (tile % P.tiles_i) * TX, j0 = (tile / P.tiles_i) * TY;
  const int pin = (iter - 1) & 1;
  const double* __restrict__ uin = P.u[pin];
  double* __restrict__ uout = P.u[pin ^ 1];
  const int qin = (P.qpar + iter - 1) & 1;
  const double* __restrict__ qxin = P.q[qin][0];
  const double* __restrict__ qyin = P.q[qin][1];
  double* __restrict__ qxout = P.q[qin ^ 1][0];
  double* __restrict__ qyout = P.q[qin ^ 1][1];
  const int ni = P.ni, nj = P.nj;

  // phase 1: ring cells
  int bad = 0;
  for (int r = tid; r < RX * RY; r += NT) {
    const int rb = r / RX, ra = r - rb * RX;
    const int a = i0 - 1 + ra, b = j0 - 1 + rb;
    int bcell = 0;
    stage_cell(P, uin, iter, a, b, 0, s_u[rb][ra], s_a[rb][ra], s_t[rb][ra], s_d[rb][ra], bcell);
    // validity is tracked for tile cells and first-layer ghosts only
    const bool own = (ra >= 1 && ra <= TX && rb >= 1 && rb <= TY) ||
                     ((a == -1 || a == ni) && rb >= 1 && rb <= TY) ||
                     ((b == -1 || b == nj) && ra >= 1 && ra <= TX);
    if (own) bad |= bcell;
  }
  __syncthreads();

  // phase 2: faces.  i+1/2 faces (a in [i0-1, i0+TX-1], b in [j0-1, j0+TY])
  for (int f = tid; f < RY * (TX + 1); f += NT) {
    const int fb = f / (TX + 1), fa = f - fb * (TX + 1);
    const int a = i0 - 1 + fa, b = j0 - 1 + fb;
    double qn = 0.0, qp = 0.0;
    if (a >= -1 && a <= ni - 1 && b >= 0 && b <= nj - 1) {
      const int64_t id = fidx(P, a, b);
      const double af = face_mean(P.mean, s_a[fb][fa], s_a[fb][fa + 1]);
      const double tf = face_mean(P.mean, s_t[fb][fa], s_t[fb][fa + 1]);
      const double du = s_u[fb][fa + 1] - s_u[fb][fa];
      qn = (qxin[id] * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
      if (fb >= 1 && fb <= TY && (fa >= 1 || a == -1)) qxout[id] = qn;
    }
    s_qx[fb][fa] = qn;
    s_px[fb][fa] = qp;
  }
  // j+1/2 faces (a in [i0-1, i0+TX], b in [j0-1, j0+TY-1])
  for (int f = tid; f < (TY + 1) * RX; f += NT) {
    const int fb = f / RX, fa = f - fb * RX;
    const int a = i0 - 1 + fa, b = j0 - 1 + fb;
    double qn = 0.0, qp = 0.0;
    if (a >= 0 && a <= ni - 1 && b >= -1 && b <= nj - 1) {
      const int64_t id = fidx(P, a, b);
      const double af = face_mean(P.mean, s_a[fb][fa], s_a[fb + 1][fa]);
      const double tf = face_mean(P.mean, s_t[fb][fa], s_t[fb + 1][fa]);
      const double du = s_u[fb + 1][fa] - s_u[fb][fa];
      qn = (qyin[id] * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
      if (fa >= 1 && fa <= TX && (fb >= 1 || b == -1)) qyout[id] = qn;
    }
    s_qy[fb][fa] = qn;
    s_py[fb][fa] = qp;
  }
  __syncthreads();

  // phase 3: cell update (+ residual)
  const double dt = P.dt;
  const double* __restrict__ g11 = P.coef[0];
  const double* __restrict__ g22 = P.coef[1];
  const double* __restrict__ c12 = P.coef[2];
  const double* __restrict__ cal = P.coef[3];
  const double* __restrict__ cbe = P.coef[4];
  double local = 0.0;
  bool local_nan = false;
  const bool rms = C->norm_kind == 1;
  for (int e = tid; e < TX * TY; e += NT) {
    const int cb = e / TX, ca = e - cb * TX;
    const int a = i0 + ca, b = j0 + cb;
    if (a >= ni || b >= nj) continue;
    const int64_t id = fidx(P, a, b);
    const int x = ca + 1, y = cb + 1;
    // flux_divergence.jl:7-42 on the new damped fluxes
    const double G11 = g11[id], G22 = g22[id], C12 = c12[id], CA = cal[id], CB = cbe[id];
    const double dq = G11 * (s_qx[y][x] - s_qx[y][x - 1]) + G22 * (s_qy[y][x] - s_qy[y - 1][x]) +
                      C12 * ((s_qx[y + 1][x] + s_qx[y + 1][x - 1]) - (s_qx[y - 1][x] + s_qx[y - 1][x - 1])) +
                      C12 * ((s_qy[y][x + 1] + s_qy[y - 1][x + 1]) - (s_qy[y][x - 1] + s_qy[y - 1][x - 1])) +
                      CA * (0.5 * (s_qx[y][x] + s_qx[y][x - 1])) + CB * (0.5 * (s_qy[y][x] + s_qy[y - 1][x]));
    const double up = P.u_prev[id], S = P.S[id];
    const double dtau = s_d[y][x];
    // update.jl:13-15
    const double un = (s_u[y][x] + dtau * (up / dt - dq + S)) / (1.0 + dtau / dt);
    uout[id] = un;
    // ghosts of u after applybcs! of this iteration (copy!(T, u) returns them)
    if (a == 0) uout[fidx(P, -1, b)] = s_u[y][0];
    if (a == ni - 1) uout[fidx(P, ni, b)] = s_u[y][x + 1];
    if (b == 0) uout[fidx(P, a, -1)] = s_u[0][x];
    if (b == nj - 1) uout[fidx(P, a, nj)] = s_u[y + 1][x];
    if (check) {
      // residuals.jl:36-46 with the undamped fluxes of this iteration
      const double dqp = G11 * (s_px[y][x] - s_px[y][x - 1]) + G22 * (s_py[y][x] - s_py[y - 1][x]) +
                         C12 * ((s_px[y + 1][x] + s_px[y + 1][x - 1]) - (s_px[y - 1][x] + s_px[y - 1][x - 1])) +
                         C12 * ((s_py[y][x + 1] + s_py[y - 1][x + 1]) - (s_py[y][x - 1] + s_py[y - 1][x - 1])) +
                         CA * (0.5 * (s_px[y][x] + s_px[y][x - 1])) + CB * (0.5 * (s_py[y][x] + s_py[y - 1][x]));
      double du = un - up;
      if (isapprox_eps(un, up)) du = 0.0;
      const double r = -du / dt - dqp + S;
      if (rms) local += r * r;
      else {
        const double ar = fabs(r);
        if (ar != ar) local_nan = true;
        else local = fmax(local, ar);
      }
    }
  }
  finish_iteration<NT>(P, C, tile, iter, check, local, local_nan, bad, s_red, &s_flag);
}

// ---------------------------------------------------------------------------
// 3D: tile TX x TY x TZ cells, dynamic shared memory
template <int TX, int TY, int TZ>
struct Smem3 {
  static constexpr int RX = TX + 2, RY = TY + 2, RZ = TZ + 2;
  static constexpr int NR = RX * RY * RZ;
  static constexpr int NQI = RZ * RY * (TX + 1);
  static constexpr int NQJ = RZ * (TY + 1) * RX;
  static constexpr int NQK = (TZ + 1) * RY * RX;
  static constexpr size_t bytes = sizeof(double) * (4 * NR + 2 * (NQI + NQJ + NQK));
};

template <int TX, int TY, int TZ, int NT>
__global__ void __launch_bounds__(NT) sweep3d_fp64(const Problem* __restrict__ probs,
                                                   const int2* __restrict__ items) {
  using SM = Smem3<TX, TY, TZ>;
  constexpr int RX = SM::RX, RY = SM::RY;
  extern __shared__ double smem[];
  double* s_u = smem;
  double* s_a = s_u + SM::NR;
  double* s_t = s_a + SM::NR;
  double* s_d = s_t + SM::NR;
  double* s_qi = s_d + SM::NR;
  double* s_qj = s_qi + SM::NQI;
  double* s_qk = s_qj + SM::NQJ;
  double* s_pi = s_qk + SM::NQK;
  double* s_pj = s_pi + SM::NQI;
  double* s_pk = s_pj + SM::NQJ;
  __shared__ double s_red[NT / 32];
  __shared__ int s_flag;
  auto R = [](int x, int y, int z) { return x + RX * (y + RY * z); };
  auto QI = [](int x, int y, int z) { return x + (TX + 1) * (y + RY * z); };
  auto QJ = [](int x, int y, int z) { return x + RX * (y + (TY + 1) * z); };
  auto QK = [](int x, int y, int z) { return x + RX * (y + RY * z); };

  const int2 item = items[blockIdx.x];
  const Problem& P = probs[item.x];
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->done)) return;
  const int iter = ld_cg_int(&C->iter) + 1;
  const bool check = is_check_iter(C, iter);
  const int tid = threadIdx.x;
  const int tile = item.y;
  const int ti = tile % P.tiles_i, tj = (tile / P.tiles_i) % P.tiles_j, tk = tile / (P.tiles_i * P.tiles_j);
  const int i0 = ti * TX, j0 = tj * TY, k0 = tk * TZ;
  const int pin = (iter - 1) & 1;
  const double* __restrict__ uin = P.u[pin];
  double* __restrict__ uout = P.u[pin ^ 1];
  const int qin = (P.qpar + iter - 1) & 1;
  const double* qiin = P.q[qin][0];
  const double* qjin = P.q[qin][1];
  const double* qkin = P.q[qin][2];
  double* qiout = P.q[qin ^ 1][0];
  double* qjout = P.q[qin ^ 1][1];
  double* qkout = P.q[qin ^ 1][2];
  const int ni = P.ni, nj = P.nj, nk = P.nk;

  int bad = 0;
  for (int r = tid; r < SM::NR; r += NT) {
    const int rz = r / (RX * RY), rem = r - rz * RX * RY, ry = rem / RX, rx = rem - ry * RX;
    const int a = i0 - 1 + rx, b = j0 - 1 + ry, c = k0 - 1 + rz;
    int bcell = 0;
    stage_cell(P, uin, iter, a, b, c, s_u[r], s_a[r], s_t[r], s_d[r], bcell);
    const bool inx = rx >= 1 && rx <= TX, iny = ry >= 1 && ry <= TY, inz = rz >= 1 && rz <= TZ;
    const bool own = (inx && iny && inz) || ((a == -1 || a == ni) && iny && inz) ||
                     ((b == -1 || b == nj) && inx && inz) || ((c == -1 || c == nk) && inx && iny);
    if (own) bad |= bcell;
  }
  __syncthreads();

  // i+1/2 faces: a in [i0-1, i0+TX-1], b in [j0-1, j0+TY], c in [k0-1, k0+TZ]
  for (int f = tid; f < SM::NQI; f += NT) {
    const int z = f / ((TX + 1) * RY), rem = f - z * (TX + 1) * RY, y = rem / (TX + 1), x = rem - y * (TX + 1);
    const int a = i0 - 1 + x, b = j0 - 1 + y, c = k0 - 1 + z;
    double qn = 0.0, qp = 0.0;
    if (a >= -1 && a <= ni - 1 && b >= 0 && b <= nj - 1 && c >= 0 && c <= nk - 1) {
      const int64_t id = fidx(P, a, b, c);
      const int r0 = R(x, y, z), r1 = R(x + 1, y, z);
      const double af = face_mean(P.mean, s_a[r0], s_a[r1]);
      const double tf = face_mean(P.mean, s_t[r0], s_t[r1]);
      const double du = s_u[r1] - s_u[r0];
      qn = (qiin[id] * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
      if (y >= 1 && y <= TY && z >= 1 && z <= TZ && (x >= 1 || a == -1)) qiout[id] = qn;
    }
    s_qi[f] = qn;
    s_pi[f] = qp;
  }
  // j+1/2 faces: a in [i0-1, i0+TX], b in [j0-1, j0+TY-1], c in [k0-1, k0+TZ]
  for (int f = tid; f < SM::NQJ; f += NT) {
    const int z = f / (RX * (TY + 1)), rem = f - z * RX * (TY + 1), y = rem / RX, x = rem - y * RX;
    const int a = i0 - 1 + x, b = j0 - 1 + y, c = k0 - 1 + z;
    double qn = 0.0, qp = 0.0;
    if (a >= 0 && a <= ni - 1 && b >= -1 && b <= nj - 1 && c >= 0 && c <= nk - 1) {
      const int64_t id = fidx(P, a, b, c);
      const int r0 = R(x, y, z), r1 = R(x, y + 1, z);
      const double af = face_mean(P.mean, s_a[r0], s_a[r1]);
      const double tf = face_mean(P.mean, s_t[r0], s_t[r1]);
      const double du = s_u[r1] - s_u[r0];
      qn = (qjin[id] * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
      if (x >= 1 && x <= TX && z >= 1 && z <= TZ && (y >= 1 || b == -1)) qjout[id] = qn;
    }
    s_qj[f] = qn;
    s_pj[f] = qp;
  }
  // k+1/2 faces: a in [i0-1, i0+TX], b in [j0-1, j0+TY], c in [k0-1, k0+TZ-1]
  for (int f = tid; f < SM::NQK; f += NT) {
    const int z = f / (RX * RY), rem = f - z * RX * RY, y = rem / RX, x = rem - y * RX;
    const int a = i0 - 1 + x, b = j0 - 1 + y, c = k0 - 1 + z;
    double qn = 0.0, qp = 0.0;
    if (a >= 0 && a <= ni - 1 && b >= 0 && b <= nj - 1 && c >= -1 && c <= nk - 1) {
      const int64_t id = fidx(P, a, b, c);
      const int r0 = R(x, y, z), r1 = R(x, y, z + 1);
      const double af = face_mean(P.mean, s_a[r0], s_a[r1]);
      const double tf = face_mean(P.mean, s_t[r0], s_t[r1]);
      const double du = s_u[r1] - s_u[r0];
      qn = (qkin[id] * tf + (-af * du)) / (1.0 + tf);
      qp = -af * du;
      if (x >= 1 && x <= TX && y >= 1 && y <= TY && (z >= 1 || c == -1)) qkout[id] = qn;
    }
    s_qk[f] = qn;
    s_pk[f] = qp;
  }
  __syncthreads();

  const double dt = P.dt;
  double local = 0.0;
  bool local_nan = false;
  const bool rms = C->norm_kind == 1;
  for (int e = tid; e < TX * TY * TZ; e += NT) {
    const int cz = e / (TX * TY), rem = e - cz * TX * TY, cy = rem / TX, cx = rem - cy * TX;
    const int a = i0 + cx, b = j0 + cy, c = k0 + cz;
    if (a >= ni || b >= nj || c >= nk) continue;
    const int64_t id = fidx(P, a, b, c);
    const int x = cx + 1, y = cy + 1, z = cz + 1;
    const double G11 = P.coef[0][id], G22 = P.coef[1][id], G33 = P.coef[2][id];
    const double Cxe = P.coef[3][id], Cez = P.coef[4][id], Cxz = P.coef[5][id];
    const double CA = P.coef[6][id], CB = P.coef[7][id], CC = P.coef[8][id];
    // flux_divergence.jl:119-239; q_i at face (x', y', z') -> QI(x', y', z') with x' = face i-index + 1
    auto div = [&](const double* qi, const double* qj, const double* qk) -> double {
      const double t_ii = G11 * (qi[QI(x, y, z)] - qi[QI(x - 1, y, z)]);
      const double t_jj = G22 * (qj[QJ(x, y, z)] - qj[QJ(x, y - 1, z)]);
      const double t_kk = G33 * (qk[QK(x, y, z)] - qk[QK(x, y, z - 1)]);
      const double qi_eta = Cxe * (0.5 * (qi[QI(x, y + 1, z)] + qi[QI(x - 1, y + 1, z)]) -
                                   0.5 * (qi[QI(x, y - 1, z)] + qi[QI(x - 1, y - 1, z)]));
      const double qj_xi = Cxe * (0.5 * (qj[QJ(x + 1, y, z)] + qj[QJ(x + 1, y - 1, z)]) -
                                  0.5 * (qj[QJ(x - 1, y, z)] + qj[QJ(x - 1, y - 1, z)]));
      const double qj_zeta = Cez * (0.5 * (qj[QJ(x, y, z + 1)] + qj[QJ(x, y - 1, z + 1)]) -
                                    0.5 * (qj[QJ(x, y, z - 1)] + qj[QJ(x, y - 1, z - 1)]));
      const double qk_eta = Cez * (0.5 * (qk[QK(x, y + 1, z)] + qk[QK(x, y + 1, z - 1)]) -
                                   0.5 * (qk[QK(x, y - 1, z)] + qk[QK(x, y - 1, z - 1)]));
      const double qi_zeta = Cxz * (0.5 * (qi[QI(x, y, z + 1)] + qi[QI(x - 1, y, z + 1)]) -
                                    0.5 * (qi[QI(x, y, z - 1)] + qi[QI(x - 1, y, z - 1)]));
      const double qk_xi = Cxz * (0.5 * (qk[QK(x + 1, y, z)] + qk[QK(x + 1, y, z - 1)]) -
                                  0.5 * (qk[QK(x - 1, y, z)] + qk[QK(x - 1, y, z - 1)]));
      const double h_a = CA * (0.5 * (qi[QI(x, y, z)] + qi[QI(x - 1, y, z)]));
      const double h_b = CB * (0.5 * (qj[QJ(x, y, z)] + qj[QJ(x, y - 1, z)]));
      const double h_c = CC * (0.5 * (qk[QK(x, y, z)] + qk[QK(x, y, z - 1)]));
      return t_ii + t_jj + t_kk + qi_eta + qi_zeta + qj_xi + qj_zeta + qk_eta + qk_xi + h_a + h_b + h_c;
    };
    const double dq = div(s_qi, s_qj, s_qk);
    const double up = P.u_prev[id], S = P.S[id];
    const int rc = R(x, y, z);
    const double dtau = s_d[rc];
    const double un = (s_u[rc] + dtau * (up / dt - dq + S)) / (1.0 + dtau / dt);
    uout[id] = un;
    if (a == 0) uout[fidx(P, -1, b, c)] = s_u[R(0, y, z)];
    if (a == ni - 1) uout[fidx(P, ni, b, c)] = s_u[R(x + 1, y, z)];
    if (b == 0) uout[fidx(P, a, -1, c)] = s_u[R(x, 0, z)];
    if (b == nj - 1) uout[fidx(P, a, nj, c)] = s_u[R(x, y + 1, z)];
    if (c == 0) uout[fidx(P, a, b, -1)] = s_u[R(x, y, 0)];
    if (c == nk - 1) uout[fidx(P, a, b, nk)] = s_u[R(x, y, z + 1)];
    if (check) {
      const double dqp = div(s_pi, s_pj, s_pk);
      double du = un - up;
      if (isapprox_eps(un, up)) du = 0.0;
      const double r = -du / dt - dqp + S;
      if (rms) local += r * r;
      else {
        const double ar = fabs(r);
        if (ar != ar) local_nan = true;
        else local = fmax(local, ar);
      }
    }
  }
  finish_iteration<NT>(P, C, tile, iter, check, local, local_nan, bad, s_red, &s_flag);
}

// ---------------------------------------------------------------------------
// tile shape table (the autotuner picks among these)
static const TileShape kShapes2D[] = {
    {128, 0, 0, 128, 1}, {64, 0, 0, 64, 1}, {32, 16, 1, 256, 0}, {32, 8, 1, 256, 0}, {128, 0, 0, 128, 3},
    {64, 0, 0, 64, 3},
};
// 3D: variants 0 and 3 are the plane-marching kernel (reciprocal form) on
// 32 x 8 and 16 x 16 column tiles; the tile kernels (1, 2) keep the
// operation-for-operation form
static const TileShape kShapes3D[] = {
    {32, 8, 1, 256, 2}, {32, 4, 4, 256, 0}, {16, 8, 4, 256, 0}, {16, 16, 1, 256, 2},
};

int num_tile_shapes(int ndim) { return ndim == 2 ? 6 : 4; }
TileShape tile_shape(int ndim, int v) { return ndim == 2 ? kShapes2D[v] : kShapes3D[v]; }

template <int TX, int TY, int TZ, int NT>
static cudaError_t launch3(const Problem* probs, const int2* items, int nitems, cudaStream_t s) {
  const size_t bytes = Smem3<TX, TY, TZ>::bytes;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(sweep3d_fp64<TX, TY, TZ, NT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  sweep3d_fp64<TX, TY, TZ, NT><<<nitems, NT, bytes, s>>>(probs, items);
  return cudaGetLastError();
}

cudaError_t launch_sweep_fp64(int ndim, int variant, int exact, int harmonic, const Problem* probs,
                              const int2* items, int nitems, int n_edge, unsigned int* counters,
                              const SweepStreams& ss, int tz) {
  if (nitems <= 0) return cudaSuccess;
  cudaStream_t s = ss.main;
  if (ndim == 2) {
    switch (variant) {
      case 0:
      case 1:
        if (exact || tz) return launch_march2d_fp64(variant, tz, probs, items, nitems, s);
        return launch_march2d_fast(variant, harmonic, probs, items, n_edge, nitems - n_edge, counters, ss);
      case 4:  // the wavefront variants launch through launch_march2d_wave (tagged items)
      case 5:
        return cudaErrorInvalidValue;
      case 2: sweep2d_fp64<32, 16, 256><<<nitems, 256, 0, s>>>(probs, items); break;
      default: sweep2d_fp64<32, 8, 256><<<nitems, 256, 0, s>>>(probs, items); break;
    }
    return cudaGetLastError();
  }
  switch (variant) {
    case 0:
    case 3: {
      const TileShape ts = kShapes3D[variant];
      return launch_march3d_fast(harmonic, ts.tx, ts.ty, probs, items, n_edge, nitems - n_edge, ss);
    }
    case 1: return launch3<32, 4, 4, 256>(probs, items, nitems, s);
    default: return launch3<16, 8, 4, 256>(probs, items, nitems, s);
  }
}

}  // namespace cdm
