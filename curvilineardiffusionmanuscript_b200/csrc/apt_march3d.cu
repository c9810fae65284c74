// apt_march3d.cu — plane-marching FP64 APT pseudo-iteration in 3D, reciprocal form.
//
// The iteration of step! (PseudoTransientSolver.jl:253-319) with the 3D flux
// divergence of flux_divergence.jl:119-239, in the reciprocal ("fast") form of
// apt_march2d_fast.cu: the same discrete iteration as the operation-for-
// operation tile kernel (sweep3d_fp64), last-bit differences only.
//
// Organisation: a block of 256 threads owns a 32 x 8 column of cells in (i, j)
// and marches a strip of k-planes.  Each thread owns one (i, j) position and
// keeps its own cell's update factors in registers; 84 threads also stage one
// cell of the one-cell (i, j) ring.  Shared memory holds two staged cell planes
// (u, α⁻¹ or α, θ⁻¹ or θ), three planes of i- and j-face fluxes and two planes
// of k-face fluxes (damped, and undamped on check iterations): the divergence
// of plane z reads the i/j fluxes of planes z-1, z, z+1 and the k fluxes below
// and above it.  Every face is computed once per strip; the ring costs 1.33x
// the owned cells per plane and nothing along k.  Ghost cells come from the
// boundary rules of every side applied on the fly (boundary_operators.jl).
//
// Both kinds of tile issue the loads that stage plane z + 2 (u, ρ, uⁿ) while
// plane z is updated, so that their latency overlaps a whole plane of work,
// and resolve the k-ghost planes once per plane (block-uniform).  Two
// instantiations: the interior one, for tiles whose cells and ring are all
// domain cells in (i, j), and EDGE, for tiles whose ring touches the (i, j)
// boundary, where every thread resolves its own and its ring cell's column
// once per strip (a domain column, an i- or j-ghost column with its side's
// rule, or no cell) and which adds the domain-range tests of partial tiles,
// the boundary-face writes and the ghost writes of the update.  The two run as
// concurrent launches.
#include "cdm_device.cuh"
#include "cdm_fast.cuh"
#include "cdm_finish.cuh"
#include "cdm_kernels.h"

namespace cdm {

namespace {

using fastmath::pow_fast;
using fastmath::rcp_nr;
using fastmath::rcp_pos;

// column tile of TX x TY cells, one thread per column; RX x RY with the ring
template <int TX, int TY>
struct M3Smem {
  static constexpr int RX = TX + 2, RY = TY + 2, NT = TX * TY;
  double U[2][RY][RX], IA[2][RY][RX], IT[2][RY][RX];  // staged cells of planes z, z+1
  double QI[3][RY][TX + 1], QJ[3][TY + 1][RX], QK[2][RY][RX];  // new damped fluxes
  double PI[3][RY][TX + 1], PJ[3][TY + 1][RX], PK[2][RY][RX];  // undamped (check iterations)
  double red[NT / 32];
  int flag;
};

struct C3 {
  double u, ia, it, g, f;
};

}  // namespace

template <bool HARM, bool EDGE, int TX, int TY>
__global__ void __launch_bounds__(TX * TY, 2) march3d_fast(const Problem* __restrict__ probs,
                                                           const int2* __restrict__ items) {
  constexpr int NT = TX * TY, RX = TX + 2, RY = TY + 2;
  constexpr int NRING = RX * RY - NT;  // ring cells per plane (84 for 32 x 8, 68 for 16 x 16)
  static_assert(NRING <= NT, "one ring cell per thread at most");
  using Smem = M3Smem<TX, TY>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int2 item = items[blockIdx.x];
  __shared__ __align__(16) Problem sP;
  stage_problem<NT>(sP, probs + item.x);
  const Problem& P = sP;
  Ctrl* C = P.ctrl;
  if (ld_cg_int(&C->done)) return;
  const int iter = ld_cg_int(&C->iter) + 1;
  const bool check = is_check_iter(C, iter);
  const int tid = threadIdx.x;
  const int tile = item.y;
  const int ti = tile % P.tiles_i, tj = (tile / P.tiles_i) % P.tiles_j, sk = tile / (P.tiles_i * P.tiles_j);
  const int ni = P.ni, nj = P.nj, nk = P.nk;
  const int i0 = ti * TX, j0 = tj * TY;
  const int k0 = sk * P.strip_h, k1 = min(k0 + P.strip_h, nk);
  const int pin = (iter - 1) & 1;
  const double* __restrict__ uin = P.u[pin];
  double* __restrict__ uout = P.u[pin ^ 1];
  const int qin = (P.qpar + iter - 1) & 1;
  const double* __restrict__ qiin = P.q[qin][0];
  const double* __restrict__ qjin = P.q[qin][1];
  const double* __restrict__ qkin = P.q[qin][2];
  double* __restrict__ qiout = P.q[qin ^ 1][0];
  double* __restrict__ qjout = P.q[qin ^ 1][1];
  double* __restrict__ qkout = P.q[qin ^ 1][2];
  const bool alpha_from_u = P.subcycle || iter == 1;
  const bool rms = C->norm_kind == 1;
  const double dt = P.dt, cp = P.cp, k0c = P.k0;
  const double inv_dt = 1.0 / dt;
  const double LLdt = P.LL / dt, VpL = P.VpL, LoVp = P.L / P.Vpdtau, VpoL = P.Vpdtau / P.L;
  const int kmode = P.kmode, km = P.km, khalf = P.khalf;
  const double kn = P.kn;

  // own (i, j) position in ring coordinates, and this thread's ring cell
  const int ox = tid % TX + 1, oy = tid / TX + 1;
  const int oa = i0 + ox - 1, ob = j0 + oy - 1;
  const bool own_in = EDGE ? (oa < ni && ob < nj) : true;
  int rx = -1, ry = -1;
  if (tid < NRING) {
    if (tid < RX) {
      rx = tid;
      ry = 0;
    } else if (tid < 2 * RX) {
      rx = tid - RX;
      ry = RY - 1;
    } else {
      const int t = tid - 2 * RX;  // 0 .. 2(RY-2)-1
      rx = (t & 1) ? RX - 1 : 0;
      ry = 1 + (t >> 1);
    }
  }
  const int ra = i0 + rx - 1, rb = j0 + ry - 1;

  int bad = 0;
  // validity bits of α: read for a step's last iteration only (a check iteration or the one past max_iter)
  const bool track_iter = check || iter > C->max_iter;
  // raw loads of a cell of plane c (u and uⁿ from the cell the ghost rules
  // read, ρ of the cell itself), issued a plane ahead of stage_pre; mode: 0
  // copy, 1 negate, 2 constant (the value already in u and up), 3 no cell (a
  // corner ghost or a position outside the ghost layer: staged as zeros)
  struct Pre3 {
    double u, rho, up;
    int mode;
  };
  const int64_t plane_sz = (int64_t)P.nx * P.ny;
  const int64_t own_col = fidx(P, oa, ob, 0);
  const int64_t ring_col = rx >= 0 ? fidx(P, ra, rb, 0) : own_col;
  // (i, j) source of a cell's column, fixed for the strip: kind 0 a domain
  // column (the k-ghost rule of each plane applies), 1 / 2 / 3 a first-layer i-
  // or j-ghost column whose side's rule copies / negates the column at `off`
  // or is the side's constant (boundary_operators.jl), 4 neither; the side
  // sits in bits 3 and up.  Interior tiles have domain columns only.
  struct ColSrc {
    int64_t off;
    int code;
  };
  auto col_src = [&](int a, int b) -> ColSrc {
    ColSrc r{0, 0};
    if (!EDGE) return r;
    const bool ia = a >= 0 && a < ni, ib = b >= 0 && b < nj;
    if (ia && ib) return r;
    int side = -1;
    if (ib && (a == -1 || a == ni)) side = a < 0 ? 0 : 1;
    else if (ia && (b == -1 || b == nj)) side = b < 0 ? 2 : 3;
    r.code = 4;
    if (side < 0) return r;
    const int rule = P.rule[side];
    if (rule == GR_DIRICHLET) {
      r.code = 3 | (side << 3);
      return r;
    }
    const bool lo = (side & 1) == 0;
    const int n = side < 2 ? ni : nj;
    const int pos = rule == GR_NONE ? (lo ? -1 : n) : rule == GR_PERIODIC ? (lo ? n - 1 : 0) : (lo ? 0 : n - 1);
    r.off = side < 2 ? fidx(P, pos, b, 0) : fidx(P, a, pos, 0);
    r.code = rule == GR_NEGSYM ? 2 : 1;
    return r;
  };
  const ColSrc own_src = col_src(oa, ob);
  const ColSrc ring_src = rx >= 0 ? col_src(ra, rb) : ColSrc{0, 4};
  // k-ghost rule of plane c (block-uniform): source plane, 1 negate, 2 constant
  auto kplane = [&](int c, int& cs, int& mode, double& cv) {
    cs = c;
    mode = 0;
    cv = 0.0;
    if (c >= 0 && c < nk) return;
    const int side = c < 0 ? 4 : 5;
    const int rule = P.rule[side];
    const bool lo = side == 4;
    if (rule == GR_DIRICHLET) {
      mode = 2;
      cv = P.val[side];
    } else if (rule == GR_PERIODIC) {
      cs = lo ? nk - 1 : 0;
    } else if (rule != GR_NONE) {
      cs = lo ? 0 : nk - 1;
      mode = rule == GR_NEGSYM ? 1 : 0;
    }
  };
  auto load_cell = [&](const ColSrc& cd, int64_t col, int c, int cs, int kmode, double kcv, Pre3& L) {
    const int kind = cd.code & 7;
    if (kind == 0) {
      L.mode = kmode;
      L.rho = P.rho[col + plane_sz * c];
      L.u = kmode == 2 ? kcv : uin[col + plane_sz * cs];
      L.up = (!alpha_from_u && kmode != 2) ? P.u_prev[col + plane_sz * cs] : kcv;
    } else if (kind == 4 || c < 0 || c >= nk) {
      L.mode = 3;
    } else {
      L.mode = kind == 3 ? 2 : kind - 1;
      const double val = kind == 3 ? P.val[cd.code >> 3] : 0.0;
      L.rho = P.rho[col + plane_sz * c];
      L.u = L.mode == 2 ? val : uin[cd.off + plane_sz * c];
      L.up = (!alpha_from_u && L.mode != 2) ? P.u_prev[cd.off + plane_sz * c] : val;
    }
  };
  // the loads of plane c; `mode` returns the plane's k rule (the mode of every
  // cell of an interior tile)
  auto prefetch = [&](int c, Pre3& own, Pre3& rg, int& mode) {
    int cs;
    double cv;
    kplane(c, cs, mode, cv);
    load_cell(own_src, own_col, c, cs, mode, cv, own);
    if (rx >= 0) load_cell(ring_src, ring_col, c, cs, mode, cv, rg);
  };
  // the diffusivity, pseudo-time parameters and update factors from raw loads
  // (iteration_parameters.jl:2-15 in reciprocal form)
  auto stage_pre = [&](const Pre3& L, int mode, bool track) -> C3 {
    C3 r{0.0, 0.0, 0.0, 0.0, 0.0};
    if (EDGE && mode == 3) return r;
    const double u = mode == 1 ? -L.u : L.u;
    const double src = alpha_from_u ? u : (mode == 1 ? -L.up : L.up);
    const double rho = L.rho;
    const double kap = isfinite(src) ? k0c * pow_fast(fabs(src), kmode, km, khalf, kn) : 0.0;
    const double rc = rho * cp;
    const double inva = rc * rcp_nr(kap);
    const double Re = kPi + sqrt(kPi * kPi + LLdt * rho * inva);
    r.u = u;
    if (HARM) {
      // g = Δt·Re/D, f = Vp·L·α⁻¹·Δt/D with D = Δt·Re + Vp·L·α⁻¹ (one reciprocal);
      // a cell whose dτ is not finite (κ = 0) keeps its value
      const double VA = VpL * inva;
      const double dRe = dt * Re;
      const double D = dRe + VA;
      const bool fin = isfinite(D);
      const double iD = rcp_pos(fin ? D : 1.0);
      r.g = fin ? dRe * iD : 1.0;
      r.f = fin ? VA * dt * iD : 0.0;
      r.ia = inva;
      r.it = VpoL * Re;
    } else {
      const double iRe = rcp_nr(Re);
      double dtau = VpL * inva * iRe;
      double th = LoVp * iRe;
      dtau = isfinite(dtau) ? dtau : 0.0;
      th = isfinite(th) ? th : 0.0;
      const double idd = rcp_nr(dt + dtau);
      r.g = dt * idd;
      r.f = dtau * dt * idd;
      r.ia = kap * rcp_nr(rc);
      r.it = th;
    }
    // validity of α = κ/(ρcₚ) on owned cells and first-layer ghosts
    if (track && track_iter) {
      if (!(isfinite(kap) && isfinite(rc) && rc != 0.0)) bad |= 1;
      if (kap != 0.0 && ((kap < 0.0) != (rc < 0.0))) bad |= 2;
    }
    return r;
  };
  auto publish = [&](int s, const C3& own, const C3& rg) {
    sm.U[s][oy][ox] = own.u;
    sm.IA[s][oy][ox] = own.ia;
    sm.IT[s][oy][ox] = own.it;
    if (rx >= 0) {
      sm.U[s][ry][rx] = rg.u;
      sm.IA[s][ry][rx] = rg.ia;
      sm.IT[s][ry][rx] = rg.it;
    }
  };
  // stage plane c into cell slot s from loads prefetched earlier; `mode` is the
  // plane's k rule, every cell's mode on interior tiles
  auto stage_plane_pre = [&](int c, int s, const Pre3& own_l, const Pre3& rg_l, int mode) -> C3 {
    const bool inz = c >= k0 && c < k1;
    const C3 own = stage_pre(own_l, EDGE ? own_l.mode : mode, inz || c == -1 || c == nk);
    const C3 rg = rx >= 0 ? stage_pre(rg_l, EDGE ? rg_l.mode : mode, inz) : C3{0.0, 0.0, 0.0, 0.0, 0.0};
    publish(s, own, rg);
    return own;
  };
  // stage plane c into cell slot s: the own cell (returned) and the ring cell
  auto stage_plane = [&](int c, int s) -> C3 {
    Pre3 lo, lr;
    int mode;
    prefetch(c, lo, lr, mode);
    return stage_plane_pre(c, s, lo, lr, mode);
  };
  auto flux = [&](double ia0, double ia1, double it0, double it1, double du, double qold, double& qp) -> double {
    if (HARM) {
      // (2qA − 2Δu·S_θ)/(A(S_θ + 2)) and −2Δu(S_θ + 2)/(A(S_θ + 2)) over one
      // reciprocal, A = α⁻¹ₐ + α⁻¹_b; θ̄ = 0 (S_θ infinite): q ← −ᾱΔu
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
  // Face assignment, fixed for the whole strip: every thread computes the i-, j-
  // and k-faces on the high side of its own cell (face slots x = ox, y = oy);
  // NRI + NRJ + NRK threads compute one face of the ring each: the i-faces of
  // column x = 0 and of rows y = 0, RY-1; the j-faces of row y = 0 and of
  // columns x = 0, RX-1; the k-faces of the ring cells.  Per plane only the
  // plane offset and the plane's bounds change.
  constexpr int NRI = RY + 2 * TX, NRJ = RX + 2 * TY, NRK = 2 * RX + 2 * TY;
  // each kind starts on a warp boundary, so that no warp computes two kinds
  constexpr int BJ = (NRI + 31) / 32 * 32, BK = BJ + (NRJ + 31) / 32 * 32;
  static_assert(BK + NRK <= NT, "ring faces fit the block");
  int fk = -1, fx = 0, fy = 0;
  if (tid < NRI) {
    fk = 0;
    if (tid < RY) {
      fy = tid;
    } else {
      const int t = tid - RY;
      fy = t < TX ? 0 : RY - 1;
      fx = 1 + (t < TX ? t : t - TX);
    }
  } else if (tid >= BJ && tid < BJ + NRJ) {
    fk = 1;
    const int t = tid - BJ;
    if (t < RX) {
      fx = t;
    } else {
      const int u = t - RX;
      fx = (u & 1) ? RX - 1 : 0;
      fy = 1 + (u >> 1);
    }
  } else if (tid >= BK && tid < BK + NRK) {
    fk = 2;
    const int t = tid - BK;
    if (t < 2 * RX) {
      fy = t < RX ? 0 : RY - 1;
      fx = t < RX ? t : t - RX;
    } else {
      const int u = t - 2 * RX;
      fx = (u & 1) ? RX - 1 : 0;
      fy = 1 + (u >> 1);
    }
  }
  const int fa = i0 - 1 + fx, fb = j0 - 1 + fy;
  // the ring face's (a, b) range test (faces.jl ranges: an i-face joins cells a and a+1, ...)
  const bool f_ab = !EDGE ? fk >= 0
                    : fk == 0 ? (fa >= -1 && fa <= ni - 1 && fb >= 0 && fb <= nj - 1)
                    : fk == 1 ? (fa >= 0 && fa <= ni - 1 && fb >= -1 && fb <= nj - 1)
                              : (fa >= 0 && fa <= ni - 1 && fb >= 0 && fb <= nj - 1);
  // ring i-faces of column 0 and j-faces of row 0 are the domain's low boundary faces
  const bool f_wr = EDGE && ((fk == 0 && fx == 0 && i0 == 0 && fy >= 1 && fy <= TY) ||
                             (fk == 1 && fy == 0 && j0 == 0 && fx >= 1 && fx <= TX));
  const int64_t plane = (int64_t)P.nx * P.ny;
  const int64_t o_col = fidx(P, oa, ob, 0), f_col = fidx(P, fa, fb, 0);
  // old fluxes at plane c (i, j) and of the k-faces above plane ck, into
  // qv = {own i, own j, own k, ring face}
  auto load_faces = [&](int c, int ck, bool do_k, double* qv) {
    const bool cin = c >= 0 && c < nk, kin = do_k && ck >= -1 && ck <= nk - 1;
    const int64_t oc = o_col + plane * c;
    qv[0] = (own_in && cin) ? qiin[oc] : 0.0;
    qv[1] = (own_in && cin) ? qjin[oc] : 0.0;
    qv[2] = (own_in && kin) ? qkin[o_col + plane * ck] : 0.0;
    qv[3] = 0.0;
    if (f_ab) {
      if (fk == 0 && cin) qv[3] = qiin[f_col + plane * c];
      else if (fk == 1 && cin) qv[3] = qjin[f_col + plane * c];
      else if (fk == 2 && kin) qv[3] = qkin[f_col + plane * ck];
    }
  };
  // new fluxes: i/j faces of plane c (cells in slot s) into face slot fs; k-faces
  // between planes ck (slot sl) and ck + 1 (slot sh) into k-slot kf
  auto faces = [&](int c, int s, int fs, int ck, int sl, int sh, int kf, bool do_k, const double* qv) {
    const bool inz = c >= k0 && c < k1;
    const bool kown = (ck >= k0 && ck < k1) || ck == -1;
    const bool cin = c >= 0 && c < nk, kin = ck >= -1 && ck <= nk - 1;
    const int x = ox, y = oy;
    const int64_t oc = o_col + plane * c;
    {  // own i-face
      double qn = 0.0, qp = 0.0;
      if (own_in && cin) {
        qn = flux(sm.IA[s][y][x], sm.IA[s][y][x + 1], sm.IT[s][y][x], sm.IT[s][y][x + 1],
                  sm.U[s][y][x + 1] - sm.U[s][y][x], qv[0], qp);
        if (inz) qiout[oc] = qn;
      }
      sm.QI[fs][y][x] = qn;
      if (check) sm.PI[fs][y][x] = qp;
    }
    {  // own j-face
      double qn = 0.0, qp = 0.0;
      if (own_in && cin) {
        qn = flux(sm.IA[s][y][x], sm.IA[s][y + 1][x], sm.IT[s][y][x], sm.IT[s][y + 1][x],
                  sm.U[s][y + 1][x] - sm.U[s][y][x], qv[1], qp);
        if (inz) qjout[oc] = qn;
      }
      sm.QJ[fs][y][x] = qn;
      if (check) sm.PJ[fs][y][x] = qp;
    }
    if (do_k) {  // own k-face
      double qn = 0.0, qp = 0.0;
      if (own_in && kin) {
        qn = flux(sm.IA[sl][y][x], sm.IA[sh][y][x], sm.IT[sl][y][x], sm.IT[sh][y][x],
                  sm.U[sh][y][x] - sm.U[sl][y][x], qv[2], qp);
        if (kown) qkout[o_col + plane * ck] = qn;
      }
      sm.QK[kf][y][x] = qn;
      if (check) sm.PK[kf][y][x] = qp;
    }
    if (fk == 0) {
      double qn = 0.0, qp = 0.0;
      if (f_ab && cin) {
        qn = flux(sm.IA[s][fy][fx], sm.IA[s][fy][fx + 1], sm.IT[s][fy][fx], sm.IT[s][fy][fx + 1],
                  sm.U[s][fy][fx + 1] - sm.U[s][fy][fx], qv[3], qp);
        if (inz && f_wr) qiout[f_col + plane * c] = qn;
      }
      sm.QI[fs][fy][fx] = qn;
      if (check) sm.PI[fs][fy][fx] = qp;
    } else if (fk == 1) {
      double qn = 0.0, qp = 0.0;
      if (f_ab && cin) {
        qn = flux(sm.IA[s][fy][fx], sm.IA[s][fy + 1][fx], sm.IT[s][fy][fx], sm.IT[s][fy + 1][fx],
                  sm.U[s][fy + 1][fx] - sm.U[s][fy][fx], qv[3], qp);
        if (inz && f_wr) qjout[f_col + plane * c] = qn;
      }
      sm.QJ[fs][fy][fx] = qn;
      if (check) sm.PJ[fs][fy][fx] = qp;
    } else if (fk == 2 && do_k) {
      double qn = 0.0, qp = 0.0;
      if (f_ab && kin)
        qn = flux(sm.IA[sl][fy][fx], sm.IA[sh][fy][fx], sm.IT[sl][fy][fx], sm.IT[sh][fy][fx],
                  sm.U[sh][fy][fx] - sm.U[sl][fy][fx], qv[3], qp);
      sm.QK[kf][fy][fx] = qn;
      if (check) sm.PK[kf][fy][fx] = qp;
    }
  };
  // flux_divergence.jl:119-239 at the own cell from face slots (zm, z0, zp) and k-slots (km, kp)
  auto divergence = [&](const double (*QI)[RY][TX + 1], const double (*QJ)[TY + 1][RX],
                        const double (*QK)[RY][RX], int zm, int z0, int zp, int kmn, int kpl, const double* cf) {
    const int x = ox, y = oy;
    const double t_ii = cf[0] * (QI[z0][y][x] - QI[z0][y][x - 1]);
    const double t_jj = cf[1] * (QJ[z0][y][x] - QJ[z0][y - 1][x]);
    const double t_kk = cf[2] * (QK[kpl][y][x] - QK[kmn][y][x]);
    const double qi_eta = cf[3] * (0.5 * (QI[z0][y + 1][x] + QI[z0][y + 1][x - 1]) -
                                   0.5 * (QI[z0][y - 1][x] + QI[z0][y - 1][x - 1]));
    const double qj_xi = cf[3] * (0.5 * (QJ[z0][y][x + 1] + QJ[z0][y - 1][x + 1]) -
                                  0.5 * (QJ[z0][y][x - 1] + QJ[z0][y - 1][x - 1]));
    const double qj_zeta = cf[4] * (0.5 * (QJ[zp][y][x] + QJ[zp][y - 1][x]) - 0.5 * (QJ[zm][y][x] + QJ[zm][y - 1][x]));
    const double qk_eta = cf[4] * (0.5 * (QK[kpl][y + 1][x] + QK[kmn][y + 1][x]) -
                                   0.5 * (QK[kpl][y - 1][x] + QK[kmn][y - 1][x]));
    const double qi_zeta = cf[5] * (0.5 * (QI[zp][y][x] + QI[zp][y][x - 1]) - 0.5 * (QI[zm][y][x] + QI[zm][y][x - 1]));
    const double qk_xi = cf[5] * (0.5 * (QK[kpl][y][x + 1] + QK[kmn][y][x + 1]) -
                                  0.5 * (QK[kpl][y][x - 1] + QK[kmn][y][x - 1]));
    const double h_a = cf[6] * (0.5 * (QI[z0][y][x] + QI[z0][y][x - 1]));
    const double h_b = cf[7] * (0.5 * (QJ[z0][y][x] + QJ[z0][y - 1][x]));
    const double h_c = cf[8] * (0.5 * (QK[kpl][y][x] + QK[kmn][y][x]));
    return t_ii + t_jj + t_kk + qi_eta + qi_zeta + qj_xi + qj_zeta + qk_eta + qk_xi + h_a + h_b + h_c;
  };

  // prologue: planes k0-1 and k0, their i/j faces and the k faces between them
  int s_0 = 1, s_p = 0;  // cell slots of planes z and z+1 (z-1 staged into 0 first)
  int f_m = 0, f_0 = 1, f_p = 2, k_m = 0, k_p = 1;
  double qa[4], qb[4];
  load_faces(k0 - 1, k0 - 1, true, qa);
  load_faces(k0, 0, false, qb);
  double prv_u = stage_plane(k0 - 1, 0).u;  // own cell of the plane below (ghost write at z = 0)
  C3 cur = stage_plane(k0, 1);
  __syncthreads();
  faces(k0 - 1, 0, f_m, k0 - 1, 0, 1, k_m, true, qa);
  faces(k0, 1, f_0, 0, 0, 0, 0, false, qb);
  load_faces(k0 + 1, k0, true, qa);  // used by the first plane of the loop
  __syncthreads();

  // the stage loads of plane k0 + 1, for the first loop iteration
  Pre3 p_own{0.0, 0.0, 0.0, 3}, p_rg{0.0, 0.0, 0.0, 3};
  int p_mode = 0;
  prefetch(k0 + 1, p_own, p_rg, p_mode);

  double local = 0.0;
  bool local_nan = false;
  for (int z = k0; z < k1; ++z) {
    // old fluxes of the next plane's faces, one plane ahead of their use
    if (z + 1 < k1) load_faces(z + 2, z + 1, true, qb);
    // stage plane z + 1 from its loads, then issue those of plane z + 2
    const C3 nxt = stage_plane_pre(z + 1, s_p, p_own, p_rg, p_mode);
    if (z + 1 < k1) prefetch(z + 2, p_own, p_rg, p_mode);
    __syncthreads();
    // own cell's coefficients: their loads overlap the face computations
    double cf[9], up = 0.0, S = 0.0;
    const int64_t id = fidx(P, oa, ob, z);
    if (own_in) {
#pragma unroll
      for (int q = 0; q < 9; ++q) cf[q] = P.coef[q][id];
      up = P.u_prev[id];
      S = P.S[id];
    }
    faces(z + 1, s_p, f_p, z, s_0, s_p, k_p, true, qa);
    // ghost neighbours of plane z, read before the barrier after which the next
    // plane may overwrite this cell slot
    const double g_im = sm.U[s_0][oy][ox - 1], g_ip = sm.U[s_0][oy][ox + 1];
    const double g_jm = sm.U[s_0][oy - 1][ox], g_jp = sm.U[s_0][oy + 1][ox];
    __syncthreads();
    if (own_in) {
      const double dq = divergence(sm.QI, sm.QJ, sm.QK, f_m, f_0, f_p, k_m, k_p, cf);
      const double un = cur.g * cur.u + cur.f * (up * inv_dt - dq + S);
      uout[id] = un;
      // ghosts of u after applybcs! of this iteration (copy!(T, u) returns them)
      if (EDGE) {
        if (oa == 0) uout[fidx(P, -1, ob, z)] = g_im;
        if (oa == ni - 1) uout[fidx(P, ni, ob, z)] = g_ip;
        if (ob == 0) uout[fidx(P, oa, -1, z)] = g_jm;
        if (ob == nj - 1) uout[fidx(P, oa, nj, z)] = g_jp;
      }
      if (z == 0) uout[fidx(P, oa, ob, -1)] = prv_u;
      if (z == nk - 1) uout[fidx(P, oa, ob, nk)] = nxt.u;
      if (check) {
        const double dqp = divergence(sm.PI, sm.PJ, sm.PK, f_m, f_0, f_p, k_m, k_p, cf);
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
    }
    // rotate: planes (z, z+1) become (z-1, z)
    prv_u = cur.u;
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
    for (int r = 0; r < 4; ++r) qa[r] = qb[r];
  }
  finish_iteration<NT>(P, C, tile, iter, check, local, local_nan, bad, sm.red, &sm.flag);
}

template <bool HARM, int TX, int TY>
static cudaError_t launch3m(const Problem* probs, const int2* items, int n_edge, int n_int, const SweepStreams& ss) {
  constexpr int NT = TX * TY, bytes = (int)sizeof(M3Smem<TX, TY>);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(march3d_fast<HARM, true, TX, TY>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(march3d_fast<HARM, false, TX, TY>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               bytes);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  // boundary tiles on the side stream, concurrently with the interior tiles
  const bool fork = n_edge > 0 && n_int > 0 && ss.side != nullptr;
  cudaError_t e = cudaSuccess;
  if (fork) {
    if ((e = cudaEventRecord(ss.ev_fork, ss.main)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.side, ss.ev_fork, 0)) != cudaSuccess) return e;
  }
  if (n_edge > 0)
    march3d_fast<HARM, true, TX, TY><<<n_edge, NT, bytes, fork ? ss.side : ss.main>>>(probs, items);
  if (n_int > 0) march3d_fast<HARM, false, TX, TY><<<n_int, NT, bytes, ss.main>>>(probs, items + n_edge);
  if (fork) {
    if ((e = cudaEventRecord(ss.ev_join, ss.side)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(ss.main, ss.ev_join, 0)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

// column tiles of tx x ty cells: 32 x 8 or 16 x 16 (a shorter ring: 68 ring cells
// and 164 ring faces per 256 cells instead of 84 and 208)
cudaError_t launch_march3d_fast(int harmonic, int tx, int ty, const Problem* probs, const int2* items, int n_edge,
                                int n_int, const SweepStreams& ss) {
  if (tx == 32 && ty == 8)
    return harmonic ? launch3m<true, 32, 8>(probs, items, n_edge, n_int, ss)
                    : launch3m<false, 32, 8>(probs, items, n_edge, n_int, ss);
  if (tx == 16 && ty == 16)
    return harmonic ? launch3m<true, 16, 16>(probs, items, n_edge, n_int, ss)
                    : launch3m<false, 16, 16>(probs, items, n_edge, n_int, ss);
  return cudaErrorInvalidValue;
}

// Is column tile `tile` (any strip) of a 3D problem free of (i, j) ghost logic:
// its cells and their one-cell ring all domain cells?
bool march3d_tile_interior(int ni, int nj, int tiles_i, int tiles_j, int tx, int ty, int tile) {
  const int ti = tile % tiles_i, tj = (tile / tiles_i) % tiles_j;
  const int i0 = ti * tx, j0 = tj * ty;
  return i0 >= 1 && i0 + tx + 1 <= ni && j0 >= 1 && j0 + ty + 1 <= nj;
}

}  // namespace cdm
