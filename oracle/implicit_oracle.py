"""CPU restatement of the reference's implicit (backward-Euler + Krylov) scheme.

Test infrastructure: only the tests, smoke() and the bench's CPU arms use this
module, as the checker of the library's implicit path.

What it restates (paths inside the reference project):
* ImplicitScheme(mesh, bcs; mean)                 src/implicit/ImplictSolver.jl:49-160
* the matrix pattern and its boundary rows        src/implicit/init_matrix.jl:1-170
  (diagonal 1 on every row; Neumann / periodic sides add -1 at the interior /
  opposite cell on the side's rows without the corners; Dirichlet adds nothing)
* assemble!, _assembly_kernel_2d / _3d           src/implicit/matrix_assembly.jl:5-59,
                                                  src/implicit/inner_operators.jl:62-160
* edge_diffusivity, conservative_edge_terms       inner_operators.jl:254-280, src/edge_terms.jl:31-87, :146-263
* stencil_2d, stencil_3d                          src/implicit/stencils.jl:14-40, :42-137
* bc_operator / bc_rhs_coefficient                inner_operators.jl:188-211,
                                                  src/boundary_conditions/boundary_operators.jl:271-273
* update_conductivity! (scalar cp)                src/conductivity.jl:13-31, :93-104
* nonlinear_thermal_conduction_step!(::ImplicitScheme)   src/nonlinear_thermal_conduction.jl:4-48
* _iterative_solve!: cutoff, next_dt, copy        ImplictSolver.jl:249-330, src/timestep_control.jl:33-73

The linear system is solved here by a sparse direct solve (scipy), so the
oracle's solution is the exact solution of the assembled system to rounding;
the reference's GMRES + ILU(0) and the library's BiCGSTAB both stop at the
reference's rule ||b - A x||_2 <= atol + rtol ||b - A x0||_2.

Element arithmetic follows Julia's evaluation order (a + b + c left to
right, x^2 as x*x, a*b/c as (a*b)/c), elementwise in IEEE double, so the
assembled coefficients are comparable bit for bit.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle.oracle import applybcs

NEUMANN, DIRICHLET, PERIODIC, NEG_SYMMETRY = 0, 1, 2, 3
# stencil entries in the order of stencils.jl:35 and :108-136 (offsets2d / offsets3d,
# inner_operators.jl:19-49): i fastest, then j, then k
OFFSETS_2D = [(-1, -1), (0, -1), (1, -1), (-1, 0), (0, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]
OFFSETS_3D = [(di, dj, dk) for dk in (-1, 0, 1) for dj in (-1, 0, 1) for di in (-1, 0, 1)]


def pow_model(x, n):
    """|T|^n as the library and the APT oracle evaluate it: products for the
    integer part, one correctly rounded sqrt for a half, pow otherwise."""
    if n == 0.0:
        return np.ones_like(x)
    twice = 2.0 * n
    if 0.0 < n <= 16.0 and twice == np.floor(twice):
        m = int(np.floor(n))
        p = None
        if m >= 1:
            p = x.copy()
            for _ in range(1, m):
                p = p * x
        if twice != 2.0 * m:
            p = p * np.sqrt(x) if p is not None else np.sqrt(x)
        return p
    return np.power(x, n)


def kappa(k0, n, T):
    with np.errstate(invalid="ignore", over="ignore"):
        out = k0 * pow_model(np.abs(T), n)
    return np.where(np.isfinite(T), out, 0.0)


def _mean(mean, a, b):
    if mean == "harmonic":
        return (2.0 * a * b) / (a + b)
    return (a + b) / 2.0


class ImplicitOracle:
    """ImplicitScheme + nonlinear_thermal_conduction_step! on one 2D or 3D mesh (nhalo >= 1).

    The diffusion problem covers the domain and one halo layer (region 2 of
    ImplictSolver.jl:77-98); rows are numbered column-major over it."""

    def __init__(self, mesh, bcs, mean="harmonic"):
        self.mesh = mesh
        self.nd = mesh.ndim
        self.bcs = list(bcs.values()) if isinstance(bcs, dict) else list(bcs)
        self.kinds = [b.kind for b in self.bcs]
        self.vals = [float(getattr(b, "value", 0.0)) for b in self.bcs]
        # init_matrix.jl:7-12 and :184-192 (in 3D the k sides are not part of the test)
        for lo, hi in ((0, 1), (2, 3)):
            if (self.kinds[lo] == PERIODIC) != (self.kinds[hi] == PERIODIC):
                raise ValueError("Inconsistent periodic boundary conditions")
        if NEG_SYMMETRY in self.kinds:
            raise ValueError("the implicit scheme has no FixedNegSymmetryBC rows")
        self.mean = mean
        m = mesh
        h = m.nhalo
        self.n1, self.n2 = m.ni + 2, m.nj + 2
        self.n3 = m.nk + 2 if self.nd == 3 else 1
        self.N = self.n1 * self.n2 * self.n3
        # region 2 inside the mesh arrays ([k,] j, i views)
        self.sl = (slice(h - 1, h + m.nj + 1), slice(h - 1, h + m.ni + 1))
        if self.nd == 3:
            self.sl = (slice(h - 1, h + m.nk + 1),) + self.sl
        self.shape = (self.n3, self.n2, self.n1) if self.nd == 3 else (self.n2, self.n1)
        self.source = np.zeros(self.shape)
        self.x = None

    def _full_shape(self):
        m, h = self.mesh, self.mesh.nhalo
        fs = (m.nj + 2 * h, m.ni + 2 * h)
        return ((m.nk + 2 * h),) + fs if self.nd == 3 else fs

    def _r2(self, a):
        """Region 2 of a full mesh array, as a ([nk+2,] nj+2, ni+2) view."""
        a = np.asarray(a, dtype=np.float64).reshape(self._full_shape())
        return a[self.sl]

    def set_source(self, S):
        self.source = self._r2(S).copy()

    # ---------------------------------------------------------------- assembly
    def assemble(self, T, rho, cp, k0, n, dt):
        """A (scipy CSR), b, the stencil coefficients of the interior rows
        (9 or 27, region-2 shape; zero elsewhere) and alpha, for T and rho
        already carrying their boundary conditions."""
        m = self.mesh
        Tr, rr = self._r2(T), self._r2(rho)
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha = np.abs(kappa(k0, n, Tr) / (rr * cp))
        J = self._r2(m.cell_J)
        nf = self.nd
        eJ = [self._r2(m.edge_J[f]) for f in range(nf)]
        eh = [[self._r2(m.edge_hat[f][k]) if m.edge_hat[f][k] is not None else None for k in range(9)]
              for f in range(nf)]
        c = self._stencil2(alpha, J, eJ, eh, dt) if self.nd == 2 else self._stencil3(alpha, J, eJ, eh, dt)
        I = (slice(1, -1),) * self.nd
        b = np.zeros(self.shape)
        b[I] = (self.source[I] * dt + Tr[I]) * J[I]
        rhs = [0.0 if k != DIRICHLET else v for k, v in zip(self.kinds, self.vals)]
        # bc_operator priority ilo, ihi, jlo, jhi[, klo, khi]: later assignments win here
        if self.nd == 3:
            b[-1, :, :] = rhs[5]
            b[0, :, :] = rhs[4]
            b[:, -1, :] = rhs[3]
            b[:, 0, :] = rhs[2]
            b[:, :, -1] = rhs[1]
            b[:, :, 0] = rhs[0]
        else:
            b[-1, :] = rhs[3]
            b[0, :] = rhs[2]
            b[:, -1] = rhs[1]
            b[:, 0] = rhs[0]
        A = self._matrix(c)
        return A, b.ravel(), c, alpha

    def _stencil2(self, alpha, J, eJ, eh, dt):
        I = slice(1, -1)
        a_c = alpha[I, I]
        a_ip = _mean(self.mean, a_c, alpha[I, 2:])
        a_im = _mean(self.mean, a_c, alpha[I, :-2])
        a_jp = _mean(self.mean, a_c, alpha[2:, I])
        a_jm = _mean(self.mean, a_c, alpha[:-2, I])

        def cur(f, k):  # face value at the cell
            return eh[f][k][I, I]

        def im1(f, k):  # face of the i-1 cell (the i-1/2 face)
            return eh[f][k][I, :-2]

        def jm1(f, k):
            return eh[f][k][:-2, I]

        Jip, Jjp, Jim, Jjm = eJ[0][I, I], eJ[1][I, I], eJ[0][I, :-2], eJ[1][:-2, I]
        # edge_terms.jl:66-76 (ξ̂.x₁ = [0], ξ̂.x₂ = [1], η̂.x₁ = [3], η̂.x₂ = [4])
        xx, xy, ex, ey = cur(0, 0), cur(0, 1), cur(0, 3), cur(0, 4)
        a_xi2_ip = a_ip * (xx * xx + xy * xy) / Jip
        a_xieta_ip = a_ip * (xx * ex + xy * ey) / (4.0 * Jip)
        xx, xy, ex, ey = im1(0, 0), im1(0, 1), im1(0, 3), im1(0, 4)
        a_xi2_im = a_im * (xx * xx + xy * xy) / Jim
        a_xieta_im = a_im * (xx * ex + xy * ey) / (4.0 * Jim)
        xx, xy, ex, ey = cur(1, 0), cur(1, 1), cur(1, 3), cur(1, 4)
        a_eta2_jp = a_jp * (ex * ex + ey * ey) / Jjp
        a_etaxi_jp = a_jp * (xx * ex + xy * ey) / (4.0 * Jjp)
        xx, xy, ex, ey = jm1(1, 0), jm1(1, 1), jm1(1, 3), jm1(1, 4)
        a_eta2_jm = a_jm * (ex * ex + ey * ey) / Jjm
        a_etaxi_jm = a_jm * (xx * ex + xy * ey) / (4.0 * Jjm)
        # stencils.jl:14-40
        c = np.zeros((9, self.n2, self.n1))
        Jc = J[I, I]
        c[4][I, I] = Jc + (a_eta2_jp + a_eta2_jm + a_xi2_ip + a_xi2_im) * dt
        c[2][I, I] = (a_etaxi_jm + a_xieta_ip) * dt            # i+1, j-1
        c[6][I, I] = (a_etaxi_jp + a_xieta_im) * dt            # i-1, j+1
        c[0][I, I] = (-a_etaxi_jm - a_xieta_im) * dt           # i-1, j-1
        c[8][I, I] = (-a_etaxi_jp - a_xieta_ip) * dt           # i+1, j+1
        c[5][I, I] = (-a_etaxi_jp + a_etaxi_jm - a_xi2_ip) * dt  # i+1, j
        c[3][I, I] = (a_etaxi_jp - a_etaxi_jm - a_xi2_im) * dt   # i-1, j
        c[7][I, I] = (-a_eta2_jp - a_xieta_ip + a_xieta_im) * dt  # i, j+1
        c[1][I, I] = (-a_eta2_jm + a_xieta_ip - a_xieta_im) * dt  # i, j-1
        return c

    def _stencil3(self, alpha, J, eJ, eh, dt):
        I = slice(1, -1)
        C3 = (I, I, I)
        a_c = alpha[C3]
        sh = {"c": C3, "i": (I, I, slice(None, -2)), "j": (I, slice(None, -2), I), "k": (slice(None, -2), I, I)}
        a = {"ip": _mean(self.mean, a_c, alpha[I, I, 2:]), "im": _mean(self.mean, a_c, alpha[I, I, :-2]),
             "jp": _mean(self.mean, a_c, alpha[I, 2:, I]), "jm": _mean(self.mean, a_c, alpha[I, :-2, I]),
             "kp": _mean(self.mean, a_c, alpha[2:, I, I]), "km": _mean(self.mean, a_c, alpha[:-2, I, I])}

        def face(f, where):
            """J and the three J-scaled metric vectors (ξ̂, η̂, ζ̂) of a face (edge_terms.jl:158-233)."""
            s = sh[where]
            vec = [[eh[f][3 * v + cc][s] for cc in range(3)] for v in range(3)]
            return eJ[f][s], vec

        def dot(u, v):
            return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]

        t = {}
        for name, f, where in (("ip", 0, "c"), ("im", 0, "i"), ("jp", 1, "c"), ("jm", 1, "j"), ("kp", 2, "c"),
                               ("km", 2, "k")):
            Jf, (xi, eta, zeta) = face(f, where)
            al = a[name]
            if f == 0:  # edge_terms.jl:235-243
                t["xi2_" + name] = al * dot(xi, xi) / Jf
                t["xieta_" + name] = al * dot(xi, eta) / (4.0 * Jf)
                t["xizeta_" + name] = al * dot(xi, zeta) / (4.0 * Jf)
            elif f == 1:  # :245-250
                t["eta2_" + name] = al * dot(eta, eta) / Jf
                t["etaxi_" + name] = al * dot(xi, eta) / (4.0 * Jf)
                t["etazeta_" + name] = al * dot(eta, zeta) / (4.0 * Jf)
            else:  # :252-257
                t["zeta2_" + name] = al * dot(zeta, zeta) / Jf
                t["zetaxi_" + name] = al * dot(zeta, xi) / (4.0 * Jf)
                t["zetaeta_" + name] = al * dot(zeta, eta) / (4.0 * Jf)
        T = t
        c = np.zeros((27, self.n3, self.n2, self.n1))
        slot = lambda di, dj, dk: (di + 1) + 3 * (dj + 1) + 9 * (dk + 1)
        # stencils.jl:84-106
        c[slot(0, -1, -1)][C3] = (-T["zetaeta_km"] - T["etazeta_jm"]) * dt
        c[slot(-1, 0, -1)][C3] = (-T["zetaxi_km"] - T["xizeta_im"]) * dt
        c[slot(1, 0, -1)][C3] = (T["zetaxi_km"] + T["xizeta_ip"]) * dt
        c[slot(0, 1, -1)][C3] = (T["zetaeta_km"] + T["etazeta_jp"]) * dt
        c[slot(-1, -1, 0)][C3] = (-T["etaxi_jm"] - T["xieta_im"]) * dt
        c[slot(1, -1, 0)][C3] = (T["etaxi_jm"] + T["xieta_ip"]) * dt
        c[slot(-1, 1, 0)][C3] = (T["etaxi_jp"] + T["xieta_im"]) * dt
        c[slot(1, 1, 0)][C3] = (-T["etaxi_jp"] - T["xieta_ip"]) * dt
        c[slot(0, -1, 1)][C3] = (T["zetaeta_kp"] + T["etazeta_jm"]) * dt
        c[slot(-1, 0, 1)][C3] = (T["zetaxi_kp"] + T["xizeta_im"]) * dt
        c[slot(1, 0, 1)][C3] = (-T["zetaxi_kp"] - T["xizeta_ip"]) * dt
        c[slot(0, 1, 1)][C3] = (-T["zetaeta_kp"] - T["etazeta_jp"]) * dt
        c[slot(0, 0, 0)][C3] = J[C3] + (T["zeta2_kp"] + T["zeta2_km"] + T["eta2_jp"] + T["eta2_jm"] + T["xi2_ip"]
                                        + T["xi2_im"]) * dt
        c[slot(1, 0, 0)][C3] = (-T["xi2_ip"] - T["etaxi_jp"] + T["etaxi_jm"] - T["zetaxi_kp"] + T["zetaxi_km"]) * dt
        c[slot(-1, 0, 0)][C3] = (-T["xi2_im"] + T["etaxi_jp"] - T["etaxi_jm"] + T["zetaxi_kp"] - T["zetaxi_km"]) * dt
        c[slot(0, 1, 0)][C3] = (-T["eta2_jp"] - T["xieta_ip"] + T["xieta_im"] - T["zetaeta_kp"] + T["zetaeta_km"]) * dt
        c[slot(0, -1, 0)][C3] = (-T["eta2_jm"] + T["xieta_ip"] - T["xieta_im"] + T["zetaeta_kp"] - T["zetaeta_km"]) * dt
        c[slot(0, 0, 1)][C3] = (-T["zeta2_kp"] - T["xizeta_ip"] + T["xizeta_im"] - T["etazeta_jp"]
                                + T["etazeta_jm"]) * dt
        c[slot(0, 0, -1)][C3] = (-T["zeta2_km"] + T["xizeta_ip"] - T["xizeta_im"] + T["etazeta_jp"]
                                 - T["etazeta_jm"]) * dt
        return c

    def _matrix(self, c):
        idx = np.arange(self.N).reshape(self.shape)
        offs = OFFSETS_2D if self.nd == 2 else OFFSETS_3D
        strides = (1, self.n1, self.n1 * self.n2)
        inner_sl = (slice(1, -1),) * self.nd
        inner = idx[inner_sl].ravel()
        rows, cols, vals = [], [], []
        diag = np.ones(self.N)
        for s, off in enumerate(offs):
            if all(o == 0 for o in off):
                diag[inner] = c[s][inner_sl].ravel()
                continue
            rows.append(inner)
            cols.append(inner + sum(o * st for o, st in zip(off, strides)))
            vals.append(c[s][inner_sl].ravel())
        rows.insert(0, idx.ravel())
        cols.insert(0, idx.ravel())
        vals.insert(0, diag)
        # boundary rows (init_matrix.jl:69-167, :252-390): every side over the
        # interior range of the other axes (edges and corners: the diagonal only)
        n = (self.n1, self.n2, self.n3)[:self.nd]
        for side in range(2 * self.nd):
            axis, lo = side // 2, side % 2 == 0
            kind = self.kinds[side]
            if kind not in (NEUMANN, PERIODIC):
                continue
            # region-2 coordinates of the side's rows, arrays indexed [k, j, i] -> reverse axis
            sel = [slice(1, -1)] * self.nd
            ax = self.nd - 1 - axis
            sel[ax] = 0 if lo else -1
            r = idx[tuple(sel)].ravel()
            st = strides[axis]
            if kind == NEUMANN:
                col = r + st if lo else r - st
            else:  # periodic: the cell next to the opposite side's ghost
                col = r + (n[axis] - 2) * st if lo else r - (n[axis] - 2) * st
            rows.append(r), cols.append(col), vals.append(-np.ones(len(r)))
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(self.N, self.N))

    # ------------------------------------------------------------------ step
    def step(self, T, rho, cp, k0, n, dt, *, enforce_positivity=True, apply_density_bc=True,
             ndt_tol=1e-3, maximum_u_change=0.05, timestep_growth_factor=1.1):
        """nonlinear_thermal_conduction_step!: T (full mesh array) is updated
        in place over region 2; returns (stats, next_dt, A, b, c) with c the
        stencil entries of the interior rows (9, nj+2, ni+2)."""
        m = self.mesh
        nk = m.nk if self.nd == 3 else 1
        applybcs(self.nd, m.ni, m.nj, nk, m.nhalo, self.bcs, T)
        rho = rho.copy()
        if apply_density_bc:
            applybcs(self.nd, m.ni, m.nj, nk, m.nhalo, self.bcs, rho)
        A, b, c, alpha = self.assemble(T, rho, cp, k0, n, dt)
        dom = alpha[(slice(1, -1),) * self.nd]
        if not np.all(np.isfinite(dom)):
            raise ValueError("invalid diffusivity")
        x = spla.spsolve(A.tocsc(), b)
        resid = float(np.linalg.norm(b - A @ x))
        if enforce_positivity:  # cutoff: (0.5(|a| + a)) * isfinite(a), Julia's false a strong zero
            with np.errstate(invalid="ignore"):
                x = np.where(np.isfinite(x), 0.5 * (np.abs(x) + x), 0.0)
        un = self._r2(T).ravel().copy()
        umax = un.max()
        u0 = umax * ndt_tol
        with np.errstate(divide="ignore", invalid="ignore"):
            d = np.abs(x - un) / (x + u0)
        d = np.where(np.isfinite(d), d, 0.0) * 1.0
        mr = d.max()
        ndt = min(dt * np.sqrt(abs(maximum_u_change / mr)), timestep_growth_factor * dt)
        self._r2(T)[...] = x.reshape(self.shape)
        self.x = x
        return {"abs_err": resid, "rel_err": resid}, ndt, A, b, c


def true_residual(A, b, x):
    return float(np.linalg.norm(b - A @ x))
