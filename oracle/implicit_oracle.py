"""CPU restatement of the reference's implicit (backward-Euler + Krylov) scheme.

Test infrastructure: only the tests, smoke() and the bench's CPU arms use this
module, as the checker of the library's implicit path.

What it restates (paths inside the reference project):
* ImplicitScheme(mesh, bcs; mean)                 src/implicit/ImplictSolver.jl:49-160
* the matrix pattern and its boundary rows        src/implicit/init_matrix.jl:1-170
  (diagonal 1 on every row; Neumann / periodic sides add -1 at the interior /
  opposite cell on the side's rows without the corners; Dirichlet adds nothing)
* assemble!, _assembly_kernel_2d                  src/implicit/matrix_assembly.jl:5-31,
                                                  src/implicit/inner_operators.jl:62-105
* edge_diffusivity, conservative_edge_terms       inner_operators.jl:265-280, src/edge_terms.jl:31-87
* stencil_2d                                      src/implicit/stencils.jl:14-40
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
# stencil entries in the order of stencils.jl:35 (offsets2d, inner_operators.jl:19-21)
OFFSETS_2D = [(-1, -1), (0, -1), (1, -1), (-1, 0), (0, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]


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
    """ImplicitScheme + nonlinear_thermal_conduction_step! on one 2D mesh (nhalo >= 1).

    The diffusion problem covers the domain and one halo layer (region 2 of
    ImplictSolver.jl:77-98); rows are numbered column-major over it."""

    def __init__(self, mesh, bcs, mean="harmonic"):
        assert mesh.ndim == 2, "the implicit oracle restates the 2D scheme"
        self.mesh = mesh
        self.bcs = list(bcs.values()) if isinstance(bcs, dict) else list(bcs)
        self.kinds = [b.kind for b in self.bcs]
        self.vals = [float(getattr(b, "value", 0.0)) for b in self.bcs]
        for lo, hi in ((0, 1), (2, 3)):
            if (self.kinds[lo] == PERIODIC) != (self.kinds[hi] == PERIODIC):
                raise ValueError("Inconsistent periodic boundary conditions")  # init_matrix.jl:7-12
        if NEG_SYMMETRY in self.kinds:
            raise ValueError("the implicit scheme has no FixedNegSymmetryBC rows")
        self.mean = mean
        m = mesh
        self.n1, self.n2 = m.ni + 2, m.nj + 2
        self.N = self.n1 * self.n2
        h = m.nhalo
        # region 2 inside the mesh arrays
        self.sl = (slice(h - 1, h + m.nj + 1), slice(h - 1, h + m.ni + 1))  # [j, i] on (ny, nx) views
        self.source = np.zeros((self.n2, self.n1))
        self.x = None  # Krylov warm start (the previous solution)

    def _r2(self, a):
        """Region 2 of a full mesh array, as a (nj+2, ni+2) [j, i] view."""
        m = self.mesh
        a = np.asarray(a, dtype=np.float64).reshape(m.nj + 2 * m.nhalo, m.ni + 2 * m.nhalo)
        return a[self.sl]

    def set_source(self, S):
        self.source = self._r2(S).copy()

    # ---------------------------------------------------------------- assembly
    def assemble(self, T, rho, cp, k0, n, dt):
        """A (scipy CSR), b, the 9 stencil coefficients of the interior rows
        (9, nj+2, ni+2; zero elsewhere) and alpha, for temperatures T and
        densities rho already carrying their boundary conditions."""
        m = self.mesh
        Tr, rr = self._r2(T), self._r2(rho)
        with np.errstate(divide="ignore", invalid="ignore"):
            alpha = np.abs(kappa(k0, n, Tr) / (rr * cp))
        J = self._r2(m.cell_J)
        eJ = [self._r2(m.edge_J[f]) for f in range(2)]
        eh = [[self._r2(m.edge_hat[f][k]) if m.edge_hat[f][k] is not None else None for k in range(9)]
              for f in range(2)]
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
        # right-hand side: (S dt + u) J inside, bc_operator on the boundary rows
        b = np.zeros((self.n2, self.n1))
        b[I, I] = (self.source[I, I] * dt + Tr[I, I]) * Jc
        rhs = [0.0 if k != DIRICHLET else v for k, v in zip(self.kinds, self.vals)]
        # priority of bc_operator: ilo, ihi, jlo, jhi (later assignments first here)
        b[-1, :] = rhs[3]
        b[0, :] = rhs[2]
        b[:, -1] = rhs[1]
        b[:, 0] = rhs[0]
        A = self._matrix(c)
        return A, b.ravel(), c, alpha

    def _matrix(self, c):
        n1, n2 = self.n1, self.n2
        idx = np.arange(self.N).reshape(n2, n1)
        rows, cols, vals = [idx.ravel()], [idx.ravel()], [np.ones(self.N)]
        inner = idx[1:-1, 1:-1].ravel()
        for s, (di, dj) in enumerate(OFFSETS_2D):
            if (di, dj) == (0, 0):
                continue
            rows.append(inner)
            cols.append(inner + di + dj * n1)
            vals.append(c[s][1:-1, 1:-1].ravel())
        diag = np.ones(self.N)
        diag[inner] = c[4][1:-1, 1:-1].ravel()
        vals[0] = diag
        # boundary rows (init_matrix.jl:69-167), corners excluded
        jj = np.arange(1, n2 - 1)
        ii = np.arange(1, n1 - 1)
        sides = [
            (self.kinds[0], idx[jj, 0], idx[jj, 1], idx[jj, n1 - 2]),
            (self.kinds[1], idx[jj, n1 - 1], idx[jj, n1 - 2], idx[jj, 1]),
            (self.kinds[2], idx[0, ii], idx[1, ii], idx[n2 - 2, ii]),
            (self.kinds[3], idx[n2 - 1, ii], idx[n2 - 2, ii], idx[1, ii]),
        ]
        for kind, r, neumann_col, periodic_col in sides:
            if kind == NEUMANN:
                rows.append(r), cols.append(neumann_col), vals.append(-np.ones(len(r)))
            elif kind == PERIODIC:
                rows.append(r), cols.append(periodic_col), vals.append(-np.ones(len(r)))
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(self.N, self.N))

    # ------------------------------------------------------------------ step
    def step(self, T, rho, cp, k0, n, dt, *, enforce_positivity=True, apply_density_bc=True,
             ndt_tol=1e-3, maximum_u_change=0.05, timestep_growth_factor=1.1):
        """nonlinear_thermal_conduction_step!: T (full mesh array) is updated
        in place over region 2; returns (stats, next_dt, A, b, c) with c the
        stencil entries of the interior rows (9, nj+2, ni+2)."""
        m = self.mesh
        applybcs(2, m.ni, m.nj, 1, m.nhalo, self.bcs, T)
        rho = rho.copy()
        if apply_density_bc:
            applybcs(2, m.ni, m.nj, 1, m.nhalo, self.bcs, rho)
        A, b, c, alpha = self.assemble(T, rho, cp, k0, n, dt)
        dom = alpha[1:-1, 1:-1]
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
        self._r2(T)[...] = x.reshape(self.n2, self.n1)
        self.x = x
        return {"abs_err": resid, "rel_err": resid}, ndt, A, b, c


def true_residual(A, b, x):
    return float(np.linalg.norm(b - A @ x))
