"""Curvilinear meshes in the layout the APT path reads.

The reference takes its meshes from CurvilinearGrids (not vendored; compat
"0.6" in Project.toml) and reads these fields of them:

* ``mesh.cell_center_metrics.{ξ,η,ζ}.{x₁,x₂,x₃}`` and ``.J``
  (src/pseudo_transient/flux_divergence.jl:11-14, :125-135;
  src/pseudo_transient/PseudoTransientSolver.jl:127),
* ``mesh.edge_metrics.{i₊½,j₊½,k₊½}.{J, ξ̂, η̂, ζ̂}``
  (src/pseudo_transient/mesh_metric_cache.jl:51-85, :117-207),
* node coordinates for ``phys_dims`` (PseudoTransientSolver.jl:122-153) and
  centroids for initial conditions (test/integrated/2d/gaussian/run.jl:114-118).

Metrics are derivatives with respect to the *index* coordinates (one cell is
one unit of ξ), which is what the discrete operators of the reference assume
(`qᵢ[i] - qᵢ[i-1]` is ∂q/∂ξ).  This module evaluates them exactly from the
closed-form mappings of the benchmark meshes (the default, independent of any
halo extrapolation) or, for arbitrary node coordinates, by second-order
differences (``mesh_from_nodes_2d``).

All arrays are full size including ``nhalo`` halo layers, stored as torch
float64 tensors of shape (ny, nx) or (nz, ny, nx), C-contiguous, i.e.
column-major in (i, j, k) like the reference's Julia arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import torch

TWO_PI = 2.0 * math.pi


@dataclass
class CurvilinearMesh:
    ndim: int
    ni: int
    nj: int
    nk: int
    nhalo: int
    cell_inv: List[Optional[torch.Tensor]]           # [3*a + c], a = ξ,η,ζ ; c = x,y,z
    cell_J: torch.Tensor
    edge_J: List[Optional[torch.Tensor]]             # face family i+½, j+½, k+½
    edge_hat: List[List[Optional[torch.Tensor]]]     # [f][3*a + c]
    centroids: List[torch.Tensor]                    # full-size cell centres
    nodes: List[torch.Tensor]                        # domain node coordinates
    L: float = 0.0
    spacing: Sequence[float] = field(default_factory=lambda: (0.0, 0.0, 0.0))
    # cell_center_metrics.{x₁,x₂}.{ξ,η} (forward metrics x_ξ, x_η, y_ξ, y_η), read by
    # the twilight-zone forcing only (twilight_zone.jl:115-118); 2D analytic meshes
    cell_fwd: Optional[List[torch.Tensor]] = None

    @property
    def nnodes(self):
        """mesh.nnodes: domain nodes per axis."""
        return (self.ni + 1, self.nj + 1) if self.ndim == 2 else (self.ni + 1, self.nj + 1, self.nk + 1)

    @property
    def full_shape(self):
        h2 = 2 * self.nhalo
        if self.ndim == 2:
            return (self.nj + h2, self.ni + h2)
        return (self.nk + h2, self.nj + h2, self.ni + h2)

    @property
    def ncells_full(self) -> int:
        return int(math.prod(self.full_shape))

    @property
    def ncells(self) -> int:
        return self.ni * self.nj * (self.nk if self.ndim == 3 else 1)

    def domain(self):
        """Index tuple selecting the domain cells of a full-size array."""
        h = self.nhalo
        if self.ndim == 2:
            return (slice(h, h + self.nj), slice(h, h + self.ni))
        return (slice(h, h + self.nk), slice(h, h + self.nj), slice(h, h + self.ni))

    def to(self, device) -> "CurvilinearMesh":
        mv = lambda t: None if t is None else t.to(device)
        return CurvilinearMesh(
            self.ndim, self.ni, self.nj, self.nk, self.nhalo,
            [mv(t) for t in self.cell_inv], mv(self.cell_J),
            [mv(t) for t in self.edge_J], [[mv(t) for t in row] for row in self.edge_hat],
            [mv(t) for t in self.centroids], [t for t in self.nodes], self.L, tuple(self.spacing),
            None if self.cell_fwd is None else [mv(t) for t in self.cell_fwd])


def _phys_dims(ndim, nodes, cell_J_domain):
    """phys_dims (PseudoTransientSolver.jl:122-153)."""
    if ndim == 2:
        ds = math.sqrt(float(cell_J_domain.min()))
        spacing = (ds, ds, 0.0)
        L = min(float(nodes[0].max() - nodes[0].min()), float(nodes[1].max() - nodes[1].min()))
    else:
        x, y, z = nodes  # shapes (nk+1, nj+1, ni+1)
        spacing = (float(torch.diff(x, dim=2).min()), float(torch.diff(y, dim=1).min()),
                   float(torch.diff(z, dim=0).min()))
        L = min(float(t.max() - t.min()) for t in nodes)
    return L, spacing


def _index_grid(n, nhalo, offset, device):
    """Computational unit coordinate of full index I: ((I - nhalo) + offset) / n."""
    idx = torch.arange(n + 2 * nhalo, dtype=torch.float64, device=device) - nhalo
    return (idx + offset) / n


def wavy_mesh_2d(ni: int, nj: int, amp: float = 0.05, nhalo: int = 1,
                 device="cpu") -> CurvilinearMesh:
    """x = ξ + a sin(2πξ) sin(2πη), y = η + a sin(2πξ) sin(2πη) on [0,1]²."""

    def mapping(s, t):
        ss, st = torch.sin(TWO_PI * s), torch.sin(TWO_PI * t)
        cs, ct = torch.cos(TWO_PI * s), torch.cos(TWO_PI * t)
        w = amp * ss * st
        x, y = s + w, t + w
        ws, wt = amp * TWO_PI * cs * st, amp * TWO_PI * ss * ct
        # derivatives w.r.t. index coordinates (i = ni*s, j = nj*t)
        xi, xj = (1.0 + ws) / ni, wt / nj
        yi, yj = ws / ni, (1.0 + wt) / nj
        return x, y, xi, xj, yi, yj

    def at(off_i, off_j):
        s = _index_grid(ni, nhalo, off_i, device)
        t = _index_grid(nj, nhalo, off_j, device)
        T, S = torch.meshgrid(t, s, indexing="ij")  # shape (ny, nx), i fastest
        return mapping(S, T)

    x, y, xi, xj, yi, yj = at(0.5, 0.5)
    J = xi * yj - xj * yi
    cell_inv = [yj / J, -xj / J, None, -yi / J, xi / J, None, None, None, None]
    edge_J, edge_hat = [None] * 3, [[None] * 9 for _ in range(3)]
    for f, (oi, oj) in enumerate(((1.0, 0.5), (0.5, 1.0))):
        _, _, fxi, fxj, fyi, fyj = at(oi, oj)
        edge_J[f] = fxi * fyj - fxj * fyi
        edge_hat[f][0], edge_hat[f][1] = fyj, -fxj      # ξ̂ = J ∇ξ
        edge_hat[f][3], edge_hat[f][4] = -fyi, fxi      # η̂ = J ∇η
    s_n = torch.arange(ni + 1, dtype=torch.float64, device=device) / ni
    t_n = torch.arange(nj + 1, dtype=torch.float64, device=device) / nj
    Tn, Sn = torch.meshgrid(t_n, s_n, indexing="ij")
    xn, yn, *_ = mapping(Sn, Tn)
    m = CurvilinearMesh(2, ni, nj, 1, nhalo, cell_inv, J, edge_J, edge_hat, [x, y], [xn, yn])
    m.cell_fwd = [xi, xj, yi, yj]
    h = nhalo
    m.L, m.spacing = _phys_dims(2, m.nodes, J[h:h + nj, h:h + ni])
    return m


def tz_wavy_mesh_2d(ni: int, nj: Optional[int] = None, nhalo: int = 5, device="cpu") -> CurvilinearMesh:
    """The wavy grid of the reference's twilight-zone study
    (test/integrated/2d/wavy_manufactured_solution/run.jl:71-96) on [-6, 6]²:
    node (i, j) at x = xmin + Δx0((i−1) + Ax sinpi(n_xy (j−1) Δy0/Ly)),
    y = ymin + Δy0((j−1) + Ay sinpi(n_yx (i−1) Δx0/Lx)), Lx = Ly = 12,
    n_xy = n_yx = 6, Ax = 0.2/Δx0, Ay = 0.4/Δy0, with the metrics evaluated
    exactly from the mapping (the reference builds them with CurvilinearGrids'
    :meg6 scheme).  The forcing of that study (twilight_zone.jl:100-101, :123-124)
    places cell (i, j) at node coordinate i − 4.5, i.e. it assumes 5 halo
    layers, hence the default nhalo."""
    nj = ni if nj is None else nj
    Lx = Ly = 12.0
    dx0, dy0 = Lx / ni, Ly / nj
    kx, ky = math.pi * 6.0 * dy0 / Ly, math.pi * 6.0 * dx0 / Lx

    def mapping(S, T):  # S, T: 0-based node index coordinates along i and j
        x = -Lx / 2 + dx0 * S + 0.2 * torch.sin(kx * T)
        y = -Ly / 2 + dy0 * T + 0.4 * torch.sin(ky * S)
        xi, xj = torch.full_like(S, dx0), 0.2 * kx * torch.cos(kx * T)
        yi, yj = 0.4 * ky * torch.cos(ky * S), torch.full_like(T, dy0)
        return x, y, xi, xj, yi, yj

    def at(off_i, off_j):
        s = torch.arange(ni + 2 * nhalo, dtype=torch.float64, device=device) - nhalo + off_i
        t = torch.arange(nj + 2 * nhalo, dtype=torch.float64, device=device) - nhalo + off_j
        T, S = torch.meshgrid(t, s, indexing="ij")
        return mapping(S, T)

    x, y, xi, xj, yi, yj = at(0.5, 0.5)
    J = xi * yj - xj * yi
    cell_inv = [yj / J, -xj / J, None, -yi / J, xi / J, None, None, None, None]
    edge_J, edge_hat = [None] * 3, [[None] * 9 for _ in range(3)]
    for f, (oi, oj) in enumerate(((1.0, 0.5), (0.5, 1.0))):
        _, _, fxi, fxj, fyi, fyj = at(oi, oj)
        edge_J[f] = fxi * fyj - fxj * fyi
        edge_hat[f][0], edge_hat[f][1] = fyj, -fxj
        edge_hat[f][3], edge_hat[f][4] = -fyi, fxi
    Tn, Sn = torch.meshgrid(torch.arange(nj + 1, dtype=torch.float64, device=device),
                            torch.arange(ni + 1, dtype=torch.float64, device=device), indexing="ij")
    xn, yn, *_ = mapping(Sn, Tn)
    m = CurvilinearMesh(2, ni, nj, 1, nhalo, cell_inv, J, edge_J, edge_hat, [x, y], [xn, yn])
    m.cell_fwd = [xi, xj, yi, yj]
    h = nhalo
    m.L, m.spacing = _phys_dims(2, m.nodes, J[h:h + nj, h:h + ni])
    return m


def _jacobian_3d(dP, ns):
    """Index-space Jacobian M[c][d] = ∂x_c/∂ξ_d of x_c = s_c + a P(s)."""
    return [[((1.0 if c == d else 0.0) + dP[d]) / ns[d] for d in range(3)] for c in range(3)]


def _adjugate_3d(M):
    """adj(M)[a][c] so that ∇ξ_a = adj(M)[a] / det(M) (rows of the inverse)."""
    A = [[None] * 3 for _ in range(3)]
    for a in range(3):
        for c in range(3):
            r0, r1 = [r for r in range(3) if r != c]
            c0, c1 = [q for q in range(3) if q != a]
            minor = M[r0][c0] * M[r1][c1] - M[r0][c1] * M[r1][c0]
            A[a][c] = minor if (a + c) % 2 == 0 else -minor
    det = M[0][0] * A[0][0] + M[0][1] * A[1][0] + M[0][2] * A[2][0]
    return A, det


def wavy_mesh_3d(ni: int, nj: int, nk: int, amp: float = 0.04, nhalo: int = 1,
                 device="cpu") -> CurvilinearMesh:
    """x_c = ξ_c + a sin(2πξ) sin(2πη) sin(2πζ) for each coordinate, on [0,1]³."""
    ns = (ni, nj, nk)

    def fields(off):
        s = _index_grid(ni, nhalo, off[0], device)
        t = _index_grid(nj, nhalo, off[1], device)
        u = _index_grid(nk, nhalo, off[2], device)
        U, T, S = torch.meshgrid(u, t, s, indexing="ij")  # (nz, ny, nx)
        sn = [torch.sin(TWO_PI * v) for v in (S, T, U)]
        cn = [torch.cos(TWO_PI * v) for v in (S, T, U)]
        P = amp * sn[0] * sn[1] * sn[2]
        dP = [amp * TWO_PI * cn[0] * sn[1] * sn[2], amp * TWO_PI * sn[0] * cn[1] * sn[2],
              amp * TWO_PI * sn[0] * sn[1] * cn[2]]
        return (S + P, T + P, U + P), dP

    (x, y, z), dP = fields((0.5, 0.5, 0.5))
    A, J = _adjugate_3d(_jacobian_3d(dP, ns))
    cell_inv = [A[a][c] / J for a in range(3) for c in range(3)]
    edge_J, edge_hat = [None] * 3, [[None] * 9 for _ in range(3)]
    for f in range(3):
        off = [0.5, 0.5, 0.5]
        off[f] = 1.0
        _, dPf = fields(off)
        Af, Jf = _adjugate_3d(_jacobian_3d(dPf, ns))
        edge_J[f] = Jf
        edge_hat[f] = [Af[a][c] for a in range(3) for c in range(3)]
        del dPf
    sn = [torch.arange(n + 1, dtype=torch.float64, device=device) / n for n in ns]
    Un, Tn, Sn = torch.meshgrid(sn[2], sn[1], sn[0], indexing="ij")
    Pn = amp * torch.sin(TWO_PI * Sn) * torch.sin(TWO_PI * Tn) * torch.sin(TWO_PI * Un)
    nodes = [Sn + Pn, Tn + Pn, Un + Pn]
    m = CurvilinearMesh(3, ni, nj, nk, nhalo, cell_inv, J, edge_J, edge_hat, [x, y, z], nodes)
    m.L, m.spacing = _phys_dims(3, nodes, None)
    return m


def uniform_mesh_2d(ni: int, nj: int, lx: float = 1.0, ly: float = 1.0, nhalo: int = 1,
                    device="cpu") -> CurvilinearMesh:
    """Rectilinear mesh (RectlinearGrid in the reference's tests)."""
    m = wavy_mesh_2d(ni, nj, amp=0.0, nhalo=nhalo, device=device)
    sx, sy = lx, ly
    m.cell_inv[0] = m.cell_inv[0] / sx
    m.cell_inv[4] = m.cell_inv[4] / sy
    m.cell_J = m.cell_J * sx * sy
    for f in range(2):
        m.edge_J[f] = m.edge_J[f] * sx * sy
        m.edge_hat[f][0] = m.edge_hat[f][0] * sy
        m.edge_hat[f][4] = m.edge_hat[f][4] * sx
    m.centroids = [m.centroids[0] * sx, m.centroids[1] * sy]
    m.nodes = [m.nodes[0] * sx, m.nodes[1] * sy]
    h = nhalo
    m.L, m.spacing = _phys_dims(2, m.nodes, m.cell_J[h:h + nj, h:h + ni])
    return m


def mesh_from_nodes_2d(xn: torch.Tensor, yn: torch.Tensor, nhalo: int = 1) -> CurvilinearMesh:
    """Second-order metrics from domain node coordinates of shape (nj+1, ni+1).

    Halo nodes are extrapolated linearly.  Cell-centre derivatives average the
    two opposite edges of the cell; at a face, the derivative along the face is
    the exact edge difference and the one across it averages the two cells.
    """
    nj, ni = xn.shape[0] - 1, xn.shape[1] - 1
    h = nhalo
    ny, nx = nj + 2 * h, ni + 2 * h
    X, Y = _extrapolate_2d(xn, h + 1), _extrapolate_2d(yn, h + 1)   # (ny+3, nx+3)

    def cell_d(A):  # over (ny+1, nx+1) cells: the full cells plus one ring on the high side
        a00, a10 = A[1:ny + 2, 1:nx + 2], A[1:ny + 2, 2:nx + 3]
        a01, a11 = A[2:ny + 3, 1:nx + 2], A[2:ny + 3, 2:nx + 3]
        return (0.5 * ((a10 - a00) + (a11 - a01)), 0.5 * ((a01 - a00) + (a11 - a10)),
                0.25 * (a00 + a10 + a01 + a11))

    xi, xj, xc = cell_d(X)
    yi, yj, yc = cell_d(Y)
    c = (slice(0, ny), slice(0, nx))
    J = xi * yj - xj * yi
    cell_inv = [(yj / J)[c], (-xj / J)[c], None, (-yi / J)[c], (xi / J)[c], None, None, None, None]
    # face i+1/2 of full cell (I, J)
    fxj = X[2:ny + 2, 2:nx + 2] - X[1:ny + 1, 2:nx + 2]
    fyj = Y[2:ny + 2, 2:nx + 2] - Y[1:ny + 1, 2:nx + 2]
    fxi = 0.5 * (xi[0:ny, 0:nx] + xi[0:ny, 1:nx + 1])
    fyi = 0.5 * (yi[0:ny, 0:nx] + yi[0:ny, 1:nx + 1])
    # face j+1/2 of full cell (I, J)
    gxi = X[2:ny + 2, 2:nx + 2] - X[2:ny + 2, 1:nx + 1]
    gyi = Y[2:ny + 2, 2:nx + 2] - Y[2:ny + 2, 1:nx + 1]
    gxj = 0.5 * (xj[0:ny, 0:nx] + xj[1:ny + 1, 0:nx])
    gyj = 0.5 * (yj[0:ny, 0:nx] + yj[1:ny + 1, 0:nx])
    edge_J = [fxi * fyj - fxj * fyi, gxi * gyj - gxj * gyi, None]
    edge_hat = [[fyj, -fxj, None, -fyi, fxi, None, None, None, None],
                [gyj, -gxj, None, -gyi, gxi, None, None, None, None], [None] * 9]
    cont = lambda t: None if t is None else t.contiguous()
    m = CurvilinearMesh(2, ni, nj, 1, h, [cont(t) for t in cell_inv], J[c].contiguous(),
                        [cont(t) for t in edge_J], [[cont(t) for t in row] for row in edge_hat],
                        [xc[c].contiguous(), yc[c].contiguous()], [xn, yn])
    m.L, m.spacing = _phys_dims(2, m.nodes, m.cell_J[h:h + nj, h:h + ni])
    return m


def _extrapolate_2d(a: torch.Tensor, p: int) -> torch.Tensor:
    """Pad a node array by p layers on each side by linear extrapolation."""
    for dim in (0, 1):
        lo = a.narrow(dim, 0, 1)
        d_lo = a.narrow(dim, 1, 1) - lo
        hi = a.narrow(dim, a.shape[dim] - 1, 1)
        d_hi = hi - a.narrow(dim, a.shape[dim] - 2, 1)
        los = [lo - (p - r) * d_lo for r in range(p)]
        his = [hi + (r + 1) * d_hi for r in range(p)]
        a = torch.cat(los + [a] + his, dim=dim)
    return a
