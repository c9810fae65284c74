"""CPU checks of the implicit-scheme oracle (oracle/implicit_oracle.py), the
checker of the library's implicit comparator: known answers of the
conservative curvilinear stencil (stencils.jl:14-40, edge_terms.jl:31-87)."""
import numpy as np

from helpers import small_case_2d
from oracle.implicit_oracle import ImplicitOracle
from curvilineardiffusionmanuscript_b200.mesh import wavy_mesh_2d
from curvilineardiffusionmanuscript_b200.solver import DirichletBC, NeumannBC, PeriodicBC


def _assemble(pr, dt=None):
    o = ImplicitOracle(pr.mesh, pr.bcs)
    T, rho = pr.T0.numpy().copy(), pr.rho.numpy().copy()
    from oracle.oracle import applybcs
    m = pr.mesh
    nk = m.nk if m.ndim == 3 else 1
    applybcs(m.ndim, m.ni, m.nj, nk, m.nhalo, pr.bcs, T)
    applybcs(m.ndim, m.ni, m.nj, nk, m.nhalo, pr.bcs, rho)
    A, b, c, alpha = o.assemble(T, rho, pr.cp, pr.kappa.k0, pr.kappa.n, dt or pr.dt)
    return o, A, b, c, alpha


def test_stencil_rows_sum_to_the_cell_volume():
    """The conservative form: every flux term appears with both signs, so an
    interior row applied to a constant field gives J (wavy mesh, κ = T³)."""
    pr = small_case_2d(ni=31, nj=23, amp=0.07)
    o, A, b, c, _ = _assemble(pr, dt=1e-3)
    J = o._r2(pr.mesh.cell_J)[1:-1, 1:-1]
    rows = c[:, 1:-1, 1:-1].sum(axis=0)
    assert np.max(np.abs(rows - J) / J) < 1e-11
    # boundary rows: Neumann constraints annihilate constants too
    y = (A @ np.ones(o.N)).reshape(o.n2, o.n1)
    assert np.allclose(y[0, 1:-1], 0.0) and np.allclose(y[1:-1, 0], 0.0)


def test_uniform_mesh_gives_the_five_point_operator():
    """Rectilinear h x h cells, constant α: no cross terms, neighbour entries
    -αΔt, diagonal J + 4αΔt."""
    n = 12
    m = wavy_mesh_2d(n, n, amp=0.0)
    x, y = m.centroids
    import torch
    from curvilineardiffusionmanuscript_b200 import problems
    from curvilineardiffusionmanuscript_b200.solver import PowerLawConductivity
    T0 = (1.0 + 0.0 * x).contiguous()
    pr = problems.Problem("u", m, [NeumannBC()] * 4, T0, torch.ones_like(T0), 1.0, PowerLawConductivity(2.0, 0.0),
                          1e-3, 1)
    o, A, b, c, alpha = _assemble(pr)
    I = (slice(1, -1), slice(1, -1))
    h2 = (1.0 / n) ** 2
    for e in (0, 2, 6, 8):
        assert np.max(np.abs(c[e][I])) < 1e-17
    for e in (1, 3, 5, 7):
        assert np.allclose(c[e][I], -2.0 * 1e-3, rtol=1e-12)
    assert np.allclose(c[4][I], h2 + 8.0 * 1e-3, rtol=1e-12)
    assert np.allclose(b.reshape(o.n2, o.n1)[I], h2, rtol=1e-12)


def test_boundary_rows_follow_the_side_kinds():
    pr = small_case_2d(ni=9, nj=7, bcs=[DirichletBC(1.5), DirichletBC(0.5), PeriodicBC(), PeriodicBC()])
    o, A, b, c, _ = _assemble(pr)
    b2 = b.reshape(o.n2, o.n1)
    assert np.all(b2[:, 0] == 1.5) and np.all(b2[:, -1] == 0.5)  # ilo/ihi first, corners included
    assert np.all(b2[0, 1:-1] == 0.0) and np.all(b2[-1, 1:-1] == 0.0)
    A = A.tocsr()
    r = 0 * o.n1 + 3  # jlo row, i = 3: periodic partner (3, nj) with -1
    assert A[r, r] == 1.0 and A[r, (o.n2 - 2) * o.n1 + 3] == -1.0 and A[r].nnz == 2
    r = 4 * o.n1  # ilo row (Dirichlet): the diagonal only
    assert A[r].nnz == 1 and A[r, r] == 1.0


def test_small_time_step_returns_the_input():
    pr = small_case_2d(ni=16, nj=16)
    o = ImplicitOracle(pr.mesh, pr.bcs)
    T = pr.T0.numpy().copy()
    o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, 1e-16)
    d = o._r2(T)[1:-1, 1:-1] - o._r2(pr.T0.numpy())[1:-1, 1:-1]
    assert np.max(np.abs(d)) < 1e-8


def test_3d_rows_sum_to_the_cell_volume_and_uniform_seven_point():
    from helpers import small_case_3d
    from curvilineardiffusionmanuscript_b200.mesh import wavy_mesh_3d
    pr = small_case_3d(n=(9, 8, 7), amp=0.06)
    o, A, b, c, _ = _assemble(pr, dt=1e-3)
    I = (slice(1, -1),) * 3
    J = o._r2(pr.mesh.cell_J)[I]
    assert np.max(np.abs(c[(slice(None),) + I].sum(axis=0) - J) / J) < 1e-11
    corners = [s for s in range(27) if s in (0, 2, 6, 8, 18, 20, 24, 26)]
    assert all(np.all(c[s] == 0.0) for s in corners)  # stencils.jl:75-82
    # uniform mesh, constant α: the seven-point operator
    import torch
    from curvilineardiffusionmanuscript_b200 import problems
    from curvilineardiffusionmanuscript_b200.solver import PowerLawConductivity
    n = 6
    m = wavy_mesh_3d(n, n, n, amp=0.0, nhalo=1)
    T0 = torch.ones_like(m.cell_J).contiguous()
    pru = problems.Problem("u3", m, [NeumannBC()] * 6, T0, torch.ones_like(T0), 1.0,
                           PowerLawConductivity(2.0, 0.0), 1e-3, 1)
    o, A, b, c, _ = _assemble(pru)
    h3 = (1.0 / n) ** 3
    h = 1.0 / n
    face = [4, 10, 12, 14, 16, 22]
    for s in range(27):
        if s == 13:
            assert np.allclose(c[s][I], h3 + 6 * 2.0 * h * 1e-3, rtol=1e-12)
        elif s in face:
            assert np.allclose(c[s][I], -2.0 * h * 1e-3, rtol=1e-12)
        else:
            assert np.max(np.abs(c[s][I])) < 1e-17


def test_oracle_matches_its_golden_fixtures():
    """The implicit oracle's stencil entries, right-hand sides and solutions of
    two steps (tests/golden/make_golden.py) against regressions: the entries and
    b bit for bit, the direct solutions to rounding."""
    import sys
    from pathlib import Path
    here = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(here))
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", here / "make_golden.py")
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    for name, sp in mg.IMPLICIT_CASES.items():
        ref = np.load(here / f"{name}.npz")
        res = mg.run_implicit(name, sp)
        assert np.array_equal(res["c"], ref["c"]) and np.array_equal(res["b"], ref["b"]), name
        assert np.max(np.abs(res["T"] - ref["T"])) <= 1e-12 * np.max(np.abs(ref["T"])), name
        assert np.allclose(res["next_dt"], ref["next_dt"], rtol=1e-10), name


def test_3d_boundary_rows_follow_the_side_kinds():
    """init_matrix.jl:252-390: each side's rows over the interior range of the
    other two axes; Neumann and periodic rows pair with the interior / opposite
    cell, Dirichlet rows and edge or corner rows keep the diagonal only."""
    from helpers import small_case_3d
    bcs = [DirichletBC(1.5), NeumannBC(), NeumannBC(), NeumannBC(), PeriodicBC(), PeriodicBC()]
    pr = small_case_3d(n=(5, 4, 6), bcs=bcs)
    o, A, b, c, _ = _assemble(pr)
    A = A.tocsr()
    n1, n2, n3 = o.n1, o.n2, o.n3
    rid = lambda i, j, k: i + n1 * (j + n2 * k)
    r = rid(0, 2, 3)  # ilo, Dirichlet: the diagonal only, b = 1.5
    assert A[r].nnz == 1 and A[r, r] == 1.0 and b[r] == 1.5
    r = rid(n1 - 1, 2, 3)  # ihi, Neumann: -1 at the interior neighbour
    assert A[r].nnz == 2 and A[r, rid(n1 - 2, 2, 3)] == -1.0 and b[r] == 0.0
    r = rid(2, 1, 0)  # klo, periodic: -1 at (i, j, khi - 1)
    assert A[r].nnz == 2 and A[r, rid(2, 1, n3 - 2)] == -1.0
    r = rid(2, 1, n3 - 1)  # khi, periodic: -1 at (i, j, klo + 1)
    assert A[r].nnz == 2 and A[r, rid(2, 1, 1)] == -1.0
    r = rid(0, 0, 2)  # an edge (ilo and jlo): the diagonal only, bc_operator takes ilo first
    assert A[r].nnz == 1 and b[r] == 1.5
