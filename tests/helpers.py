"""Shared helpers of the test-suite (seeded cases, oracle vs library runs)."""
from __future__ import annotations

import math

import numpy as np
import torch

from curvilineardiffusionmanuscript_b200 import problems
from curvilineardiffusionmanuscript_b200.mesh import wavy_mesh_2d, wavy_mesh_3d
from curvilineardiffusionmanuscript_b200.solver import (DirichletBC, FixedNegSymmetryBC, NeumannBC, PeriodicBC,
                                                        PowerLawConductivity)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_case_2d(ni=24, nj=17, amp=0.05, kn=3.0, bcs=None, seed=0, nhalo=1, source=False):
    """Seeded small 2D problem on the wavy mesh."""
    m = wavy_mesh_2d(ni, nj, amp, nhalo=nhalo)
    x, y = m.centroids
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.3, 0.7, size=2)
    T0 = (1.0 + 10.0 * torch.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2) / 0.02)).contiguous()
    rho = (1.0 + 0.1 * torch.sin(3.0 * x) * torch.cos(2.0 * y)).contiguous()
    bcs = bcs or [NeumannBC(), NeumannBC(), NeumannBC(), NeumannBC()]
    S = None
    if source:
        S = (5.0 * torch.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2) / 0.05)).contiguous()
    return problems.Problem("small2d", m, bcs, T0, rho, 1.3, PowerLawConductivity(1.0, kn), 1e-5, 3,
                            source=S)


def small_case_3d(n=(10, 9, 8), amp=0.04, kn=2.5, bcs=None):
    m = wavy_mesh_3d(*n, amp=amp, nhalo=1)
    x, y, z = m.centroids
    T0 = (1.0 + 10.0 * torch.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2) / 0.05)).contiguous()
    rho = torch.ones_like(T0)
    bcs = bcs or [NeumannBC() for _ in range(6)]
    return problems.Problem("small3d", m, bcs, T0, rho, 1.0, PowerLawConductivity(1.0, kn), 1e-5, 3)


def decaying_mode_error(n, run_steps, nsteps=10, dt=2e-6, ndim=2):
    """Known answer of the reference's analytic case: u = sin(3πx)·exp(−9π²t)
    with κ = 1, ρ = cₚ = 1, negative-symmetry ghosts on the x sides (u = 0 at
    the walls) and periodic other sides, on a rectilinear mesh of n cells per
    side of [0,1]^ndim.
    `run_steps(mesh, bcs, T0, rho, dt, nsteps)` advances T0 and returns the
    domain field; the result is the RMS error against the exact solution."""
    m = wavy_mesh_2d(n, n, 0.0) if ndim == 2 else wavy_mesh_3d(n, n, n, amp=0.0)
    x = m.centroids[0]
    T0 = torch.sin(3 * math.pi * x).contiguous()
    rho = torch.ones_like(T0)
    bcs = [FixedNegSymmetryBC(), FixedNegSymmetryBC()] + [PeriodicBC()] * (2 * ndim - 2)
    T = run_steps(m, bcs, T0, rho, dt, nsteps)
    exact = (torch.sin(3 * math.pi * x) * math.exp(-9 * math.pi ** 2 * dt * nsteps))[m.domain()]
    d = np.asarray(T, dtype=np.float64) - exact.numpy()
    return float(np.sqrt((d * d).mean()))


def richardson_order(run_steps, sizes=(9, 27, 81), dt=1e-3, nsteps=5):
    """The reference's Richardson study (test/integrated/2d/richardson_wavy_2D/run.jl:
    κ = 2.5, Neumann sides, wavy mesh, grids refined by 3 so that coarse cell centres
    are fine cell centres): log₃ of ‖u_h − u_{h/3}‖∞ / ‖u_{h/3} − u_{h/9}‖∞ on the
    coarse points, for a pulse 1 + exp(−|x − (½, ½)|²/0.05) that stays off the walls.
    `run_steps(mesh, bcs, T0, rho, dt, nsteps)` returns the domain field."""
    u = []
    for n in sizes:
        m = wavy_mesh_2d(n, n, 0.05)
        x, y = m.centroids
        T0 = (1.0 + torch.exp(-((x - 0.5) ** 2 + (y - 0.5) ** 2) / 0.05)).contiguous()
        u.append(np.asarray(run_steps(m, [NeumannBC()] * 4, T0, torch.ones_like(T0), dt, nsteps)))
    c0, c1, c2 = u[0], u[1][1::3, 1::3], u[2][4::9, 4::9]
    return math.log(np.abs(c0 - c1).max() / np.abs(c1 - c2).max(), 3)
