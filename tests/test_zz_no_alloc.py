"""The allocation-free end-of-step reductions, through the C ABI.

cdm_step_reductions_noalloc serves callers that cannot allocate device memory
while they run — for example a Julia host whose CUDA.jl memory pool owns the
device memory, or a service that forbids allocation on its latency path.  It
recomputes next_dt and the energy balance of a time step from arrays the
caller owns, with scratch that lives inside the library.  These tests compare
it with what cdm_apt_step itself reported for the same step, on two calls in a
row (the scratch keeps the previous call's contents, which must not matter).
This file is collected last so that a failure here comes after every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from helpers import small_case_2d, small_case_3d
from curvilineardiffusionmanuscript_b200 import _lib as L
from curvilineardiffusionmanuscript_b200.solver import PseudoTransientSolver, step

pytestmark = pytest.mark.gpu


def noalloc(mesh, u_new, u_prev, rho, S, J, cp, dt, tol=1e-3, max_change=0.05, growth=1.1):
    out = (C.c_double * 4)()
    nk = mesh.nk if mesh.ndim == 3 else 1
    rc = L.load().cdm_step_reductions_noalloc(mesh.ndim, mesh.ni, mesh.nj, nk, mesh.nhalo, u_new.data_ptr(),
                                              u_prev.data_ptr(), rho.data_ptr(),
                                              S.data_ptr() if S is not None else None, J.data_ptr(), cp, dt, tol,
                                              max_change, growth, out, None)
    assert rc == 0, L.last_error()
    return list(out)


@pytest.mark.parametrize("case", ["2d", "2d_source", "3d"])
def test_noalloc_matches_step(case):
    source = case == "2d_source"
    pr = small_case_3d(n=(41, 30, 23)) if case == "3d" else small_case_2d(ni=150, nj=97, source=source)
    g = PseudoTransientSolver(pr.mesh, pr.bcs)
    S = pr.source.cuda() if source else None
    if source:
        g.set_source(S)
    u_prev = pr.T0.clone().cuda()
    T = u_prev.clone()
    rho = pr.rho.cuda()
    stats, next_dt = step(g, pr.mesh, T, rho, pr.cp, pr.kappa, pr.dt, rtol=1e-8, atol=1e-8)
    J = pr.mesh.cell_J.cuda()
    for _ in range(2):  # two calls in a row share the scratch
        nd, e0, e1, sw = noalloc(pr.mesh, T, u_prev, rho, S, J, pr.cp, pr.dt)
        assert nd == pytest.approx(next_dt, rel=1e-14, abs=0.0)
        assert e0 == pytest.approx(stats["energy_before"], rel=1e-12)
        assert e1 == pytest.approx(stats["energy_after"], rel=1e-12)
        if source:
            assert sw == pytest.approx(stats["source_work"], rel=1e-12)


def test_noalloc_rejects_oversized_mesh():
    z = torch.zeros(1, dtype=torch.float64, device="cuda")
    out = (C.c_double * 4)()
    rc = L.load().cdm_step_reductions_noalloc(2, 20000, 20000, 1, 1, z.data_ptr(), z.data_ptr(), z.data_ptr(),
                                              None, z.data_ptr(), 1.0, 1e-5, 1e-3, 0.05, 1.1, out, None)
    assert rc == L.CDM_BAD_INPUT
    assert "at most" in L.last_error()


def test_noalloc_rejects_host_and_short_arrays():
    """Arrays the device cannot read over the full mesh are refused before
    anything is launched: a host array, and a device array shorter than the
    full array (larger than the allocation it sits in)."""
    pr = small_case_2d(ni=40, nj=30)
    J = pr.mesh.cell_J.cuda()
    u = pr.T0.clone().cuda()
    rho = pr.rho.cuda()
    lib = L.load()
    out = (C.c_double * 4)()
    host = pr.T0.clone()
    rc = lib.cdm_step_reductions_noalloc(2, 40, 30, 1, 1, u.data_ptr(), host.data_ptr(), rho.data_ptr(), None,
                                         J.data_ptr(), 1.0, 1e-5, 1e-3, 0.05, 1.1, out, None)
    assert rc == L.CDM_BAD_INPUT and "u_prev" in L.last_error()
    short = torch.zeros(1000, dtype=torch.float64, device="cuda")
    rc = lib.cdm_step_reductions_noalloc(2, 2000, 2000, 1, 1, short.data_ptr(), short.data_ptr(), short.data_ptr(),
                                         None, short.data_ptr(), 1.0, 1e-5, 1e-3, 0.05, 1.1, out, None)
    assert rc == L.CDM_BAD_INPUT and "holds" in L.last_error()
    # the entry point still works afterwards
    nd, *_ = noalloc(pr.mesh, u, u.clone(), rho, None, J, 1.0, 1e-5)
    assert nd == pytest.approx(1.1e-5, rel=1e-15)
