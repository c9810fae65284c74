"""Python mirror of the reference's APT interface, running on the B200 library.

Reference interface (smillerc/CurvilinearDiffusionManuscript):

* ``PseudoTransientSolver(mesh, bcs; backend, mean=:harmonic, T=Float64)``
  — src/pseudo_transient/PseudoTransientSolver.jl:48-103
* ``step!(solver, mesh, T, ρ, cₚ, κ, dt; kwargs...) -> (stats, next_Δt)``
  — PseudoTransientSolver.jl:180-351
* ``nonlinear_thermal_conduction_step!(solver, mesh, T, ρ, cₚ, κ, Δt; ...)``
  — src/nonlinear_thermal_conduction.jl:51-72
* boundary-condition types — src/boundary_conditions/boundary_operators.jl:9-17

Every call goes through the C ABI of ``libcdm_apt.so``; nothing here computes
the solution.  Like the reference, a failed step raises an error (the
reference calls ``error(...)``; here :class:`APTError` carries the status).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Dict, Iterable, List, Optional, Sequence, Union

import numpy as np
import torch

from . import _lib as L
from .mesh import CurvilinearMesh


# --------------------------------------------------------------------------- BCs
class NeumannBC:
    """Ghost cell <- adjacent interior cell (boundary_operators.jl:55-119)."""
    kind = L.CDM_BC_NEUMANN
    value = 0.0


class DirichletBC:
    """Ghost cells <- val (boundary_operators.jl:137-155, :178-200)."""
    kind = L.CDM_BC_DIRICHLET

    def __init__(self, val: float):
        self.value = float(val)


class PeriodicBC:
    """Ghost cells <- opposite interior; acts at LO locations (boundary_operators.jl:220-263)."""
    kind = L.CDM_BC_PERIODIC
    value = 0.0


class FixedNegSymmetryBC:
    """Ghost cell <- -adjacent interior (boundary_operators.jl:157-175)."""
    kind = L.CDM_BC_NEG_SYMMETRY
    value = 0.0


BCType = Union[NeumannBC, DirichletBC, PeriodicBC, FixedNegSymmetryBC]


def bc_list(bcs) -> List[BCType]:
    """The reference enumerates the bcs NamedTuple: position, not name, is the location."""
    if isinstance(bcs, dict):
        return list(bcs.values())
    return list(bcs)


# ------------------------------------------------------------------ conductivity
@dataclass(frozen=True)
class PowerLawConductivity:
    """κ(ρ, T) = k0·|T|ⁿ, 0 for non-finite T (the drivers' closures, e.g.
    test/integrated/2d/gaussian/run.jl:129-135)."""
    k0: float = 1.0
    n: float = 0.0

    def __call__(self, rho, T):
        T = np.asarray(T, dtype=np.float64)
        out = self.k0 * np.abs(T) ** self.n
        return np.where(np.isfinite(T), out, 0.0)

    def as_c(self) -> L.Kappa:
        return L.Kappa(self.k0, self.n)


class APTError(RuntimeError):
    def __init__(self, status: int, message: str, stats: Optional[dict] = None):
        super().__init__(f"{L.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.stats = stats


# ----------------------------------------------------------------------- helpers
def _ptr(a) -> int:
    if isinstance(a, torch.Tensor):
        if a.dtype != torch.float64 or not a.is_contiguous():
            raise ValueError("arrays must be contiguous float64")
        if a.is_cuda:
            _order_after_torch(a.device)
        return a.data_ptr()
    if isinstance(a, np.ndarray):
        if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous float64")
        return a.ctypes.data
    raise TypeError(f"unsupported array type {type(a)}")


def _order_after_torch(device) -> None:
    """The library orders its reads after the legacy default stream (torch's
    default stream); work queued on another torch stream is waited for here."""
    cur = torch.cuda.current_stream(device)
    if cur.cuda_stream != 0:
        cur.synchronize()


def _mem(a) -> int:
    return L.CDM_MEM_DEVICE if isinstance(a, torch.Tensor) and a.is_cuda else L.CDM_MEM_HOST


def mesh_desc(mesh: CurvilinearMesh):
    """cdm_mesh_desc for a mesh; returns (desc, keepalive)."""
    d = L.MeshDesc()
    keep = []
    d.ndim, d.ni, d.nj, d.nk, d.nhalo = mesh.ndim, mesh.ni, mesh.nj, mesh.nk, mesh.nhalo
    d.mem = _mem(mesh.cell_J)

    def p(t):
        if t is None:
            return None
        t = t.contiguous()
        keep.append(t)
        return _ptr(t)

    for k in range(9):
        d.cell_inv[k] = p(mesh.cell_inv[k])
    d.cell_J = p(mesh.cell_J)
    for f in range(3):
        d.edge_J[f] = p(mesh.edge_J[f])
        for k in range(9):
            d.edge_hat[f][k] = p(mesh.edge_hat[f][k])
    d.L = mesh.L
    for k in range(3):
        d.spacing[k] = float(mesh.spacing[k]) if k < len(mesh.spacing) else 0.0
    return d, keep


def tz_desc(mesh: CurvilinearMesh, nnodes=None):
    """cdm_tz_desc of a 2D mesh with forward metrics; returns (desc, keepalive)."""
    if mesh.ndim != 2 or mesh.cell_fwd is None:
        raise ValueError("the twilight-zone forcing needs a 2D mesh with forward metrics (mesh.cell_fwd)")
    d = L.TzDesc()
    keep = [t.contiguous() for t in (*mesh.centroids[:2], *mesh.cell_fwd)]
    d.mem = _mem(keep[0])
    nn = nnodes or mesh.nnodes
    d.nnodes[0], d.nnodes[1] = int(nn[0]), int(nn[1])
    d.x, d.y, d.x_xi, d.x_eta, d.y_xi, d.y_eta = [_ptr(t) for t in keep]
    return d, keep


def _bcs_c(bcs, ndim) -> "C.Array":
    lst = bc_list(bcs)
    if len(lst) != 2 * ndim:
        raise ValueError(f"expected {2 * ndim} boundary conditions, got {len(lst)}")
    arr = (L.BC * len(lst))()
    for i, b in enumerate(lst):
        arr[i].kind = b.kind
        arr[i].value = float(getattr(b, "value", 0.0))
    return arr


_STEP_KW = {
    "t": float, "tz": int, "tz_dim": int, "no_t": int, "max_iter": int, "rtol": float, "atol": float,
    "error_check_interval": int, "apply_cutoff": int, "calculate_next_dt": int,
    "subcycle_conductivity": int, "enforce_positivity": int, "CFL": float,
    "norm": int, "check_every": int, "guess": int, "iter_block": int, "use_graph": int,
}
_NEXT_DT_KW = {"tol": "ndt_tol", "maximum_u_change": "maximum_u_change",
               "timestep_growth_factor": "timestep_growth_factor"}


def step_opts(**kwargs) -> L.StepOpts:
    o = L.default_opts()
    for k, v in kwargs.items():
        if k in _STEP_KW:
            setattr(o, k, _STEP_KW[k](v))
        elif k in _NEXT_DT_KW:
            setattr(o, _NEXT_DT_KW[k], float(v))
        elif k == "norm_kind":
            o.norm = {"max": L.CDM_NORM_MAX, "rms": L.CDM_NORM_RMS}[v]
        # other keywords are accepted and ignored, like the reference's kwargs...
    return o


def stats_dict(s: L.Stats) -> dict:
    return {"rel_err": s.rel_err, "abs_err": s.abs_err, "niter": s.niter, "time": s.time,
            "status": s.status, "energy_before": s.energy_before, "energy_after": s.energy_after,
            "source_work": s.source_work, "n_restarts": s.n_restarts, "n_checks": s.n_checks}


# ------------------------------------------------------------------------ solver
class PseudoTransientSolver:
    """PseudoTransientSolver(mesh, bcs; mean=:harmonic, T=Float64) on one B200."""

    def __init__(self, mesh: CurvilinearMesh, bcs, backend: str = "cuda", mean: str = "harmonic",
                 T=torch.float64, precision: str = "fp64", device: int = 0, stream: Optional[int] = None):
        if T not in (torch.float64, np.float64, float):
            raise ValueError("the APT library computes in Float64 (precision='mixed' for FP32 sweeps)")
        self._lib = L.load()
        self.mesh = mesh
        self.bcs = bc_list(bcs)
        cfg = L.default_config()
        cfg.mean = L.CDM_MEAN_HARMONIC if mean == "harmonic" else L.CDM_MEAN_ARITHMETIC
        cfg.precision = {"fp64": L.CDM_PREC_FP64, "mixed": L.CDM_PREC_MIXED,
                         "fp64_exact": L.CDM_PREC_FP64_EXACT}[precision]
        cfg.device = device
        cfg.stream = stream
        desc, keep = mesh_desc(mesh)
        h = C.c_void_p()
        rc = self._lib.cdm_apt_create(C.byref(desc), _bcs_c(self.bcs, mesh.ndim), C.byref(cfg), C.byref(h))
        del keep
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        self._h = h
        self.nfull = mesh.ncells_full

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cdm_apt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # solver.source_term (PseudoTransientSolver.jl:31)
    def set_source(self, S):
        S = S.contiguous() if isinstance(S, torch.Tensor) else np.ascontiguousarray(S, dtype=np.float64)
        rc = self._lib.cdm_apt_set_source(self._h, _ptr(S), _mem(S))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def set_twilight_zone(self, mesh: Optional[CurvilinearMesh] = None, nnodes=None):
        """Mesh inputs of the tz=True path (define_forcing_wavy, twilight_zone.jl:54-195):
        centroids and forward metrics of `mesh` (default: the solver's), mesh.nnodes."""
        d, keep = tz_desc(mesh or self.mesh, nnodes)
        rc = self._lib.cdm_apt_set_twilight_zone(self._h, C.byref(d))
        del keep
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def set_guess(self, u0):
        u0 = u0.contiguous() if isinstance(u0, torch.Tensor) else np.ascontiguousarray(u0, dtype=np.float64)
        rc = self._lib.cdm_apt_set_guess(self._h, _ptr(u0), _mem(u0))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def get_state(self):
        """(q, last_err_check): the state that carries across steps."""
        q = np.zeros((self.mesh.ndim,) + tuple(self.mesh.full_shape), dtype=np.float64)
        last = C.c_int(0)
        rc = self._lib.cdm_apt_get_state(self._h, q.ctypes.data, C.byref(last))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        return q, last.value

    def set_state(self, q: np.ndarray, last_err_check: int):
        q = np.ascontiguousarray(q, dtype=np.float64)
        rc = self._lib.cdm_apt_set_state(self._h, q.ctypes.data, int(last_err_check))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def profile(self) -> dict:
        p = L.Profile()
        self._lib.cdm_apt_get_profile(self._h, C.byref(p))
        return {k: getattr(p, k) for k, _ in L.Profile._fields_}

    def metric_cache(self) -> np.ndarray:
        out = np.zeros((self.mesh.ndim,) + tuple(self.mesh.full_shape), dtype=np.float64)
        rc = self._lib.cdm_apt_get_metric_cache(self._h, out.ctypes.data)
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        return out


def step(solver: PseudoTransientSolver, mesh, T, rho, cp: float, kappa: PowerLawConductivity, dt: float,
         **kwargs):
    """step!(solver, mesh, T, ρ, cₚ, κ, dt; kwargs...) -> (stats, next_Δt); T is updated in place."""
    o = step_opts(**kwargs)
    o.mem = _mem(T)
    if _mem(rho) != o.mem:
        raise ValueError("T and rho must live in the same memory space")
    st = L.Stats()
    ndt = C.c_double(0.0)
    rc = solver._lib.cdm_apt_step(solver._h, _ptr(T), _ptr(rho), float(cp), kappa.as_c(), float(dt),
                                  C.byref(o), C.byref(st), C.byref(ndt))
    stats = stats_dict(st)
    if rc != L.CDM_OK:
        raise APTError(rc, L.last_error(), stats)
    return stats, ndt.value


def nonlinear_thermal_conduction_step(solver, mesh, T, rho, cp, kappa, dt, *, show_convergence=True, **kwargs):
    """nonlinear_thermal_conduction_step! for the PT solver (nonlinear_thermal_conduction.jl:51-72)
    and, given an :class:`ImplicitScheme`, for the implicit scheme (:4-48)."""
    if isinstance(solver, ImplicitScheme):
        stats, next_dt = solver.step(mesh, T, rho, cp, kappa, dt, **kwargs)
        if show_convergence:
            print("\tKrylov stats: L2: %.1e, iterations: %i" % (stats["abs_err"], stats["niter"]))
        return stats, next_dt
    stats, next_dt = step(solver, mesh, T, rho, cp, kappa, dt, **kwargs)
    if show_convergence:
        print("\trel error: %.3e, abs err: %.3e, %i" % (stats["rel_err"], stats["abs_err"], stats["niter"]))
    return stats, next_dt


# --------------------------------------------------------------- implicit scheme
_IMPLICIT_KW = {"atol": float, "rtol": float, "max_iter": int, "enforce_positivity": int,
                "apply_density_bc": int, "maximum_u_change": float, "timestep_growth_factor": float}


class ImplicitScheme:
    """ImplicitScheme(mesh, bcs; mean=:harmonic) — the reference's implicit
    comparator (src/implicit/ImplictSolver.jl:49-160) on one B200: backward
    Euler with the diffusivity at Tⁿ, one linear system per step solved by a
    Krylov method to ||b - A x|| <= atol + rtol ||b - A x0||."""

    def __init__(self, mesh: CurvilinearMesh, bcs, mean: str = "harmonic", device: int = 0,
                 stream: Optional[int] = None):
        self._lib = L.load()
        self.mesh = mesh
        self.bcs = bc_list(bcs)
        cfg = L.default_config()
        cfg.mean = L.CDM_MEAN_HARMONIC if mean == "harmonic" else L.CDM_MEAN_ARITHMETIC
        cfg.device = device
        cfg.stream = stream
        desc, keep = mesh_desc(mesh)
        h = C.c_void_p()
        rc = self._lib.cdm_implicit_create(C.byref(desc), _bcs_c(self.bcs, mesh.ndim), C.byref(cfg), C.byref(h))
        del keep
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        self._h = h
        self.shape = ((mesh.nk + 2,) if mesh.ndim == 3 else ()) + (mesh.nj + 2, mesh.ni + 2)
        self.rows = int(np.prod(self.shape))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cdm_implicit_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_source(self, S):
        S = S.contiguous() if isinstance(S, torch.Tensor) else np.ascontiguousarray(S, dtype=np.float64)
        rc = self._lib.cdm_implicit_set_source(self._h, _ptr(S), _mem(S))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def step(self, mesh, T, rho, cp: float, kappa: PowerLawConductivity, dt: float, **kwargs):
        """One implicit time step; T is updated in place -> (stats, next_dt)."""
        o = L.ImplicitOpts()
        self._lib.cdm_implicit_opts_default(C.byref(o))
        for k, v in kwargs.items():
            if k in _IMPLICIT_KW:
                setattr(o, k, _IMPLICIT_KW[k](v))
            elif k == "tol":
                o.ndt_tol = float(v)
        o.mem = _mem(T)
        if _mem(rho) != o.mem:
            raise ValueError("T and rho must live in the same memory space")
        st = L.Stats()
        ndt = C.c_double(0.0)
        rc = self._lib.cdm_implicit_step(self._h, _ptr(T), _ptr(rho), float(cp), kappa.as_c(), float(dt),
                                         C.byref(o), C.byref(st), C.byref(ndt))
        stats = stats_dict(st)
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error(), stats)
        return stats, ndt.value

    def system(self):
        """(A, b) of the last step: A as 9 (2D) or 27 (3D) stencil entries over the
        region ([nk+2,] nj+2, ni+2), b over the region."""
        A = np.zeros((9 if self.mesh.ndim == 2 else 27,) + self.shape)
        b = np.zeros(self.shape)
        rc = self._lib.cdm_implicit_get_system(self._h, A.ctypes.data, b.ctypes.data)
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        return A, b

    def profile(self) -> dict:
        ms, spmv, rows = C.c_double(0.0), C.c_int64(0), C.c_int64(0)
        self._lib.cdm_implicit_get_profile(self._h, C.byref(ms), C.byref(spmv), C.byref(rows))
        return {"solve_ms": ms.value, "spmv": spmv.value, "rows": rows.value}


def advance(solver: PseudoTransientSolver, mesh, T, rho, cp: float, kappa: PowerLawConductivity, dt: float,
            t: float = 0.0, t_end: float = math.inf, max_cycles: int = 2 ** 31 - 1, dt_max: float = math.inf,
            **kwargs):
    """The drivers' time loop (test/integrated/2d/gaussian/run.jl:192-231) in one
    library call: -> (t, next_dt, nsteps, last_stats); T is updated in place."""
    o = step_opts(**kwargs)
    o.mem = _mem(T)
    if _mem(rho) != o.mem:
        raise ValueError("T and rho must live in the same memory space")
    st = L.Stats()
    tc, dtc, ns = C.c_double(float(t)), C.c_double(float(dt)), C.c_int(0)
    rc = solver._lib.cdm_apt_advance(solver._h, _ptr(T), _ptr(rho), float(cp), kappa.as_c(), C.byref(tc),
                                     float(t_end), int(max_cycles), C.byref(dtc), float(dt_max), C.byref(o),
                                     C.byref(st), C.byref(ns))
    stats = stats_dict(st)
    if rc != L.CDM_OK:
        raise APTError(rc, L.last_error(), stats)
    return tc.value, dtc.value, ns.value, stats


# ------------------------------------------------------------------------- batch
class PseudoTransientBatch:
    """Many independent PseudoTransientSolver problems advanced by one launch per
    pseudo-iteration (CUDA-graph replays of the fused sweep)."""

    def __init__(self, meshes: Sequence[CurvilinearMesh], bcs_list, mean="harmonic", device=0,
                 stream: Optional[int] = None, precision: str = "fp64"):
        self._lib = L.load()
        self.meshes = list(meshes)
        n = len(self.meshes)
        descs = (L.MeshDesc * n)()
        keep = []
        for i, m in enumerate(self.meshes):
            d, k = mesh_desc(m)
            descs[i] = d
            keep.append(k)
        nd = self.meshes[0].ndim
        bcs = (L.BC * (2 * nd * n))()
        for i, b in enumerate(bcs_list):
            arr = _bcs_c(b, nd)
            for l in range(2 * nd):
                bcs[i * 2 * nd + l] = arr[l]
        cfg = L.default_config()
        cfg.mean = L.CDM_MEAN_HARMONIC if mean == "harmonic" else L.CDM_MEAN_ARITHMETIC
        cfg.device = device
        cfg.stream = stream
        cfg.precision = {"fp64": L.CDM_PREC_FP64, "mixed": L.CDM_PREC_MIXED,
                         "fp64_exact": L.CDM_PREC_FP64_EXACT}[precision]
        h = C.c_void_p()
        rc = self._lib.cdm_batch_create(n, descs, bcs, C.byref(cfg), C.byref(h))
        del keep
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        self._h = h
        self.n = n

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cdm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def profile(self) -> dict:
        p = L.Profile()
        self._lib.cdm_batch_get_profile(self._h, C.byref(p))
        return {k: getattr(p, k) for k, _ in L.Profile._fields_}

    def set_source(self, p: int, S):
        rc = self._lib.cdm_batch_set_source(self._h, p, _ptr(S), _mem(S))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def set_twilight_zone(self, p: int, mesh: Optional[CurvilinearMesh] = None, nnodes=None):
        """PseudoTransientSolver.set_twilight_zone for problem p."""
        d, keep = tz_desc(mesh or self.meshes[p], nnodes)
        rc = self._lib.cdm_batch_set_twilight_zone(self._h, int(p), C.byref(d))
        del keep
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def autotune(self, Ts, rhos, cps, kappas, dts, cache_path: Optional[str] = None, **kwargs) -> int:
        """Time one step per (strip height, iteration block) candidate on these
        inputs and keep the fastest; Ts are not modified.  Returns the candidate index."""
        n = self.n
        o = step_opts(**kwargs)
        o.mem = _mem(Ts[0])
        Tp = (C.c_void_p * n)(*[_ptr(t) for t in Ts])
        Rp = (C.c_void_p * n)(*[_ptr(r) for r in rhos])
        cpa = (C.c_double * n)(*[float(c) for c in cps])
        ka = (L.Kappa * n)(*[k.as_c() for k in kappas])
        dta = (C.c_double * n)(*[float(d) for d in dts])
        ch = C.c_int(-1)
        rc = self._lib.cdm_batch_autotune(self._h, Tp, Rp, cpa, ka, dta, C.byref(o),
                                          cache_path.encode() if cache_path else None, C.byref(ch))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())
        return ch.value

    def set_tuning(self, variant: int = 0, strip_h: int = 0, iter_block: int = 8):
        rc = self._lib.cdm_batch_set_tuning(self._h, int(variant), int(strip_h), int(iter_block))
        if rc != L.CDM_OK:
            raise APTError(rc, L.last_error())

    def tuning(self) -> dict:
        v, h, k = C.c_int(0), C.c_int(0), C.c_int(0)
        self._lib.cdm_batch_tuning(self._h, C.byref(v), C.byref(h), C.byref(k))
        return {"variant": v.value, "strip_h": h.value, "iter_block": k.value}

    def step(self, Ts, rhos, cps, kappas, dts, raise_on_error=True, **kwargs):
        n = self.n
        o = step_opts(**kwargs)
        o.mem = _mem(Ts[0])
        Tp = (C.c_void_p * n)(*[_ptr(t) for t in Ts])
        Rp = (C.c_void_p * n)(*[_ptr(r) for r in rhos])
        cpa = (C.c_double * n)(*[float(c) for c in cps])
        ka = (L.Kappa * n)(*[k.as_c() for k in kappas])
        dta = (C.c_double * n)(*[float(d) for d in dts])
        st = (L.Stats * n)()
        ndt = (C.c_double * n)()
        rc = self._lib.cdm_batch_step(self._h, Tp, Rp, cpa, ka, dta, C.byref(o), st, ndt)
        stats = [stats_dict(s) for s in st]
        if rc != L.CDM_OK and raise_on_error:
            raise APTError(rc, L.last_error(), {"per_problem": stats})
        return stats, list(ndt)
