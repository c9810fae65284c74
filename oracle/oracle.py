"""ctypes binding of the CPU oracle (oracle/apt_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py — never by the product path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        PP = C.POINTER(C.c_void_p)
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.c_int] * 5 + [PP, C.c_void_p, PP, PP, C.c_double, C.c_void_p,
                                                      C.c_void_p, C.c_void_p, C.c_int]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_set_source.argtypes = [C.c_void_p, C.c_void_p]
        lib.oracle_get_state.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        lib.oracle_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        lib.oracle_get_cache.argtypes = [C.c_void_p, C.c_void_p]
        lib.oracle_step.restype = C.c_int
        lib.oracle_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_applybcs.argtypes = [C.c_int] * 5 + [C.c_void_p, C.c_void_p, C.c_void_p]
        lib.oracle_set_tz.argtypes = [C.c_void_p] + [C.c_void_p] * 6 + [C.c_int, C.c_int]
        lib.oracle_exp_cw.restype = C.c_double
        lib.oracle_exp_cw.argtypes = [C.c_double]
        lib.oracle_sinpi.restype = C.c_double
        lib.oracle_sinpi.argtypes = [C.c_double]
        lib.oracle_num_threads.restype = C.c_int
        lib.oracle_set_num_threads.argtypes = [C.c_int]
        _lib = lib
    return _lib


def _np(t):
    if t is None:
        return None
    a = t.detach().cpu().numpy() if hasattr(t, "detach") else np.asarray(t)
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleSolver:
    """CPU restatement of PseudoTransientSolver + step! on one mesh."""

    def __init__(self, mesh, bcs, mean="harmonic"):
        lib = load()
        self._lib = lib
        self.mesh = mesh
        self._keep = []

        def arr(t):
            a = _np(t)
            if a is None:
                return None
            self._keep.append(a)
            return a.ctypes.data

        inv = (C.c_void_p * 9)(*[arr(t) for t in mesh.cell_inv])
        eJ = (C.c_void_p * 3)(*[arr(t) for t in mesh.edge_J])
        eh = (C.c_void_p * 27)(*[arr(mesh.edge_hat[f][k]) for f in range(3) for k in range(9)])
        cj = arr(mesh.cell_J)
        sp = np.array(list(mesh.spacing)[:3] + [0.0] * (3 - len(mesh.spacing)), dtype=np.float64)
        bl = list(bcs.values()) if isinstance(bcs, dict) else list(bcs)
        kinds = np.array([b.kind for b in bl], dtype=np.int32)
        vals = np.array([float(getattr(b, "value", 0.0)) for b in bl], dtype=np.float64)
        self._h = lib.oracle_create(mesh.ndim, mesh.ni, mesh.nj, mesh.nk, mesh.nhalo,
                                    C.cast(inv, C.POINTER(C.c_void_p)), cj,
                                    C.cast(eJ, C.POINTER(C.c_void_p)), C.cast(eh, C.POINTER(C.c_void_p)),
                                    float(mesh.L), sp.ctypes.data, kinds.ctypes.data, vals.ctypes.data,
                                    0 if mean == "harmonic" else 1)
        self._keep = []  # the oracle copied the arrays

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.oracle_destroy(self._h)
            self._h = None

    def set_source(self, S):
        S = _np(S)
        self._lib.oracle_set_source(self._h, S.ctypes.data)

    def set_twilight_zone(self, x, y, x_xi, x_eta, y_xi, y_eta, nnodes):
        """Inputs of define_forcing_wavy: centroids, forward metrics, mesh.nnodes."""
        arrs = [_np(a) for a in (x, y, x_xi, x_eta, y_xi, y_eta)]
        self._lib.oracle_set_tz(self._h, *[a.ctypes.data for a in arrs], int(nnodes[0]), int(nnodes[1]))

    def get_state(self):
        q = np.zeros((self.mesh.ndim,) + tuple(self.mesh.full_shape))
        last = C.c_int(0)
        self._lib.oracle_get_state(self._h, q.ctypes.data, C.byref(last))
        return q, last.value

    def set_state(self, q, last):
        q = np.ascontiguousarray(q, dtype=np.float64)
        self._lib.oracle_set_state(self._h, q.ctypes.data, int(last))

    def metric_cache(self):
        out = np.zeros((self.mesh.ndim,) + tuple(self.mesh.full_shape))
        self._lib.oracle_get_cache(self._h, out.ctypes.data)
        return out

    def step(self, T: np.ndarray, rho: np.ndarray, cp: float, k0: float, n: float, dt: float, *, t=0.0,
             rtol=1e-5, atol=np.sqrt(np.finfo(np.float64).eps), CFL=1 / np.sqrt(3.0), tol=1e-3,
             maximum_u_change=0.05, timestep_growth_factor=1.1, max_iter=1500, apply_cutoff=False,
             calculate_next_dt=True, subcycle_conductivity=True, enforce_positivity=False, norm="max",
             check_every=0, tz=False, no_t=True, **_):
        """In-place step on T (float64 numpy array); returns (stats, next_dt)."""
        assert T.dtype == np.float64 and T.flags["C_CONTIGUOUS"]
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        od = np.array([t, rtol, atol, CFL, tol, maximum_u_change, timestep_growth_factor], dtype=np.float64)
        oi = np.array([max_iter, int(apply_cutoff), int(calculate_next_dt), int(subcycle_conductivity),
                       int(enforce_positivity), 0 if norm == "max" else 1, check_every, int(tz), int(no_t)],
                      dtype=np.int32)
        outd = np.zeros(6)
        outi = np.zeros(3, dtype=np.int32)
        rc = self._lib.oracle_step(self._h, T.ctypes.data, rho.ctypes.data, float(cp), float(k0), float(n),
                                   float(dt), od.ctypes.data, oi.ctypes.data, outd.ctypes.data,
                                   outi.ctypes.data)
        stats = {"rel_err": outd[0], "abs_err": outd[1], "niter": int(outi[0]), "status": int(outi[1]),
                 "n_checks": int(outi[2]), "energy_before": outd[3], "energy_after": outd[4],
                 "source_work": outd[5]}
        return stats, outd[2]


def applybcs(ndim, ni, nj, nk, nhalo, bcs, u: np.ndarray):
    lib = load()
    bl = list(bcs.values()) if isinstance(bcs, dict) else list(bcs)
    kinds = np.array([b.kind for b in bl], dtype=np.int32)
    vals = np.array([float(getattr(b, "value", 0.0)) for b in bl], dtype=np.float64)
    lib.oracle_applybcs(ndim, ni, nj, nk, nhalo, kinds.ctypes.data, vals.ctypes.data, u.ctypes.data)


def exp_cw(x: float) -> float:
    """The oracle's exp of the twilight-zone forcing (Cody–Waite + Taylor)."""
    return load().oracle_exp_cw(float(x))


def sinpi(x: float) -> float:
    """The oracle's sinpi of the twilight-zone forcing."""
    return load().oracle_sinpi(float(x))


def set_threads(n: int):
    load().oracle_set_num_threads(int(n))


def num_threads() -> int:
    return load().oracle_num_threads()
