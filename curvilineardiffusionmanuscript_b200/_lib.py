"""ctypes binding of ``libcdm_apt.so`` (the C ABI declared in include/cdm_apt.h).

This is the same binding a Julia ``ccall`` shim makes: plain pointers, sizes
and POD structs.  The library is loaded from the package directory; if it is
missing the import fails loudly — there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libcdm_apt.so"

CDM_OK, CDM_MAX_ITER, CDM_NONFINITE, CDM_BAD_INPUT, CDM_CUDA_ERROR, CDM_TIMEOUT, CDM_NO_DEVICE = range(7)
STATUS_NAMES = {0: "OK", 1: "MAX_ITER", 2: "NONFINITE", 3: "BAD_INPUT", 4: "CUDA_ERROR", 5: "TIMEOUT",
                6: "NO_DEVICE"}
CDM_MEM_HOST, CDM_MEM_DEVICE = 0, 1
CDM_BC_NEUMANN, CDM_BC_DIRICHLET, CDM_BC_PERIODIC, CDM_BC_NEG_SYMMETRY = range(4)
CDM_MEAN_HARMONIC, CDM_MEAN_ARITHMETIC = 0, 1
CDM_NORM_MAX, CDM_NORM_RMS = 0, 1
CDM_PREC_FP64, CDM_PREC_MIXED, CDM_PREC_FP64_EXACT = 0, 1, 2
CDM_GUESS_PREV, CDM_GUESS_USER, CDM_GUESS_LEARNED, CDM_GUESS_EXTRAPOLATE = 0, 1, 2, 3

PD = C.POINTER(C.c_double)


class Kappa(C.Structure):
    _fields_ = [("k0", C.c_double), ("n", C.c_double)]


class BC(C.Structure):
    _fields_ = [("kind", C.c_int), ("value", C.c_double)]


class MeshDesc(C.Structure):
    _fields_ = [
        ("ndim", C.c_int), ("ni", C.c_int), ("nj", C.c_int), ("nk", C.c_int), ("nhalo", C.c_int),
        ("mem", C.c_int),
        ("cell_inv", C.c_void_p * 9),
        ("cell_J", C.c_void_p),
        ("edge_J", C.c_void_p * 3),
        ("edge_hat", (C.c_void_p * 9) * 3),
        ("L", C.c_double),
        ("spacing", C.c_double * 3),
        ("node_x", C.c_void_p * 3),
    ]


class TzDesc(C.Structure):
    """cdm_tz_desc (include/cdm_apt.h)."""
    _fields_ = [("mem", C.c_int), ("nnodes", C.c_int * 2), ("x", C.c_void_p), ("y", C.c_void_p),
                ("x_xi", C.c_void_p), ("x_eta", C.c_void_p), ("y_xi", C.c_void_p), ("y_eta", C.c_void_p)]


class Config(C.Structure):
    _fields_ = [("mean", C.c_int), ("precision", C.c_int), ("device", C.c_int), ("stream", C.c_void_p)]


class StepOpts(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("tz", C.c_int), ("tz_dim", C.c_int), ("no_t", C.c_int),
        ("max_iter", C.c_int), ("rtol", C.c_double), ("atol", C.c_double),
        ("error_check_interval", C.c_int), ("apply_cutoff", C.c_int), ("calculate_next_dt", C.c_int),
        ("subcycle_conductivity", C.c_int), ("enforce_positivity", C.c_int), ("CFL", C.c_double),
        ("ndt_tol", C.c_double), ("maximum_u_change", C.c_double), ("timestep_growth_factor", C.c_double),
        ("norm", C.c_int), ("check_every", C.c_int), ("guess", C.c_int), ("mem", C.c_int),
        ("iter_block", C.c_int), ("use_graph", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("rel_err", C.c_double), ("abs_err", C.c_double), ("niter", C.c_int), ("status", C.c_int),
        ("time", C.c_double), ("energy_before", C.c_double), ("energy_after", C.c_double),
        ("source_work", C.c_double), ("n_restarts", C.c_int), ("n_checks", C.c_int),
    ]


class Profile(C.Structure):
    _fields_ = [("sweep_ms", C.c_double), ("sweep_launches", C.c_int64), ("other_launches", C.c_int64),
                ("cell_iters", C.c_int64), ("fp32_cell_iters", C.c_int64), ("fp64_cell_evals", C.c_int64)]


class ImplicitOpts(C.Structure):
    """cdm_implicit_opts (include/cdm_apt.h)."""
    _fields_ = [("atol", C.c_double), ("rtol", C.c_double), ("max_iter", C.c_int), ("enforce_positivity", C.c_int),
                ("apply_density_bc", C.c_int), ("ndt_tol", C.c_double), ("maximum_u_change", C.c_double),
                ("timestep_growth_factor", C.c_double), ("mem", C.c_int)]


class NetBatch(C.Structure):
    """cdm_net_batch (include/cdm_net.h)."""
    _fields_ = [
        ("nsamp", C.c_int), ("tprev", C.POINTER(C.c_void_p)), ("tcur", C.POINTER(C.c_void_p)),
        ("tnext", C.POINTER(C.c_void_p)), ("J", C.c_void_p), ("ox", C.POINTER(C.c_int)), ("oy", C.POINTER(C.c_int)),
        ("crop", C.c_int), ("ni", C.c_int), ("nj", C.c_int), ("nhalo", C.c_int), ("k0", C.c_double),
        ("kn", C.c_double), ("log_jmean", C.c_double), ("dt", C.c_double), ("rho_cp", C.c_double),
    ]


PF = C.POINTER(C.c_float)

# every symbol declared in include/cdm_apt.h and include/cdm_net.h: name -> (restype, argtypes)
SIGNATURES = {
    "cdm_apt_version": (C.c_int, []),
    "cdm_selftest_bounded_wait": (C.c_int, [C.c_int, C.c_double, C.POINTER(C.c_int)]),
    "cdm_selftest_fastmath": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]),
    "cdm_apt_last_error": (C.c_char_p, []),
    "cdm_step_opts_default": (None, [C.POINTER(StepOpts)]),
    "cdm_apt_config_default": (None, [C.POINTER(Config)]),
    "cdm_apt_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(BC), C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "cdm_apt_destroy": (C.c_int, [C.c_void_p]),
    "cdm_apt_set_source": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "cdm_apt_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, Kappa, C.c_double,
                               C.POINTER(StepOpts), C.POINTER(Stats), PD]),
    "cdm_apt_set_guess": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "cdm_apt_set_twilight_zone": (C.c_int, [C.c_void_p, C.POINTER(TzDesc)]),
    "cdm_batch_set_twilight_zone": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(TzDesc)]),
    "cdm_apt_advance": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, Kappa, PD, C.c_double, C.c_int,
                                  PD, C.c_double, C.POINTER(StepOpts), C.POINTER(Stats), C.POINTER(C.c_int)]),
    "cdm_apt_get_state": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "cdm_apt_set_state": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "cdm_apt_get_metric_cache": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cdm_apt_full_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "cdm_batch_create": (C.c_int, [C.c_int, C.POINTER(MeshDesc), C.POINTER(BC), C.POINTER(Config),
                                   C.POINTER(C.c_void_p)]),
    "cdm_batch_destroy": (C.c_int, [C.c_void_p]),
    "cdm_batch_set_source": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "cdm_batch_step": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), PD,
                                 C.POINTER(Kappa), PD, C.POINTER(StepOpts), C.POINTER(Stats), PD]),
    "cdm_batch_autotune": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), PD,
                                     C.POINTER(Kappa), PD, C.POINTER(StepOpts), C.c_char_p, C.POINTER(C.c_int)]),
    "cdm_batch_tuning": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "cdm_batch_set_tuning": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    "cdm_apt_get_profile": (C.c_int, [C.c_void_p, C.POINTER(Profile)]),
    "cdm_batch_get_profile": (C.c_int, [C.c_void_p, C.POINTER(Profile)]),
    "cdm_step_reductions_noalloc": (C.c_int, [C.c_int] * 5 + [C.c_void_p] * 5 + [C.c_double] * 5 + [PD, C.c_void_p]),
    "cdm_implicit_opts_default": (None, [C.POINTER(ImplicitOpts)]),
    "cdm_implicit_create": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(BC), C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "cdm_implicit_destroy": (C.c_int, [C.c_void_p]),
    "cdm_implicit_set_source": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "cdm_implicit_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, Kappa, C.c_double,
                                    C.POINTER(ImplicitOpts), C.POINTER(Stats), PD]),
    "cdm_implicit_get_system": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "cdm_implicit_get_profile": (C.c_int, [C.c_void_p, PD, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "cdm_net_create": (C.c_int, [C.c_int, C.c_uint64, C.c_void_p, C.POINTER(C.c_void_p)]),
    "cdm_net_destroy": (C.c_int, [C.c_void_p]),
    "cdm_net_num_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cdm_net_set_guess_smoothing": (C.c_int, [C.c_void_p, C.c_int]),
    "cdm_net_get_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cdm_net_set_params": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cdm_net_get_grads": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cdm_net_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "cdm_net_backward": (C.c_int, [C.c_void_p, C.c_void_p, PF]),
    "cdm_net_train_step": (C.c_int, [C.c_void_p, C.POINTER(NetBatch), C.c_float, PF]),
    "cdm_net_predict": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                  C.c_double, C.c_double, C.c_double, C.c_void_p]),
    "cdm_apt_set_guess_net": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
}

_lib = None


def load() -> C.CDLL:
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with "
                               "`python -m curvilineardiffusionmanuscript_b200.build` (no CPU fallback exists)")
        lib = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def last_error() -> str:
    return load().cdm_apt_last_error().decode(errors="replace")


def default_opts() -> StepOpts:
    o = StepOpts()
    load().cdm_step_opts_default(C.byref(o))
    return o


def default_config() -> Config:
    c = Config()
    load().cdm_apt_config_default(C.byref(c))
    return c
