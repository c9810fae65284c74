"""C-ABI checks that need no GPU: the library loads and exports every symbol
that include/*.h declares; host-side logic that needs no device."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(cdm_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from curvilineardiffusionmanuscript_b200 import _lib
    lib = _lib.load()
    names = declared_symbols()
    assert "cdm_apt_step" in names and "cdm_batch_step" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares a signature for every exported entry point
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_abi_defaults_match_reference_kwargs():
    """step! defaults (PseudoTransientSolver.jl:188-202) and next_dt defaults (timestep_control.jl:33-42)."""
    from curvilineardiffusionmanuscript_b200 import _lib
    o = _lib.default_opts()
    assert o.max_iter == 1500 and o.rtol == 1e-5 and abs(o.atol - 2.220446049250313e-16 ** 0.5) < 1e-30
    assert o.subcycle_conductivity == 1 and o.calculate_next_dt == 1 and o.apply_cutoff == 0
    assert abs(o.CFL - 1 / 3 ** 0.5) < 1e-16 and o.ndt_tol == 1e-3 and o.maximum_u_change == 0.05
    assert o.timestep_growth_factor == 1.1 and o.error_check_interval == 2
    c = _lib.default_config()
    assert c.mean == _lib.CDM_MEAN_HARMONIC and c.precision == _lib.CDM_PREC_FP64
    assert _lib.load().cdm_apt_version() == 1


def test_struct_layout_matches_header():
    """sizeof of the ctypes mirrors equals the C compiler's view of the header."""
    import subprocess, tempfile, os
    src = r'''
#include <stdio.h>
#include "cdm_apt.h"
#include "cdm_net.h"
int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(cdm_mesh_desc), sizeof(cdm_step_opts),
 sizeof(cdm_stats), sizeof(cdm_apt_config), sizeof(cdm_bc), sizeof(cdm_kappa), sizeof(cdm_net_batch),
 sizeof(cdm_tz_desc));return 0;}
'''
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.c")
        open(p, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["/usr/bin/gcc", "-I", str(ROOT / "include"), p, "-o", exe], check=True)
        sizes = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    from curvilineardiffusionmanuscript_b200 import _lib
    assert sizes == [C.sizeof(_lib.MeshDesc), C.sizeof(_lib.StepOpts), C.sizeof(_lib.Stats),
                     C.sizeof(_lib.Config), C.sizeof(_lib.BC), C.sizeof(_lib.Kappa), C.sizeof(_lib.NetBatch),
                     C.sizeof(_lib.TzDesc)]


def test_create_without_device_reports_error():
    """On a host without a B200 the library reports NO_DEVICE instead of falling back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from curvilineardiffusionmanuscript_b200 import APTError, NeumannBC, PseudoTransientSolver, wavy_mesh_2d
    with pytest.raises(APTError) as ei:
        PseudoTransientSolver(wavy_mesh_2d(8, 8), [NeumannBC()] * 4)
    assert ei.value.status in (4, 6)
    from curvilineardiffusionmanuscript_b200.learned import GuessNet
    with pytest.raises(APTError) as ei:
        GuessNet(seed=0)
    assert ei.value.status in (4, 6)
