"""Headless VTK output of the solver state (the reference's `to_vtk` /
`save_vtk`, src/pseudo_transient/PseudoTransientSolver.jl:380-412 and
src/vtk.jl:20-41).

Writes a VTK XML structured grid (`.vts`, raw appended binary, little endian)
with the mesh's node coordinates, the field value `TimeValue` and cell data
over the domain: `rho`, `u`, the damped fluxes `q1..qd` (the solver state),
`diffusivity` α = κ(u)/(ρcₚ), the pseudo-time parameters `dτ_ρ` and `θr_dτ`
(iteration_parameters.jl:2-34) and `source_term`.  File names follow the
reference: `<name>_<iteration:07d>.vts`.

Arrays may live on the GPU: they are copied to host memory on the calling
thread and the file is written by a background thread when `background=True`
(the returned future completes when the file is closed).
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import struct
from typing import Dict, Optional

import numpy as np
import torch

_pool: Optional[cf.ThreadPoolExecutor] = None


def filename(iteration: int, name: str = "diffusion") -> str:
    name = name.replace(" ", "_")
    if not name.endswith("_"):
        name = name + "_"
    return f"{name}{iteration:07d}.vts"


def _host(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def write_vts(path: str, nodes, cell_data: Dict[str, np.ndarray], time_value: float = 0.0,
              dtype=np.float32) -> str:
    """Structured grid with node coordinates `nodes` (2 or 3 arrays shaped
    (nj+1, ni+1) / (nk+1, nj+1, ni+1)) and cell arrays shaped (nj, ni) / (nk, nj, ni)."""
    xs = [_host(n).astype(np.float64) for n in nodes]
    nd = len(xs)
    shape = xs[0].shape
    ext = [shape[-1] - 1, shape[-2] - 1, shape[-3] - 1 if nd == 3 else 0]
    pts = np.zeros((int(np.prod(shape)), 3), dtype=dtype)
    for c in range(nd):
        pts[:, c] = xs[c].reshape(-1)
    blocks = [pts]
    names = []
    for k, v in cell_data.items():
        arr = np.ascontiguousarray(_host(v), dtype=dtype).reshape(-1)
        blocks.append(arr)
        names.append(k)
    vtype = "Float32" if np.dtype(dtype) == np.float32 else "Float64"
    offsets, off = [], 0
    for b in blocks:
        offsets.append(off)
        off += 8 + b.nbytes
    extent = f"0 {ext[0]} 0 {ext[1]} 0 {ext[2]}"
    head = [
        '<?xml version="1.0"?>',
        '<VTKFile type="StructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">',
        f'  <StructuredGrid WholeExtent="{extent}">',
        '    <FieldData>',
        f'      <DataArray type="Float64" Name="TimeValue" NumberOfTuples="1" format="ascii">{time_value!r}</DataArray>',
        '    </FieldData>',
        f'    <Piece Extent="{extent}">',
        '      <Points>',
        f'        <DataArray type="{vtype}" NumberOfComponents="3" format="appended" offset="{offsets[0]}"/>',
        '      </Points>',
        '      <CellData>',
    ]
    for k, o in zip(names, offsets[1:]):
        head.append(f'        <DataArray type="{vtype}" Name="{k}" format="appended" offset="{o}"/>')
    head += ['      </CellData>', '    </Piece>', '  </StructuredGrid>', '  <AppendedData encoding="raw">']
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n   _").encode())
        for b in blocks:
            f.write(struct.pack("<Q", b.nbytes))
            f.write(np.ascontiguousarray(b).astype(b.dtype.newbyteorder("<"), copy=False).tobytes())
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return path


def solver_fields(solver, mesh, u, rho, cp: float, kappa, dt: Optional[float] = None, source=None,
                  CFL: float = 1.0 / math.sqrt(3.0)) -> Dict[str, np.ndarray]:
    """The reference's output fields over the domain, on the host (FP64)."""
    dom = mesh.domain()
    U = _host(u)[dom].astype(np.float64)
    R = _host(rho)[dom].astype(np.float64)
    kap = np.where(np.isfinite(U), kappa.k0 * np.abs(U) ** kappa.n if kappa.n != 0 else kappa.k0, 0.0)
    alpha = kap / (R * cp)
    out = {"rho": R, "u": U}
    q, _ = solver.get_state()
    for i in range(mesh.ndim):
        out[f"q{i + 1}"] = q[i][dom]
    out["diffusivity"] = alpha
    if dt is not None:
        # iteration_parameters.jl:2-15 with Vpdτ = CFL·min(spacing)
        L = mesh.L
        vp = CFL * min(mesh.spacing[:mesh.ndim])
        with np.errstate(divide="ignore", invalid="ignore"):
            Re = math.pi + np.sqrt(math.pi ** 2 + (L * L * R) / (alpha * dt))
            dtau = vp * L / (alpha * Re)
            theta = L / (vp * Re)
        out["dτ_ρ"] = np.where(np.isfinite(dtau), dtau, 0.0)
        out["θr_dτ"] = np.where(np.isfinite(theta), theta, 0.0)
    if source is not None:
        out["source_term"] = _host(source)[dom]
    return out


def save_vtk(solver, u, rho, mesh, iteration: int = 0, t: float = 0.0, name: str = "diffusion",
             cp: float = 1.0, kappa=None, dt: Optional[float] = None, source=None, dtype=np.float32,
             background: bool = False):
    """to_vtk(scheme, mesh, u, ρ, iteration, t, name, T): returns the file name,
    or a future of it when `background` is set."""
    from .solver import PowerLawConductivity
    kappa = kappa or PowerLawConductivity(1.0, 0.0)
    fields = solver_fields(solver, mesh, u, rho, cp, kappa, dt, source)  # host copies, taken now
    nodes = [_host(n) for n in mesh.nodes]
    fn = filename(iteration, name)
    if not background:
        return write_vts(fn, nodes, fields, t, dtype)
    global _pool
    if _pool is None:
        _pool = cf.ThreadPoolExecutor(max_workers=1, thread_name_prefix="vtk")
    return _pool.submit(write_vts, fn, nodes, fields, t, dtype)
