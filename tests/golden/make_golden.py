"""Generates the golden fixtures of the CPU oracle (tests/golden/*.npz).

The reference (pure Julia) cannot run here and publishes no output vectors
for the APT path, so these fixtures pin the oracle's own outputs on small
seeded cases: any later change of the restatement that alters a result is
caught by tests/test_oracle_cpu.py.  Run:  python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from helpers import small_case_2d, small_case_3d  # noqa: E402
from oracle.implicit_oracle import ImplicitOracle  # noqa: E402
from oracle.oracle import OracleSolver  # noqa: E402
from curvilineardiffusionmanuscript_b200.solver import DirichletBC, PeriodicBC, NeumannBC, FixedNegSymmetryBC  # noqa: E402

CASES = {
    "neumann2d": dict(dim=2, kw={}, step={}),
    "mixed_bc2d": dict(dim=2, kw=dict(bcs=[DirichletBC(1.5), NeumannBC(), PeriodicBC(), PeriodicBC()], source=True),
                       step=dict(apply_cutoff=True)),
    "negsym_arith2d": dict(dim=2, kw=dict(bcs=[FixedNegSymmetryBC(), NeumannBC(), NeumannBC(), DirichletBC(2.0)],
                                          kn=2.5), step=dict(subcycle_conductivity=False), mean="arithmetic"),
    "neumann3d": dict(dim=3, kw={}, step={}),
}


def run_case(name, spec, nsteps=3):
    pr = small_case_2d(**spec["kw"]) if spec["dim"] == 2 else small_case_3d(**spec["kw"])
    o = OracleSolver(pr.mesh, pr.bcs, mean=spec.get("mean", "harmonic"))
    if pr.source is not None:
        o.set_source(pr.source.numpy())
    T = pr.T0.numpy().copy()
    rho = pr.rho.numpy()
    out = {"niter": [], "rel": [], "abs": [], "next_dt": []}
    for _ in range(nsteps):
        st, ndt = o.step(T, rho, pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt, rtol=0.0, atol=1e-8, max_iter=20000,
                         **spec["step"])
        assert st["status"] == 0, st
        out["niter"].append(st["niter"])
        out["rel"].append(st["rel_err"])
        out["abs"].append(st["abs_err"])
        out["next_dt"].append(ndt)
    q, last = o.get_state()
    return dict(T=T, q=q, last=last, cache=o.metric_cache(), **{k: np.array(v) for k, v in out.items()})


# the implicit scheme's oracle: two steps of a 2D and a 3D case (stencil entries,
# right-hand side and solution of every step)
IMPLICIT_CASES = {
    "implicit2d": dict(dim=2, kw=dict(ni=14, nj=11, bcs=[DirichletBC(1.5), NeumannBC(), PeriodicBC(), PeriodicBC()],
                                      source=True)),
    "implicit3d": dict(dim=3, kw=dict(n=(7, 6, 5))),
}


def run_implicit(name, spec, nsteps=2):
    pr = small_case_2d(**spec["kw"]) if spec["dim"] == 2 else small_case_3d(**spec["kw"])
    o = ImplicitOracle(pr.mesh, pr.bcs)
    if pr.source is not None:
        o.set_source(pr.source.numpy())
    T = pr.T0.numpy().copy()
    out = {"c": [], "b": [], "T": [], "next_dt": []}
    for _ in range(nsteps):
        _, ndt, A, b, c = o.step(T, pr.rho.numpy(), pr.cp, pr.kappa.k0, pr.kappa.n, pr.dt)
        out["c"].append(c)
        out["b"].append(b)
        out["T"].append(T.copy())
        out["next_dt"].append(ndt)
    return {k: np.array(v) for k, v in out.items()}


if __name__ == "__main__":
    here = Path(__file__).resolve().parent
    for name, spec in CASES.items():
        res = run_case(name, spec)
        np.savez_compressed(here / f"{name}.npz", **res)
        print(name, res["niter"], res["T"].shape)
    for name, spec in IMPLICIT_CASES.items():
        res = run_implicit(name, spec)
        np.savez_compressed(here / f"{name}.npz", **res)
        print(name, res["c"].shape, res["next_dt"])
