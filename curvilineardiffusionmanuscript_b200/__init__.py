"""B200-native accelerated pseudo-transient (APT) solver — a drop-in for the
APT path of CurvilinearDiffusion (smillerc/CurvilinearDiffusionManuscript).

The solver runs in hand-written CUDA for sm_100a behind the C ABI of
``libcdm_apt.so`` (include/cdm_apt.h); this package mirrors the reference's
Julia interface on top of it.
"""
from .mesh import CurvilinearMesh, wavy_mesh_2d, wavy_mesh_3d, uniform_mesh_2d, mesh_from_nodes_2d  # noqa: F401
from .solver import (APTError, DirichletBC, FixedNegSymmetryBC, ImplicitScheme, NeumannBC,  # noqa: F401
                     PeriodicBC, PowerLawConductivity, PseudoTransientBatch, PseudoTransientSolver,
                     nonlinear_thermal_conduction_step, step)

__version__ = "0.1.0"
