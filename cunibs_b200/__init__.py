"""cunibs_b200: B200-native per-placement TMS field solve, a drop-in for cuNIBS's forward path.

Public API mirrors the reference's (cunibs/__init__.py): Subject, Placement, FieldResult, Coil,
load_mesh, HeadMesh, SolverConvergenceError, the conductivity Monte Carlo types of cunibs.uq, and
the auxiliary dipole method as the ``adm`` submodule (cunibs.adm).
"""

from . import adm
from .coil import Coil
from .fem import RECOVERY_MODES, SolverConvergenceError
from .mesh import HeadMesh, load_mesh
from .simulation import FieldResult, Placement, Subject
from .uq import ConductivityUQConfig, ConductivityUQResult

__all__ = ["Coil", "ConductivityUQConfig", "ConductivityUQResult", "FieldResult", "HeadMesh", "Placement",
           "RECOVERY_MODES", "SolverConvergenceError", "Subject", "load_mesh"]
