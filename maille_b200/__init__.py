"""maille_b200 -- B200 (sm_100a) implementation of maille-core's linear-elastic solve path:
Tet4/Tet10 element stiffness, deterministic sparse assembly and IC(0)-preconditioned conjugate
gradients, with Gauss-point stresses; and the transient heat conduction step (theta-method) on
the same machinery. The compute runs in libmaille_gpu.so (CUDA, C ABI in include/maille_gpu.h);
this package is the host-side mirror of the reference's solve interface.
"""
from .model import (Bc, Dof, Field, ITERATIVE_FROM, Load, MailleError, Material, Mesh, Model,  # noqa: F401
                    Pressure, SolverHandle, SolverKind, face_pressure_loads)
from ._lib import (MAILLE_FP64, MAILLE_MIXED, MAILLE_ORDER_AUTO, MAILLE_ORDER_MULTICOLOR,  # noqa: F401
                   MAILLE_ORDER_MULTICOLOR_BFS, MAILLE_ORDER_RCM,
                   MAILLE_ORDER_MULTICOLOR_ITERATED)

__version__ = "0.1.0"
from .batch import BatchField, BatchSolver, partition_lpt, solve_sharded  # noqa: F401,E402
from .large_strain import LargeStrainHistory, LargeStrainSolver  # noqa: F401,E402
from .thermal import Convection, HeatSource, Increment, Step, ThermalModel, thermal_loads  # noqa: F401,E402
