"""b200lbm -- B200-native LBM step behind the reference's Sim / RigidSphere API.

    from b200lbm import Sim, RigidSphere
"""
from .sim import Sim, TrackedArray  # noqa: F401
from .solid import CompositeSolid, RigidSphere  # noqa: F401
from .batch import Batch  # noqa: F401
from .slab import SlabSim  # noqa: F401
from .mesh import MeshSolid  # noqa: F401
from . import _capi  # noqa: F401

__all__ = ["Sim", "RigidSphere", "CompositeSolid", "TrackedArray", "Batch", "SlabSim"]
