"""aperi_mech_b200: B200-native (sm_100a) explicit-dynamics hot path of aperi-mech.

The compute lives in libaperi_b200.so (C ABI: include/aperi_b200.h). This package
holds its ctypes binding (capi), a Python front-end shaped like the reference's
solver objects (model), and the synthetic workload generators (mesh, problems).
"""
from .model import BoundaryCondition, ExplicitDynamics, Material, Part, complete_properties  # noqa: F401

__all__ = ["BoundaryCondition", "ExplicitDynamics", "Material", "Part", "complete_properties"]
