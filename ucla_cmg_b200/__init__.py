"""B200-native voomEP monodomain time step (sm_100a CUDA behind a C ABI).

Modules: ``capi`` (ctypes binding of include/ep_gpu.h), ``simulation``
(the reference's EPSolver/CardiacBody interface over the C ABI), ``mesh``
(synthetic linear-tet workloads), ``build`` (nvcc build of libepgpu.so).
"""
from . import mesh  # noqa: F401

__all__ = ["mesh", "capi", "simulation", "build"]
