"""sphgpu — B200-native SPH step engine behind the reference's SPHSystem seam.

Host-side mirror (Python) of the C ABI in include/sphgpu.h. All physics runs
in hand-written sm_100a CUDA kernels inside libsphgpu.so; this package only
marshals inputs and results.
"""
from . import _capi as capi
from ._capi import SPHError
from .server import SceneServer
from .system import GpuSystem, RigidInit, find_samples, kernel_function, kernel_gradient, make_config

__all__ = ["capi", "SPHError", "GpuSystem", "RigidInit", "SceneServer", "find_samples", "kernel_function",
           "kernel_gradient", "make_config"]
