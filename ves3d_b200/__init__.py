"""ves3d_b200: B200-native StokesVelocity evaluation for Ves3D vesicle suspensions.

The product is the CUDA library ves3d_b200/libves3d_b200.so (C ABI in
include/ves3d_b200.h); this package is its Python host mirror.
"""
from ._lib import Ves3dError, kernel_launches  # noqa: F401
from .stokes_velocity import StokesVelocity  # noqa: F401
