"""B200-native implementation of MCV_SW's explicit RK step.

The product is the CUDA library ``_lib/libmcv_gpu.so`` behind the C ABI of
``include/mcv_gpu.h``; this package binds it with ctypes (``api``), builds it
(``build``), and restates the reference's host-side driver pieces that feed it
(``cases`` for seeded initial states).  There is no CPU fallback.
"""
from .api import (FP64, MIXED, RK3_TVD, RK4, Geometry, MCVError, Stepper, add_harmonics, add_mountain,
                  add_rossby_haurwitz, footprint_bytes, grid_sizes, lib, lib_path, sphere_to_cov, tilted_zonal,
                  williamson)

__all__ = ["FP64", "MIXED", "RK3_TVD", "RK4", "Geometry", "MCVError", "Stepper", "add_harmonics", "add_mountain",
           "add_rossby_haurwitz", "footprint_bytes", "grid_sizes", "lib", "lib_path", "sphere_to_cov",
           "tilted_zonal", "williamson"]
