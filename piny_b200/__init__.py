"""pinyb200: B200-native force path for PINY_MD flexible point-charge water.

  water    -- models, seeded synthetic boxes, PINY input directories
  system   -- host-side set-up tables (PINY's input-stage products)
  lib      -- ctypes binding of the C ABI in include/pinyb200.h
  build    -- nvcc build of the in-tree sm_100a library
"""
__all__ = ["water", "system", "lib", "build"]
