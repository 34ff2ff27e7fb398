"""B200 (sm_100a) backend of 3dimagetoolkit's RSFE Split-Bregman segmentation path.

The package name starts with a digit, so import it with
``importlib.import_module("3dimagetoolkit_b200")``.

* ``_abi``   -- ctypes binding of the C ABI (include/im3d_b200.h, libim3d_b200.so)
* ``segm``, ``conv``, ``lapl``, ``im3d`` -- host-side mirror of the reference's classes
  (rsfe_splitbregman, filtering, unsteady_poisson_functor, image3d) over that ABI
* ``synth``  -- seeded synthetic volumes of the benchmark workloads
"""
from ._abi import (BC_DEFAULT, BC_DIR, BC_NEU, SWEEP_LEXICOGRAPHIC, SWEEP_REDBLACK, Context,
                   Im3dError, RsfeParams, RsfeStats, default_params, lib)
from . import mhd, synth

__all__ = ["Context", "Im3dError", "RsfeParams", "RsfeStats", "default_params", "lib", "mhd", "synth",
           "BC_DEFAULT", "BC_DIR", "BC_NEU", "SWEEP_LEXICOGRAPHIC", "SWEEP_REDBLACK"]
