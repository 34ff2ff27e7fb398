"""B200 (sm_100a) backend of 3dimagetoolkit's RSFE Split-Bregman segmentation path.

The package name starts with a digit, so import it with
``importlib.import_module("3dimagetoolkit_b200")``.

* ``_abi``   -- ctypes binding of the C ABI (include/im3d_b200.h, libim3d_b200.so)
* ``mhd``    -- headless MetaImage (.mhd/.raw) reader and writer
* ``synth``  -- seeded synthetic volumes of the benchmark workloads
* ``shard``  -- volumes of a batch across ranks

The C++ mirror of the reference's classes (image3d, filtering,
unsteady_poisson_functor, rsfe_splitbregman) is header-only, in include/im3d/.
"""
from ._abi import (BATCH_AUTO, BATCH_STREAMS, BATCH_WORKLIST, BC_DEFAULT, BC_DIR, BC_NEU,
                   OPT_BATCH_MODE, OPT_DEVICE_MEMORY_LIMIT, OPT_FIT_CHUNKS, OPT_TILE_LOADS,
                   SWEEP_LEXICOGRAPHIC,
                   SWEEP_REDBLACK, WS_OFF, WS_PREDICT, WS_TRAIN, Context, Im3dError, RsfeParams,
                   RsfeStats, UNet, default_params, lib)
from . import mhd, synth

__all__ = ["Context", "Im3dError", "RsfeParams", "RsfeStats", "default_params", "lib", "mhd", "synth",
           "BC_DEFAULT", "BC_DIR", "BC_NEU", "SWEEP_LEXICOGRAPHIC", "SWEEP_REDBLACK",
           "OPT_FIT_CHUNKS", "OPT_DEVICE_MEMORY_LIMIT", "OPT_BATCH_MODE", "OPT_TILE_LOADS", "BATCH_AUTO",
           "BATCH_STREAMS", "BATCH_WORKLIST", "UNet", "WS_OFF", "WS_PREDICT", "WS_TRAIN"]
