"""wam_b200: WAM Cycle 7's per-time-step hot path (IMPLSCH + PROPAGS) on B200.

The compute lives in libwamgpu.so (hand-written sm_100a CUDA behind the C ABI
of include/wamgpu.h); this package is the host-side mirror of the reference's
module procedures plus synthetic-input generation.  Importing it does not
require a GPU; every compute call fails loudly without one.
"""
from ._lib import WamgpuError, load  # noqa: F401
from .model import WamModel, make_config, effective_parameters  # noqa: F401
from .grid import regular_grid  # noqa: F401

__all__ = ["WamModel", "make_config", "effective_parameters", "regular_grid", "WamgpuError", "load"]
