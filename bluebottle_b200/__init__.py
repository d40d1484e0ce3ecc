"""bluebottle_b200 -- B200-native per-time-step hot path of the bluebottle
particle-resolved flow solver.

The product is libbbb200.so: C host code plus hand-written sm_100a CUDA
kernels behind the reference's `cuda_*` C entry points
(include/bluebottle_b200.h).  This Python package is a thin host-side
driver over that ABI (ctypes); it performs no computation itself.
"""
from . import abi, configs  # noqa: F401
from .sim import Sim, BBBError, interior  # noqa: F401


def load():
    """Load libbbb200.so (raises if it is not built)."""
    return abi.load()
