"""xdem_b200 — B200 (sm_100a) implementation of xDEM's per-timestep DEM path.

The compute path is libxdem_b200.so (CUDA kernels + the C-ABI of
include/xdem_gpu.h).  This package holds its ctypes binding (`abi`), the
reference-named world wrapper (`world`), synthetic input generators
(`inputs`) and the build recipe (`build`).  There is no CPU fallback: using a
world without the built library raises ImportError.
"""
from . import abi  # noqa: F401
from .abi import XdemError  # noqa: F401

__all__ = ["abi", "XdemError", "World", "make_params", "make_control"]


def __getattr__(name):
    if name in ("World", "make_params", "make_control", "pair_geometry", "WorldBase"):
        from . import world
        return getattr(world, name)
    raise AttributeError(name)
