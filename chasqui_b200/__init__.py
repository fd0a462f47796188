"""chasqui_b200 — B200-native (sm_100a) per-Runge-Kutta-stage ideal-MHD path of Chasqui.

The compute path is the CUDA library `_lib/libchq.so` (C ABI: include/chq.h); this package
is its host-side mirror: the reference's parameter semantics (`params`) and a ctypes binding
(`core`). There is no CPU implementation in the package.
"""
from .params import Params, ParamError, config_from_params  # noqa: F401
from .core import (ChqError, Mesh, chq_config, default_config, make_config, load_library,  # noqa: F401
                   LIB_PATH, SIGNATURES, FIELDS, PROFILE_KINDS, PinnedArray, set_device, device_count, Batch, Server)

__all__ = ["Params", "ParamError", "config_from_params", "ChqError", "Mesh", "chq_config", "default_config",
           "make_config", "load_library", "LIB_PATH", "SIGNATURES", "FIELDS", "PROFILE_KINDS", "PinnedArray",
           "set_device", "device_count", "Batch", "Server"]
