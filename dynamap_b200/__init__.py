"""dynamap_b200: B200-native rigid RGB-D mapping (DynaMap's per-frame path).

The compute lives in libdynamap_b200.so (CUDA, sm_100a) behind the C ABI of
include/dynamap.h; this package holds its ctypes binding (abi), the session
wrapper (session), workload presets (configs) and the synthetic scene
generator (scene).
"""
from . import abi, configs, scene  # noqa: F401

__all__ = ["abi", "configs", "scene"]
