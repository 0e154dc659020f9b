"""B200-native ddCOSMO solver (drop-in for the filippolipparini/ddPCM path).

The compute path is the CUDA library ``lib/libddcosmo_gpu.so`` (C ABI in
``include/ddcosmo_gpu.h``); ``ddcosmo.DDCosmo`` mirrors the reference's
module interface on top of it.
"""
from .build import LIB, build  # noqa: F401
from .ddcosmo import DDCosmo, DDCosmoError, load_library  # noqa: F401
from . import molecules  # noqa: F401
