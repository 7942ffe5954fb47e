"""rumd_b200: a B200-native (sm_100a) implementation of RUMD's LJ/NVT time step.

Layers (bottom up):
  librumd_b200.so  hand-written CUDA kernels + engine + C ABI (include/rumd_b200.h)
  capi             ctypes binding of the C ABI (Engine)
  _rumd            pybind11 module of the C++ RUMD classes (Sample, Pot_LJ_12_6,
                   IntegratorNVT, ...), which call the C ABI
  rumd             Python surface of the reference (Simulation.Run, ...)
"""
from . import initconf  # noqa: F401

__version__ = "0.1.0"
