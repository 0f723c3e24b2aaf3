"""B200-native quasi-incompressible smectic-isotropic pseudo-spectral step.

The compute path is libquasi_gpu.so (hand-written CUDA for sm_100a behind a C
ABI, include/quasi_gpu.h); this package holds its sources (csrc/), its build
(build.py) and the ctypes host mirror (quasi.py).
"""
from .quasi import (Config, Ensemble, IC, QuasiError, R2RPlan, Simulation, default_config,  # noqa: F401
                    initial_condition, lib)
