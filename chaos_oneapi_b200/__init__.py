"""B200-native Lyapunov-spectrum sweep (reference: mkaynov/chaos_oneapi).

The compute path is libchaos_lyap.so (hand-written sm_100a CUDA behind the C
ABI of include/chaos_lyap.h); this package only binds it.
"""
from .sweep import (Sweep, SweepConfig, cuda_lyapunov, make_grid, make_inits, model_info,
                    model_names)
from .native import ChaosError, LIB_PATH

__all__ = ["Sweep", "SweepConfig", "cuda_lyapunov", "make_grid", "make_inits", "model_info",
           "model_names", "ChaosError", "LIB_PATH"]
