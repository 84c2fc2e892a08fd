"""B200-native Lyapunov-spectrum sweep (reference: mkaynov/chaos_oneapi).

The compute path is libchaos_lyap.so (hand-written sm_100a CUDA behind the C
ABI of include/chaos_lyap.h); this package only binds it.  The public names
load the library on first use (so that ``python -m chaos_oneapi_b200.build``
can run before it exists); a missing library raises ImportError then.
"""
import importlib

_EXPORTS = {
    "Sweep": "sweep", "SweepConfig": "sweep", "cuda_lyapunov": "sweep", "make_grid": "sweep",
    "make_inits": "sweep", "model_info": "sweep", "model_names": "sweep",
    "fma_peak_tflops": "sweep", "run_batch": "sweep", "BatchGraph": "sweep",
    "ChaosError": "native", "LIB_PATH": "native",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    mod = _EXPORTS.get(name)
    if mod is None:
        raise AttributeError(name)
    return getattr(importlib.import_module(f"{__name__}.{mod}"), name)
