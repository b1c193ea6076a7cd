"""rsr_b200: a B200 (sm_100a) fitness-evaluation engine for rsr's stack-VM
programs -- MSE fitness and d(MSE)/d(constants) for whole populations, behind
the C ABI in include/rsr_gpu.h."""
from . import isa
from .dataset import Dataset
from .isa import Program, Scalar, pack

__all__ = ["isa", "Dataset", "Program", "Scalar", "pack", "Engine", "Server", "compute_mse",
           "compute_mse_with_gradient"]


def __getattr__(name):
    # the evaluator needs the CUDA library; import it on first use
    import importlib
    if name in ("Engine", "compute_mse", "compute_mse_with_gradient"):
        return getattr(importlib.import_module(".evaluator", __name__), name)
    if name == "Server":
        return importlib.import_module(".serving", __name__).Server
    raise AttributeError(name)
