"""mfgpu: the MiniFS iteration hot path on NVIDIA B200 (sm_100a).

Roe flux + residual gather, local time step, level-scheduled LU-SGS sweeps
with the state update, node-based Green-Gauss gradients and the residual
norm, as hand-written CUDA behind the C ABI of ``include/mfgpu.h``.
"""
from . import meshgen  # noqa: F401

__all__ = ["meshgen", "grid", "solver"]


def __getattr__(name):
    if name in ("grid", "solver", "_lib"):
        import importlib
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
