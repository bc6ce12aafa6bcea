"""B200 implementation of MillDynamics3's per-sub-step hot path (PBF slurry + XPBD ball discs +
two-way coupling) behind the reference's Params / step API.

    from milldynamics3_b200 import open_device
    sim = open_device().simulation(params)   # Simulation mirror over the CUDA library
"""
from . import capi
from .sim import Backend, MillError, Simulation


def open_device():
    """Backend over the in-tree CUDA library (builds it on first use; raises if unavailable)."""
    from . import native
    return Backend(native.load())


__all__ = ["capi", "Backend", "MillError", "Simulation", "open_device"]
