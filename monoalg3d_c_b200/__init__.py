"""B200-native operator-split monodomain step (MonoAlg3D's hot path).

Kernels: hand-written sm_100a CUDA in ``csrc/``; host driver in C; the Python
layer here is a thin ctypes mirror of the reference plugin interface.
"""
from ._lib import MonoAlgError, device_count, lib  # noqa: F401
from .monodomain import (Stim, Tissue, OdeSolver, csr_conjugate_gradient, init_cell_model_data,  # noqa: F401
                         loop_steps)

__all__ = ["MonoAlgError", "Stim", "Tissue", "OdeSolver", "csr_conjugate_gradient", "init_cell_model_data",
           "loop_steps", "device_count"]
