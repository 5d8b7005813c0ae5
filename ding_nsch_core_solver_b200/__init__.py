"""B200-native CHNS time step (Cahn-Hilliard implicit solve, momentum predictor, pressure correction) behind
the C-ABI of include/dn_cuda.h; see capi.Solver."""
from .capi import DnError, Solver, load, parse_config, step_batch  # noqa: F401

__all__ = ["Solver", "DnError", "load", "parse_config", "step_batch"]
