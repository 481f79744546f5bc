"""B200-native AUSM-family O-grid Euler solver: Python host over libausm.so (C ABI)."""
from ._lib import AusmError, AusmParams
from .solver import Batch, Solver, default_params, device_count, set_device

__all__ = ["AusmError", "AusmParams", "Batch", "Solver", "default_params", "device_count", "set_device"]
