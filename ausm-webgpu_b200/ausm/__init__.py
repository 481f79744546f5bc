"""B200-native AUSM-family O-grid Euler solver: Python host over libausm.so (C ABI)."""
from ._lib import AusmError, AusmParams
from .shard import ShardedServer, place_requests
from .solver import Batch, Server, Solver, default_params, device_count, make_request, request_bytes, set_device, set_wait_polls

__all__ = ["AusmError", "AusmParams", "Batch", "Server", "Solver", "make_request", "request_bytes", "default_params", "device_count", "set_device", "set_wait_polls", "ShardedServer", "place_requests"]
