"""ctypes binding of libausm.so (include/ausm.h).

The library is built in-tree by ausm-webgpu_b200/build.py.  There is no fallback: if
the shared library is missing, importing the solver raises, so a GPU run can never
silently take another path.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

PKG = Path(__file__).resolve().parents[1]
ROOT = PKG.parent
LIB_PATH = Path(os.environ.get("AUSM_LIB", PKG / "lib" / "libausm.so"))
HEADER = ROOT / "include" / "ausm.h"

OK = 0
ERR_INVALID, ERR_CUDA, ERR_OOM, ERR_DIVERGED, ERR_STATE, ERR_BUDGET, ERR_TIMEOUT, ERR_NOT_FOUND = range(-1, -9, -1)
SCHEMES = {"SLAU2": 0, "SLAU": 1, "AUSM+-up": 2}
ENGINES = {"fused": 0, "reference": 1, "f64": 2}
INIT = {"rest": 0, "freestream": 1}
OUTER = {"rect": 0, "circle": 1}
GRID = {"jacobi": 0, "multicolor": 1}
FIELDS = {"density": 0, "pressure": 1, "temperature": 2, "mach": 3, "entropy": 4, "wave_speed": 5}


class AusmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class AusmParams(C.Structure):
    _fields_ = [("gamma", C.c_double), ("in_rho", C.c_double), ("in_pressure", C.c_double),
                ("mach", C.c_double), ("aoa_deg", C.c_double), ("K_p", C.c_double), ("K_u", C.c_double),
                ("cfl", C.c_double), ("maxdt", C.c_double), ("muscl", C.c_int), ("scheme", C.c_int),
                ("ramp", C.c_double)]


class AusmRequest(C.Structure):
    _fields_ = [("M", C.c_int), ("N", C.c_int), ("naca4", C.c_int), ("closed_te", C.c_int),
                ("body_xy", C.POINTER(C.c_double)), ("chord", C.c_double), ("far_radius", C.c_double),
                ("first_spacing", C.c_double), ("grid_iters", C.c_int), ("init_mode", C.c_int),
                ("params", AusmParams), ("residual_drop", C.c_double), ("max_steps", C.c_int)]


class AusmResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("state", C.c_int), ("stop", C.c_int), ("M", C.c_int), ("N", C.c_int),
                ("steps", C.c_int), ("l2_first", C.c_double), ("l2_last", C.c_double),
                ("forces", C.c_double * 6), ("queue_ms", C.c_double), ("run_ms", C.c_double),
                ("latency_ms", C.c_double)]


class AusmServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("rejected", C.c_int64), ("admitted", C.c_int64),
                ("finished", C.c_int64), ("failed", C.c_int64), ("rounds", C.c_int64), ("pending", C.c_int),
                ("active", C.c_int), ("bytes_in_use", C.c_double), ("peak_bytes", C.c_double),
                ("cell_updates", C.c_double)]


REQ_DONE, REQ_QUEUED, REQ_RUNNING = 0, 1, 2
STOP_CONVERGED, STOP_MAX_STEPS, STOP_DIVERGED = 1, 2, 3
SERVE_PLAIN, SERVE_NO_GRAPH = 1, 2

_lib = None

_P = C.c_void_p
_SIGS = {
    "ausm_default_params": [C.POINTER(AusmParams)],
    "ausm_set_device": [C.c_int],
    "ausm_device_count": [C.POINTER(C.c_int)],
    "ausm_create": [C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "ausm_destroy": [_P],
    "ausm_dims": [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "ausm_set_engine": [_P, C.c_int],
    "ausm_set_params": [_P, C.POINTER(AusmParams)],
    "ausm_get_params": [_P, C.POINTER(AusmParams)],
    "ausm_set_scheme": [_P, C.c_int],
    "ausm_set_body_naca4": [_P, C.c_int, C.c_double, C.c_double, C.c_int],
    "ausm_naca4_points": [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(C.c_double)],
    "ausm_outer_points": [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)],
    "ausm_set_body_points": [_P, C.POINTER(C.c_double), C.c_int],
    "ausm_set_outer": [_P, C.c_int, C.c_double, C.c_double, C.c_double],
    "ausm_set_radial_stretch": [_P, C.c_double],
    "ausm_generate_grid": [_P, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_int)],
    "ausm_set_vertices": [_P, C.POINTER(C.c_float)],
    "ausm_get_vertices": [_P, C.POINTER(C.c_float)],
    "ausm_init_state": [_P, C.c_int],
    "ausm_set_state": [_P, C.POINTER(C.c_float)],
    "ausm_get_state": [_P, C.POINTER(C.c_float)],
    "ausm_get_state_f64": [_P, C.POINTER(C.c_double)],
    "ausm_step": [_P, C.c_int, C.POINTER(C.c_float)],
    "ausm_max_wave_speed": [_P, C.POINTER(C.c_float)],
    "ausm_forces": [_P, C.POINTER(C.c_double), C.POINTER(C.c_double)],
    "ausm_residual_l2": [_P, C.POINTER(C.c_double)],
    "ausm_field": [_P, C.c_int, C.POINTER(C.c_float)],
    "ausm_forces_noalloc": [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(AusmParams), C.POINTER(C.c_double),
                            C.POINTER(C.c_double), C.c_void_p],
    "ausm_stream": [_P, C.POINTER(C.c_void_p)],
    "ausm_synchronize": [_P],
    "ausm_time_steps": [_P, C.c_int, C.c_int, C.POINTER(C.c_float)],
    "ausm_autotune": [_P, C.c_int, C.POINTER(C.c_int)],
    "ausm_debug_set_wait_polls": [C.c_uint],
    "ausm_batch_create": [C.POINTER(C.c_void_p)],
    "ausm_batch_destroy": [_P],
    "ausm_batch_add": [_P, _P],
    "ausm_batch_remove": [_P, _P],
    "ausm_batch_size": [_P, C.POINTER(C.c_int)],
    "ausm_batch_member": [_P, C.c_int, C.POINTER(C.c_void_p)],
    "ausm_batch_set_graphs": [_P, C.c_int],
    "ausm_batch_step": [_P, C.c_int, C.POINTER(C.c_float)],
    "ausm_batch_residual_l2": [_P, C.POINTER(C.c_double)],
    "ausm_batch_synchronize": [_P],
    "ausm_batch_time_steps": [_P, C.c_int, C.c_int, C.POINTER(C.c_float)],
    "ausm_server_create": [C.c_double, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)],
    "ausm_server_destroy": [_P],
    "ausm_request_bytes": [C.POINTER(AusmRequest), C.POINTER(C.c_double)],
    "ausm_server_submit": [_P, C.POINTER(AusmRequest), C.POINTER(C.c_int64)],
    "ausm_server_pump": [_P, C.POINTER(C.c_int)],
    "ausm_server_start": [_P],
    "ausm_server_stop": [_P],
    "ausm_server_poll": [_P, C.c_int64, C.POINTER(AusmResult), C.POINTER(C.c_double)],
    "ausm_server_drain": [_P, C.c_double],
    "ausm_server_stats": [_P, C.POINTER(AusmServerStats)],
}


def header_functions() -> list[str]:
    """Names of every function declared in include/ausm.h."""
    txt = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|const char\*|void)\s+(ausm_\w+)\s*\(", txt, flags=re.M)))


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise AusmError(ERR_CUDA, f"{LIB_PATH} is not built: run python ausm-webgpu_b200/build.py")
    L = C.CDLL(str(LIB_PATH))
    for name, args in _SIGS.items():
        if hasattr(L, name):
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
    L.ausm_last_error.argtypes = [_P]
    L.ausm_last_error.restype = C.c_char_p
    for name in ("ausm_batch_last_error", "ausm_server_last_error"):
        if hasattr(L, name):
            getattr(L, name).argtypes = [_P]
            getattr(L, name).restype = C.c_char_p
    _lib = L
    return L


def check(rc: int, handle=None, batch=None, server=None):
    if rc != OK:
        if server is not None:
            msg = lib().ausm_server_last_error(server)
        elif batch is not None:
            msg = lib().ausm_batch_last_error(batch)
        else:
            msg = lib().ausm_last_error(handle)
        raise AusmError(rc, msg.decode() if msg else "")
    return rc
