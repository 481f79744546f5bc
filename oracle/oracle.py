"""ORACLE — test infrastructure only.

ctypes front ends for the two CPU checkers:
  Oracle   the restatement (oracle/ausm_oracle.cpp), float32 or float64
  RefWGSL  the reference's own WGSL compute shaders compiled for the CPU
           (oracle/wgsl_ref/, built under oracle/_ref/ from the reference tree)
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libausm_oracle.so"
REF_SO = HERE / "_ref" / "libausm_ref.so"

SCHEMES = {"SLAU2": 0, "SLAU": 1, "AUSM+-up": 2}


class Params(C.Structure):
    """Uniform fields on the path (util.js:1-29): shared by both checkers."""
    _fields_ = [("gamma", C.c_double), ("in_rho", C.c_double), ("in_pressure", C.c_double),
                ("inflow", C.c_double * 2), ("in_state", C.c_double * 4),
                ("K_p", C.c_double), ("K_u", C.c_double), ("cfl", C.c_double), ("maxdt", C.c_double),
                ("muscl", C.c_int), ("scheme", C.c_int)]


def make_params(mach=0.5, aoa_deg=0.0, gamma=1.4, in_rho=1.0, in_pressure=None, K_p=0.0, K_u=0.75,
                cfl=0.5, maxdt=float("inf"), muscl=1, scheme="SLAU2", inflow_speed=None) -> Params:
    """Freestream as the reference builds it: speed = Mach * sqrt(gamma p/rho), AoA rotates
    the inflow vector (util.js:180-185), inState = (rho, rho u, rho v, p/(g-1) + rho|V|^2/2)
    (main.js:780-784)."""
    import math
    if in_pressure is None:
        in_pressure = 1.0 / gamma
    a_inf = math.sqrt(gamma * in_pressure / in_rho)
    speed = mach * a_inf if inflow_speed is None else inflow_speed
    a = aoa_deg * math.pi / 180
    u, v = speed * math.cos(a), speed * math.sin(a)
    rhoE = in_pressure / (gamma - 1.0) + 0.5 * (speed * speed) * in_rho
    p = Params()
    p.gamma, p.in_rho, p.in_pressure = gamma, in_rho, in_pressure
    p.inflow[0], p.inflow[1] = u, v
    st = (in_rho, u * in_rho, v * in_rho, rhoE)
    for k in range(4):
        p.in_state[k] = st[k]
    p.K_p, p.K_u, p.cfl, p.maxdt = K_p, K_u, cfl, maxdt
    p.muscl = int(muscl)
    p.scheme = SCHEMES[scheme] if isinstance(scheme, str) else int(scheme)
    return p


def _load(path: Path, build):
    if not path.exists():
        build()
    if not path.exists():
        raise FileNotFoundError(path)
    return C.CDLL(str(path))


_olib = None
_rlib = None


def oracle_lib():
    global _olib
    if _olib is None:
        from . import build as _b  # type: ignore
        _olib = _load(ORACLE_SO, _b.build_oracle)
        for suf, ct in (("f32", C.c_float), ("f64", C.c_double)):
            P = C.POINTER(ct)
            L = _olib
            getattr(L, f"orc_create_{suf}").restype = C.c_void_p
            getattr(L, f"orc_create_{suf}").argtypes = [C.c_int, C.c_int]
            for name, args, res in [
                ("destroy", [C.c_void_p], None), ("set_params", [C.c_void_p, C.POINTER(Params)], None),
                ("set_vertices", [C.c_void_p, P], None), ("get_vertices", [C.c_void_p, P], None),
                ("metrics", [C.c_void_p], None), ("get_metrics", [C.c_void_p, P, P], None),
                ("init_state", [C.c_void_p, C.c_int], None), ("set_state", [C.c_void_p, P], None),
                ("get_state", [C.c_void_p, P], None), ("fill_ghosts", [C.c_void_p], None),
                ("step", [C.c_void_p, C.c_int], C.c_double), ("max_wave", [C.c_void_p], C.c_double),
                ("get_wave_speeds", [C.c_void_p, P], None), ("eval_residual", [C.c_void_p, P], None),
                ("get_fluxes", [C.c_void_p, P, P], None),
                ("forces", [C.c_void_p, C.POINTER(C.c_double)], None),
                ("residual_l2", [C.c_void_p], C.c_double), ("grid_interpolate", [C.c_void_p], None),
                ("grid_jacobi", [C.c_void_p, C.c_int, P], None),
                ("grid_multicolor", [C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_double)], C.c_int),
            ]:
                f = getattr(L, f"orc_{name}_{suf}")
                f.argtypes, f.restype = args, res
        _olib.orc_num_threads.restype = C.c_int
        _olib.orc_set_num_threads.argtypes = [C.c_int]
    return _olib


def ref_lib():
    global _rlib
    if _rlib is None:
        from . import build as _b  # type: ignore
        _rlib = _load(REF_SO, _b.build_ref)
        L = _rlib
        F = C.POINTER(C.c_float)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int]
        for name, args, res in [
            ("destroy", [C.c_void_p], None), ("set_uniforms", [C.c_void_p, C.POINTER(Params)], None),
            ("set_boundaries", [C.c_void_p, F, F], None), ("prepare_grid", [C.c_void_p, C.c_int], None),
            ("set_grid", [C.c_void_p, F], None), ("prepare_state", [C.c_void_p, C.c_int], None),
            ("set_state", [C.c_void_p, F], None), ("frame", [C.c_void_p, C.c_int], C.c_double),
            ("eval_residual", [C.c_void_p], None), ("forces", [C.c_void_p, C.POINTER(C.c_double)], None),
            ("max_wave_bits", [C.c_void_p], C.c_uint32), ("get_wave_speeds", [C.c_void_p, F], None),
            ("field", [C.c_void_p, C.c_int, F], None),
            ("texture_size", [C.c_void_p, C.c_int], C.c_longlong), ("get_texture", [C.c_void_p, C.c_int, F], None),
        ]:
            f = getattr(L, f"ref_{name}")
            f.argtypes, f.restype = args, res
    return _rlib


def ref_available() -> bool:
    try:
        ref_lib()
        return True
    except (FileNotFoundError, OSError, RuntimeError):
        return False


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Oracle:
    """The restatement on an M x N O-grid, float32 ("f32") or float64 ("f64")."""

    def __init__(self, M: int, N: int, precision: str = "f32"):
        self.M, self.N = M, N
        self.suf = precision
        self.dt_np = np.float32 if precision == "f32" else np.float64
        self.ct = C.c_float if precision == "f32" else C.c_double
        self.L = oracle_lib()
        self.h = self._f("create")(M, N)

    def _f(self, name):
        return getattr(self.L, f"orc_{name}_{self.suf}")

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, shape):
        return np.zeros(shape, dtype=self.dt_np)

    def set_params(self, p: Params):
        self._f("set_params")(self.h, C.byref(p))

    def set_vertices(self, xy):
        a = np.ascontiguousarray(xy, dtype=self.dt_np).reshape(self.N + 1, self.M, 2)
        self._f("set_vertices")(self.h, _ptr(a, self.ct))

    def vertices(self):
        a = self._arr((self.N + 1, self.M, 2))
        self._f("get_vertices")(self.h, _ptr(a, self.ct))
        return a

    def metrics(self):
        self._f("metrics")(self.h)

    def get_metrics(self):
        area = self._arr((self.N, self.M))
        fl = self._arr((self.N, self.M, 4))
        self._f("get_metrics")(self.h, _ptr(area, self.ct), _ptr(fl, self.ct))
        return area, fl

    def init_state(self, mode: int):
        self._f("init_state")(self.h, mode)

    def set_state(self, q):
        a = np.ascontiguousarray(q, dtype=self.dt_np).reshape(self.N + 3, self.M, 4)
        self._f("set_state")(self.h, _ptr(a, self.ct))

    def state(self):
        a = self._arr((self.N + 3, self.M, 4))
        self._f("get_state")(self.h, _ptr(a, self.ct))
        return a

    def fill_ghosts(self):
        self._f("fill_ghosts")(self.h)

    def step(self, n: int) -> float:
        return self._f("step")(self.h, n)

    def max_wave(self) -> float:
        return self._f("max_wave")(self.h)

    def wave_speeds(self):
        a = self._arr((self.N, self.M))
        self._f("get_wave_speeds")(self.h, _ptr(a, self.ct))
        return a

    def residual(self):
        a = self._arr((self.N, self.M, 4))
        self._f("eval_residual")(self.h, _ptr(a, self.ct))
        return a

    def fluxes(self):
        fx = self._arr((self.N, self.M, 4))
        fy = self._arr((self.N + 1, self.M, 4))
        self._f("get_fluxes")(self.h, _ptr(fx, self.ct), _ptr(fy, self.ct))
        return fx, fy

    def forces(self):
        """Fx, Fy, |F| sign(F.V), Cl, Cd, Cl/Cd (graphs.js:87-100)."""
        out = (C.c_double * 6)()
        self._f("forces")(self.h, out)
        return np.array(list(out))

    def residual_l2(self) -> float:
        return self._f("residual_l2")(self.h)

    def grid_interpolate(self):
        self._f("grid_interpolate")(self.h)

    def grid_jacobi(self, iters: int, want_prev: bool = False):
        if want_prev:
            prev = self._arr((self.N + 1, self.M, 2))
            self._f("grid_jacobi")(self.h, iters, _ptr(prev, self.ct))
            return prev
        self._f("grid_jacobi")(self.h, iters, None)
        return None

    def grid_multicolor(self, iters: int, tol: float):
        mv = C.c_double()
        s = self._f("grid_multicolor")(self.h, iters, tol, C.byref(mv))
        return s, mv.value


class RefWGSL:
    """The reference's own compute shaders on the CPU, driven in main.js's dispatch order."""

    def __init__(self, M: int, N: int):
        self.M, self.N = M, N
        self.L = ref_lib()
        self.h = self.L.ref_create(M, N)

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_uniforms(self, p: Params):
        self.L.ref_set_uniforms(self.h, C.byref(p))

    def set_boundaries(self, body, outer):
        b = np.ascontiguousarray(body, dtype=np.float32).reshape(self.M, 2)
        o = np.ascontiguousarray(outer, dtype=np.float32).reshape(self.M, 2)
        self.L.ref_set_boundaries(self.h, _ptr(b, C.c_float), _ptr(o, C.c_float))

    def prepare_grid(self, iters: int):
        self.L.ref_prepare_grid(self.h, iters)

    def set_grid(self, xy):
        a = np.ascontiguousarray(xy, dtype=np.float32).reshape(self.N + 1, self.M, 2)
        self.L.ref_set_grid(self.h, _ptr(a, C.c_float))

    def prepare_state(self, mode: int):
        self.L.ref_prepare_state(self.h, mode)

    def set_state(self, q):
        a = np.ascontiguousarray(q, dtype=np.float32).reshape(self.N + 3, self.M, 4)
        self.L.ref_set_state(self.h, _ptr(a, C.c_float))

    def frame(self, steps: int) -> float:
        return self.L.ref_frame(self.h, steps)

    def eval_residual(self):
        self.L.ref_eval_residual(self.h)

    def forces(self):
        out = (C.c_double * 6)()
        self.L.ref_forces(self.h, out)
        return np.array(list(out))

    def max_wave(self) -> float:
        return float(np.array([self.L.ref_max_wave_bits(self.h)], dtype=np.uint32).view(np.float32)[0])

    def wave_speeds(self):
        a = np.zeros((self.N, self.M), dtype=np.float32)
        self.L.ref_get_wave_speeds(self.h, _ptr(a, C.c_float))
        return a

    # display modes of the visualization shader (ausm.js:667-695) with a raw field value
    FIELD_MODES = {"density": 2, "temperature": 3, "pressure": 4, "mach": 5, "entropy": 8}

    def field(self, name: str):
        """The visualization shader's raw value of a field for state2 (M x N, before the
        colour map), from translate.py's field probe of the reference's shader."""
        a = np.zeros((self.N, self.M), dtype=np.float32)
        self.L.ref_field(self.h, self.FIELD_MODES[name], _ptr(a, C.c_float))
        return a

    TEX = {"gridPoints0": (0, 2), "gridPoints1": (1, 2), "gridArea": (2, 1), "faceLengths": (3, 4),
           "state0": (4, 4), "state1": (5, 4), "state2": (6, 4), "fluxX": (7, 4), "fluxY": (8, 4),
           "residual": (9, 4)}

    def texture(self, name: str):
        which, ch = self.TEX[name]
        n = self.L.ref_texture_size(self.h, which)
        a = np.zeros(n, dtype=np.float32)
        self.L.ref_get_texture(self.h, which, _ptr(a, C.c_float))
        shapes = {"gridPoints0": (self.N + 1, self.M), "gridPoints1": (self.N + 1, self.M),
                  "gridArea": (self.N, self.M), "faceLengths": (self.N, self.M),
                  "state0": (self.N + 3, self.M), "state1": (self.N + 3, self.M), "state2": (self.N + 3, self.M),
                  "fluxX": (self.N, self.M + 1), "fluxY": (self.N + 1, self.M), "residual": (self.N, self.M)}
        return a.reshape(*shapes[name], ch) if ch > 1 else a.reshape(shapes[name])
