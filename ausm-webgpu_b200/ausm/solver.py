"""Python host of libausm with the reference's operator surface.

Names follow the reference's hooks (src/main.js, src/util.js, src/grid.js):
  prepare_grid()     prepareGrid        main.js:658-707 (grid, then prepareState at rest)
  prepare_state()    prepareState       main.js:631-655
  update_solver()    updateSolver       main.js:629     ("SLAU2" | "SLAU" | "AUSM+-up")
  set_params()       uni.values.*.set   util.js:162-190
  step(n)            one frame of n RK3 steps with dt held fixed, main.js:744-791
  forces()           forceCalc + forceIntegration, main.js:808-810
Every call goes through the C ABI of libausm.so; errors raise AusmError with the
library's message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import AusmError, AusmParams, check, lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_device(device: int):
    """Device for the solvers this thread creates next."""
    check(lib().ausm_set_device(int(device)))


def device_count() -> int:
    n = C.c_int()
    rc = lib().ausm_device_count(C.byref(n))
    return n.value if rc == 0 else 0


def set_wait_polls(polls: int):
    """Test hook: polls (0..65536, the default) of the stage kernels' first bounded wait
    for each TMA box on the current device; 0 makes every such wait give up at once."""
    check(lib().ausm_debug_set_wait_polls(int(polls)))


def default_params() -> AusmParams:
    p = AusmParams()
    check(lib().ausm_default_params(C.byref(p)))
    return p


class Solver:
    """One O-grid solve of M (around the body) x N (radial) cells on the current GPU."""

    def __init__(self, M: int, N: int, engine: str = "fused"):
        self.M, self.N = int(M), int(N)
        h = C.c_void_p()
        check(lib().ausm_create(self.M, self.N, C.byref(h)))
        self.h = h
        if engine != "fused":
            self.set_engine(engine)

    # -- lifetime --
    def close(self):
        if getattr(self, "h", None):
            lib().ausm_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        return check(rc, self.h)

    # -- configuration --
    def set_engine(self, engine: str):
        self._c(lib().ausm_set_engine(self.h, _lib.ENGINES[engine]))

    @property
    def params(self) -> AusmParams:
        p = AusmParams()
        self._c(lib().ausm_get_params(self.h, C.byref(p)))
        return p

    def set_params(self, **kw):
        """Update any AusmParams field: gamma, in_rho, in_pressure, mach, aoa_deg, K_p, K_u,
        cfl, maxdt, muscl, scheme (name or index), ramp."""
        p = self.params
        for k, v in kw.items():
            if k == "scheme" and isinstance(v, str):
                v = _lib.SCHEMES[v]
            if not hasattr(p, k):
                raise AusmError(_lib.ERR_INVALID, f"unknown parameter {k}")
            setattr(p, k, v)
        self._c(lib().ausm_set_params(self.h, C.byref(p)))

    def update_solver(self, name: str):
        self._c(lib().ausm_set_scheme(self.h, _lib.SCHEMES[name]))

    # -- geometry --
    def set_body_naca4(self, digits: int, size: float = 0.3, x_offset: float = -0.7, closed_te: bool = True):
        self._c(lib().ausm_set_body_naca4(self.h, int(digits), float(size), float(x_offset), int(closed_te)))

    def set_body_points(self, xy):
        a = np.ascontiguousarray(xy, dtype=np.float64).reshape(-1, 2)
        self._c(lib().ausm_set_body_points(self.h, _dp(a), a.shape[0]))

    def set_body_dat(self, text: str, size: float = 0.3, x_offset: float = -0.7):
        from .geometry import sample_airfoil
        self.set_body_points(sample_airfoil(text, self.M, size, x_offset))

    def set_outer_rect(self, ratio: float = 1.5):
        self._c(lib().ausm_set_outer(self.h, 0, float(ratio), 0.0, 0.0))

    def set_outer_circle(self, radius: float, center=(0.0, 0.0)):
        self._c(lib().ausm_set_outer(self.h, 1, float(radius), float(center[0]), float(center[1])))

    def set_radial_stretch(self, first_spacing: float):
        self._c(lib().ausm_set_radial_stretch(self.h, float(first_spacing)))

    def generate_grid(self, iters: int = 10000, method: str = "jacobi", tol: float = 0.0) -> int:
        done = C.c_int()
        self._c(lib().ausm_generate_grid(self.h, int(iters), _lib.GRID[method], float(tol), C.byref(done)))
        return done.value

    def prepare_grid(self, iters: int = 10000, method: str = "jacobi", tol: float = 0.0) -> int:
        """prepareGrid: generate the grid and restart the state at rest, as main.js:706 does."""
        done = self.generate_grid(iters, method, tol)
        self.prepare_state("rest")
        return done

    def set_vertices(self, xy):
        a = np.ascontiguousarray(xy, dtype=np.float32).reshape(self.N + 1, self.M, 2)
        self._c(lib().ausm_set_vertices(self.h, _fp(a)))

    def vertices(self) -> np.ndarray:
        a = np.zeros((self.N + 1, self.M, 2), dtype=np.float32)
        self._c(lib().ausm_get_vertices(self.h, _fp(a)))
        return a

    # -- state --
    def prepare_state(self, mode: str = "rest"):
        self._c(lib().ausm_init_state(self.h, _lib.INIT[mode]))

    def set_state(self, q):
        a = np.ascontiguousarray(q, dtype=np.float32).reshape(self.N + 3, self.M, 4)
        self._c(lib().ausm_set_state(self.h, _fp(a)))

    def state(self, out: np.ndarray | None = None) -> np.ndarray:
        """State in the reference layout; `out` (float32, contiguous, e.g. pinned) is
        filled in place when given."""
        a = np.zeros((self.N + 3, self.M, 4), dtype=np.float32) if out is None else out
        if a.dtype != np.float32 or not a.flags.c_contiguous or a.size != (self.N + 3) * self.M * 4:
            raise AusmError(_lib.ERR_INVALID, "out must be a contiguous float32 array of (N+3)*M*4 values")
        self._c(lib().ausm_get_state(self.h, _fp(a)))
        return a

    def state_f64(self) -> np.ndarray:
        """State in the reference layout in double (the F64 engine's own; FP32 engines' widened)."""
        a = np.zeros((self.N + 3, self.M, 4), dtype=np.float64)
        self._c(lib().ausm_get_state_f64(self.h, _dp(a)))
        return a

    def step(self, n: int = 1, wait: bool = True) -> float | None:
        """n RK3 steps with dt fixed from the current state; returns that dt (f32)."""
        if not wait:
            self._c(lib().ausm_step(self.h, int(n), None))
            return None
        dt = C.c_float()
        self._c(lib().ausm_step(self.h, int(n), C.byref(dt)))
        return dt.value

    def max_wave_speed(self) -> float:
        w = C.c_float()
        self._c(lib().ausm_max_wave_speed(self.h, C.byref(w)))
        return w.value

    def forces(self, with_cp: bool = False, chord: float | None = None):
        """Surface force and coefficients as the reference computes them (graphs.js:89-100:
        Cl, Cd are force / dynamic pressure, not divided by the chord); with `chord`, also
        the per-unit-chord coefficients Cl_c = Cl / chord, Cd_c = Cd / chord."""
        out = np.zeros(6)
        cp = np.zeros(self.M) if with_cp else None
        self._c(lib().ausm_forces(self.h, _dp(out), _dp(cp) if cp is not None else None))
        d = dict(zip(("Fx", "Fy", "F", "Cl", "Cd", "ClCd"), out.tolist()))
        if chord is not None:
            d["Cl_c"], d["Cd_c"] = d["Cl"] / chord, d["Cd"] / chord
        if with_cp:
            d["Cp"] = cp
        return d

    def residual_l2(self) -> float:
        r = C.c_double()
        self._c(lib().ausm_residual_l2(self.h, C.byref(r)))
        return r.value

    def field(self, kind: str = "density") -> np.ndarray:
        a = np.zeros((self.N, self.M), dtype=np.float32)
        self._c(lib().ausm_field(self.h, _lib.FIELDS[kind], _fp(a)))
        return a

    def synchronize(self):
        self._c(lib().ausm_synchronize(self.h))

    def autotune(self, force: bool = False) -> int:
        """Tile height (8, 16 or 32 rows) of the fused stage kernel for this solve, measured
        on first use (or again with force); returns the height in use."""
        r = C.c_int()
        self._c(lib().ausm_autotune(self.h, int(bool(force)), C.byref(r)))
        return r.value

    def time_steps(self, n: int, reps: int) -> float:
        """Device time (ms) of `reps` calls of step(n), CUDA events on the solver's stream."""
        ms = C.c_float()
        self._c(lib().ausm_time_steps(self.h, int(n), int(reps), C.byref(ms)))
        return ms.value


class Batch:
    """Many solves stepped together: one kernel launch per RK stage and scheme over the
    tiles of every member (no counterpart in the reference, which steps one grid).

    Members keep their own dt, scheme and parameters; a member's results are the same
    alone or in any batch.  The n-step sequence is replayed from a CUDA graph."""

    def __init__(self, graphs: bool = True):
        b = C.c_void_p()
        check(lib().ausm_batch_create(C.byref(b)))
        self.b = b
        self._members: dict[int, Solver] = {}  # handle address -> Solver, kept alive here
        if not graphs:
            self.set_graphs(False)

    def close(self):
        if getattr(self, "b", None):
            lib().ausm_batch_destroy(self.b)
            self.b = None
            self._members = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        n = C.c_int()
        self._c(lib().ausm_batch_size(self.b, C.byref(n)))
        return n.value

    def _c(self, rc):
        return check(rc, batch=self.b)

    @property
    def members(self) -> list[Solver]:
        """Current members in the library's order (a destroyed solver has left)."""
        out = []
        for k in range(len(self)):
            h = C.c_void_p()
            self._c(lib().ausm_batch_member(self.b, k, C.byref(h)))
            out.append(self._members[h.value])
        return out

    def add(self, s: Solver):
        self._c(lib().ausm_batch_add(self.b, s.h))
        self._members[s.h.value] = s

    def remove(self, s: Solver):
        self._c(lib().ausm_batch_remove(self.b, s.h))
        self._members.pop(s.h.value, None)

    def set_graphs(self, enable: bool):
        self._c(lib().ausm_batch_set_graphs(self.b, int(bool(enable))))

    def step(self, n: int = 1, wait: bool = True) -> np.ndarray | None:
        """n RK3 steps of every member; with wait, returns an (members, 2) array of the
        dt used and the max wave speed after the steps."""
        if not wait:
            self._c(lib().ausm_batch_step(self.b, int(n), None))
            return None
        out = np.zeros((len(self), 2), dtype=np.float32)
        self._c(lib().ausm_batch_step(self.b, int(n), _fp(out) if out.size else None))
        return out

    def residual_l2(self) -> np.ndarray:
        out = np.zeros(len(self))
        if out.size:
            self._c(lib().ausm_batch_residual_l2(self.b, _dp(out)))
        return out

    def synchronize(self):
        self._c(lib().ausm_batch_synchronize(self.b))

    def time_steps(self, n: int, reps: int) -> float:
        """Device time (ms) of `reps` calls of step(n, wait=False)."""
        ms = C.c_float()
        self._c(lib().ausm_batch_time_steps(self.b, int(n), int(reps), C.byref(ms)))
        return ms.value


def make_request(M: int, N: int, naca4: int = 12, body_xy=None, chord: float = 1.0, far_radius: float = 20.0,
                 first_spacing: float = 1e-3, grid_iters: int = 200, init: str = "freestream",
                 residual_drop: float = 4.0, max_steps: int = 50000, closed_te: bool = True, **flow):
    """An AusmRequest; flow keywords are AusmParams fields (mach, aoa_deg, scheme, cfl, ...)
    over the library defaults with cfl 0.5 and no dt cap.  The returned request keeps
    a reference to the body array it points at."""
    p = default_params()
    p.cfl, p.maxdt = 0.5, float("inf")
    for k, v in flow.items():
        if k == "scheme" and isinstance(v, str):
            v = _lib.SCHEMES[v]
        if not hasattr(p, k):
            raise AusmError(_lib.ERR_INVALID, f"unknown parameter {k}")
        setattr(p, k, v)
    r = _lib.AusmRequest()
    r.M, r.N, r.naca4, r.closed_te = int(M), int(N), int(naca4), int(bool(closed_te))
    if body_xy is not None:
        body = np.ascontiguousarray(body_xy, dtype=np.float64).reshape(-1, 2)
        r.body_xy = _dp(body)
        r._body = body  # keeps the array alive while the request is
    r.chord, r.far_radius, r.first_spacing = float(chord), float(far_radius), float(first_spacing)
    r.grid_iters, r.init_mode = int(grid_iters), _lib.INIT[init]
    r.params = p
    r.residual_drop, r.max_steps = float(residual_drop), int(max_steps)
    return r


def request_bytes(r) -> float:
    b = C.c_double()
    check(lib().ausm_request_bytes(C.byref(r), C.byref(b)))
    return b.value


class Server:
    """Continuous-batching solve server (no counterpart in the reference): requests are
    admitted in arrival order by HBM budget and slots, stepped together in rounds of
    `chunk_steps` RK3 steps, and retired at their own stopping rule."""

    def __init__(self, hbm_budget_bytes: float = 160e9, max_active: int = 256, chunk_steps: int = 100,
                 plain: bool = False, graphs: bool = True):
        s = C.c_void_p()
        flags = (_lib.SERVE_PLAIN if plain else 0) | (0 if graphs else _lib.SERVE_NO_GRAPH)
        check(lib().ausm_server_create(float(hbm_budget_bytes), int(max_active), int(chunk_steps), flags,
                                       C.byref(s)))
        self.s = s
        self._M = {}

    def close(self):
        if getattr(self, "s", None):
            lib().ausm_server_destroy(self.s)
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        return check(rc, server=self.s)

    def submit(self, r) -> int:
        i = C.c_int64()
        self._c(lib().ausm_server_submit(self.s, C.byref(r), C.byref(i)))
        self._M[i.value] = (r.M, r.chord)
        return i.value

    def pump(self) -> int:
        left = C.c_int()
        self._c(lib().ausm_server_pump(self.s, C.byref(left)))
        return left.value

    def start(self):
        self._c(lib().ausm_server_start(self.s))

    def stop(self):
        self._c(lib().ausm_server_stop(self.s))

    def drain(self, timeout_s: float | None = None):
        self._c(lib().ausm_server_drain(self.s, -1.0 if timeout_s is None else timeout_s * 1e3))

    def poll(self, rid: int, with_cp: bool = True) -> dict:
        res = _lib.AusmResult()
        M, chord = self._M.get(rid, (0, 1.0))
        cp = np.full(M, np.nan) if with_cp else None
        self._c(lib().ausm_server_poll(self.s, int(rid), C.byref(res),
                                       _dp(cp) if cp is not None and cp.size else None))
        d = {k: getattr(res, k) for k, _ in res._fields_ if k != "forces"}
        d.update(zip(("Fx", "Fy", "F", "Cl", "Cd", "ClCd"), list(res.forces)))
        d["Cl_c"], d["Cd_c"] = d["Cl"] / chord, d["Cd"] / chord  # per unit chord
        if with_cp:
            d["Cp"] = cp
        return d

    def stats(self) -> dict:
        st = _lib.AusmServerStats()
        self._c(lib().ausm_server_stats(self.s, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}
