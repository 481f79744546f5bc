"""ausm_forces_noalloc against ausm_forces, through the C ABI.

The no-allocation entry point serves hosts that cannot call cudaMalloc where they need
the forces (hosts that own every device buffer through their own pool, hosts that must
avoid an allocation's implicit synchronisation, hosts without a solver handle).  The test
hands it device copies of a solver's wall row and body vertices, made here with torch
(the test may allocate; the entry point does not), and checks Fx, Fy, Cl, Cd and Cp
against the handle-based ausm_forces on two calls in a row, with the state advanced in
between.  Tolerance: 1e-4 relative, as the force parity tests.  The second call must
also leave the device's free memory unchanged (cudaMemGetInfo, through torch); the first
call is exempt, because its one-time set-up may load the library's device code.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _params(**kw):
    from ausm import default_params
    p = default_params()
    for k, v in dict(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=0.8, aoa_deg=2.0, cfl=0.5, maxdt=math.inf,
                     muscl=1, scheme=0, ramp=0.0, **kw).items():
        setattr(p, k, v)
    return p


def test_forces_noalloc_matches_forces_twice():
    import torch

    from ausm import Solver, _lib
    L = _lib.lib()
    M, N = 256, 96
    p = _params()
    s = Solver(M, N)
    s.set_body_naca4(2412, 0.3, -0.7)
    s.set_outer_rect(1.5)
    s.generate_grid(300)
    s._c(L.ausm_set_params(s.h, C.byref(p)))
    s.prepare_state("freestream")
    s.step(40)
    for call in range(2):
        ref = s.forces(with_cp=True)
        q, v = s.state(), s.vertices()
        wall = torch.from_numpy(np.ascontiguousarray(q[1])).cuda()  # M x float4, first interior row
        body = torch.from_numpy(np.ascontiguousarray(v[0])).cuda()  # M x float2, body vertices
        torch.cuda.synchronize()
        out = np.zeros(6)
        cp = np.zeros(M)
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.ausm_forces_noalloc(C.c_void_p(wall.data_ptr()), C.c_void_p(body.data_ptr()), M, C.byref(p),
                                   out.ctypes.data_as(C.POINTER(C.c_double)),
                                   cp.ctypes.data_as(C.POINTER(C.c_double)), None)
        assert rc == 0, L.ausm_last_error(None)
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free0, "the call changed the device's free memory"
        scale = math.hypot(ref["Fx"], ref["Fy"])
        assert abs(out[0] - ref["Fx"]) <= TOL * scale and abs(out[1] - ref["Fy"]) <= TOL * scale, call
        cscale = max(abs(ref["Cl"]), abs(ref["Cd"]))
        assert abs(out[3] - ref["Cl"]) <= TOL * cscale and abs(out[4] - ref["Cd"]) <= TOL * cscale, call
        assert np.abs(cp - ref["Cp"]).max() <= TOL * np.abs(ref["Cp"]).max(), call
        s.step(25)  # a different state for the second call
    s.close()


def test_forces_noalloc_rejects_oversized_grid():
    from ausm import _lib
    L = _lib.lib()
    p = _params()
    out = np.zeros(6)
    rc = L.ausm_forces_noalloc(C.c_void_p(16), C.c_void_p(16), 16385, C.byref(p),
                               out.ctypes.data_as(C.POINTER(C.c_double)), None, None)
    assert rc == _lib.ERR_INVALID
    assert b"16384" in L.ausm_last_error(None)
