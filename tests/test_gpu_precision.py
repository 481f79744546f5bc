"""Precision: the full-FP64 engine against the FP64 oracle, and the FP32 engines'
error against FP64.

The F64 engine (kernels_f64.cu) follows the FP32 exact path operation by operation in
double; on the same grid and parameters it must agree with the oracle's double
instantiation to 1e-12 (normwise relative, per conserved component) after several
RK3 frames.  The FP32 fused engine's error against the FP64 solution is then measured
and bounded (the FP32 arithmetic itself, ~1e-7 per operation, grows over the steps);
the bounds below are the stated accuracy of the FP32 path on these cases."""
import math

import numpy as np
import pytest

from golden_cases import grid_of, kwargs_of

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12
TOL_F32_VS_F64 = 1e-4  # after the golden cases' frames, normwise relative

CASES = ["run_slau2_m05_a2_fs", "run_ausmup_m8_a0_fs", "run_slau_m6_odd"]


def lib_kwargs(kw):
    out = dict(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=0.5, aoa_deg=0.0, K_p=0.0, K_u=0.75, cfl=0.5,
               maxdt=math.inf, muscl=1, scheme="SLAU2", ramp=0.0)
    out.update(kw)
    return out


def normwise(a, b):
    a = np.asarray(a, np.float64).reshape(-1, 4)
    b = np.asarray(b, np.float64).reshape(-1, 4)
    m = np.abs(b).max(axis=0)
    mom = max(m[1], m[2], 1.0)
    return (np.abs(a - b).max(axis=0) / np.array([m[0], mom, mom, m[3]])).max()


def setup(golden, name, engine):
    from ausm import Solver
    gname, M, N, grid = grid_of(golden, name)
    s = Solver(M, N, engine=engine)
    s.set_vertices(grid)
    kw = lib_kwargs(kwargs_of(golden, name))
    s.set_params(**kw)
    mode = int(golden[f"{name}/mode"][0])
    s.prepare_state("rest" if mode == 0 else "freestream")
    return s, M, N, grid, kw, mode


def oracle_run(M, N, grid, kw, mode, frames):
    from oracle.oracle import Oracle, make_params
    p = make_params(mach=kw["mach"], aoa_deg=kw["aoa_deg"], gamma=kw["gamma"], in_rho=kw["in_rho"],
                    in_pressure=kw["in_pressure"], K_p=kw["K_p"], K_u=kw["K_u"], cfl=kw["cfl"], maxdt=kw["maxdt"],
                    muscl=kw["muscl"], scheme=kw["scheme"])
    o = Oracle(M, N, "f64")
    o.set_params(p)
    o.set_vertices(np.asarray(grid, np.float64))
    o.metrics()
    o.init_state(mode)
    dts = [o.step(int(n)) for n in frames]
    q = o.state()
    o.close()
    return q, dts


@pytest.mark.parametrize("name", CASES)
def test_f64_engine_matches_f64_oracle(golden, name):
    s, M, N, grid, kw, mode = setup(golden, name, "f64")
    frames = [int(n) for n in golden[f"{name}/frames"]]
    dts = [s.step(n) for n in frames]
    q = s.state_f64()[1:N + 1]
    ref, rdts = oracle_run(M, N, grid, kw, mode, frames)
    d = normwise(q, ref[1:N + 1])
    assert d <= TOL_F64, f"F64 engine vs FP64 oracle: {d:.3e}"
    for a, b in zip(dts, rdts):
        assert a == pytest.approx(np.float32(b), rel=1e-6)
    s.close()


@pytest.mark.parametrize("name", CASES)
def test_f32_error_against_f64(golden, name):
    """FP32 fused engine vs the FP64 engine on the same grid, same frames."""
    frames = [int(n) for n in golden[f"{name}/frames"]]
    res = {}
    for engine in ("fused", "f64"):
        s, M, N, grid, kw, mode = setup(golden, name, engine)
        for n in frames:
            s.step(n)
        res[engine] = s.state_f64()[1:N + 1]
        res[engine, "F"] = s.forces(with_cp=True)
        s.close()
    d = normwise(res["fused"], res["f64"])
    print(f"{name}: FP32 fused vs FP64, normwise max relative error {d:.3e}")
    assert d <= TOL_F32_VS_F64
    cp32, cp64 = res["fused", "F"]["Cp"], res["f64", "F"]["Cp"]
    assert np.abs(cp32 - cp64).max() <= TOL_F32_VS_F64 * max(np.abs(cp64).max(), 1.0)


def test_engine_switch_round_trip(golden):
    """fused -> f64 -> fused carries the state through the float reference layout."""
    name = CASES[0]
    s, M, N, grid, kw, mode = setup(golden, name, "fused")
    s.step(3)
    q0 = s.state()[1:N + 1]  # interior rows; the ghost rows are recomputed by each engine
    s.set_engine("f64")
    np.testing.assert_array_equal(s.state()[1:N + 1], q0)
    s.step(2)
    q64 = s.state_f64()[1:N + 1]
    s.set_engine("fused")
    np.testing.assert_array_equal(s.state()[1:N + 1], q64.astype(np.float32))
    assert math.isfinite(s.residual_l2()) and math.isfinite(s.forces()["Cl"])
    s.close()
