"""The oracle restatement against the reference's own shaders (golden fixtures).

The fixtures were produced by tests/golden/make_golden.py from the reference's WGSL
compute shaders compiled for the CPU; in float32 without contraction the restatement
must reproduce them bit for bit.
"""
import numpy as np
import pytest

from golden_cases import GRIDS, RUNS, grid_of, params_of
from oracle.oracle import Oracle, RefWGSL, make_params, ref_available


@pytest.mark.parametrize("gname", GRIDS)
def test_grid_generation_bit_exact(golden, gname):
    M, N, naca, iters = (int(x) for x in golden[f"{gname}/meta"])
    o = Oracle(M, N, "f32")
    v = np.zeros((N + 1, M, 2), np.float32)
    v[0], v[N] = golden[f"{gname}/body"], golden[f"{gname}/outer"]
    o.set_vertices(v)
    o.grid_interpolate()
    prev = o.grid_jacobi(iters, want_prev=True)
    assert np.array_equal(o.vertices(), golden[f"{gname}/gridPoints1"])
    assert np.array_equal(prev, golden[f"{gname}/gridPoints0"])
    o.metrics()
    area, fl = o.get_metrics()
    assert np.array_equal(area, golden[f"{gname}/area"])
    assert np.array_equal(fl, golden[f"{gname}/faceLengths"])


@pytest.mark.parametrize("name", RUNS)
def test_solver_bit_exact(golden, name):
    gname, M, N, grid = grid_of(golden, name)
    o = Oracle(M, N, "f32")
    o.set_params(params_of(golden, name))
    o.set_vertices(grid)
    o.metrics()
    o.init_state(int(golden[f"{name}/mode"][0]))
    assert np.float32(o.max_wave()) == golden[f"{name}/maxwave0"][0]
    for k, n in enumerate(golden[f"{name}/frames"]):
        dt = o.step(int(n))
        assert np.float32(dt) == golden[f"{name}/dt{k}"][0]
        q = o.state()
        ref = golden[f"{name}/state{k}"]
        # interior rows are the state; ghost rows of state2 are the reference's stale
        # boundary-pass output and are not part of the result
        assert np.array_equal(q[1:N + 1], ref[1:N + 1]), f"frame {k}: max diff {np.abs(q - ref).max()}"
        assert np.float32(o.max_wave()) == golden[f"{name}/maxwave{k + 1}"][0]
    f = o.forces().astype(np.float32)
    assert np.array_equal(f, golden[f"{name}/forces"])
    assert np.array_equal(o.residual(), golden[f"{name}/residual"])


def test_oracle_f64_tracks_f32(golden):
    """The FP64 instantiation follows the same algorithm: a few steps agree to f32 round-off."""
    name = "run_slau2_m05_a2_fs"
    gname, M, N, grid = grid_of(golden, name)
    res = {}
    for prec in ("f32", "f64"):
        o = Oracle(M, N, prec)
        o.set_params(params_of(golden, name))
        o.set_vertices(grid)
        o.metrics()
        o.init_state(1)
        o.step(5)
        res[prec] = o.state()[1:N + 1].astype(np.float64)
    scale = np.abs(res["f64"]).max(axis=(0, 1))
    err = (np.abs(res["f32"] - res["f64"]).max(axis=(0, 1)) / scale)
    assert np.all(err < 1e-5), err


@pytest.mark.skipif(not ref_available(), reason="reference shader build not present")
def test_reference_build_reproduces_fixture(golden):
    """Where the reference shader build exists, it still reproduces the committed fixture."""
    name = "run_slau_m2_a0_fs"
    gname, M, N, grid = grid_of(golden, name)
    r = RefWGSL(M, N)
    r.set_uniforms(params_of(golden, name))
    r.set_grid(grid)
    r.prepare_state(1)
    r.frame(1)
    assert np.array_equal(r.texture("state2")[1:N + 1], golden[f"{name}/state0"][1:N + 1])


@pytest.mark.skipif(not ref_available(), reason="reference shader build not present")
def test_reference_field_probe(golden):
    """The field probe of the reference's visualization shader returns the shader's own
    per-cell quantities: density is state2's rho, temperature p / rho and Mach |v| / a,
    computed here in float32 in the shader's operation order."""
    name = "run_slau2_m08_a4_odd"
    gname, M, N, grid = grid_of(golden, name)
    r = RefWGSL(M, N)
    p = params_of(golden, name)
    r.set_uniforms(p)
    r.set_grid(grid)
    r.prepare_state(1)
    r.frame(2)
    q = r.texture("state2")[1:N + 1]
    rho, mx, my, E = (q[..., k] for k in range(4))
    f32 = np.float32
    u, v = mx / rho, my / rho
    pres = (E - f32(0.5) * rho * (u * u + v * v)) * (f32(p.gamma) - f32(1.0))
    T = pres / rho
    mach = np.sqrt(u * u + v * v) / np.sqrt(f32(p.gamma) * T)
    assert np.array_equal(r.field("density"), rho)
    assert np.array_equal(r.field("pressure"), pres)
    assert np.array_equal(r.field("temperature"), T)
    assert np.array_equal(r.field("mach"), mach)
    r.close()
