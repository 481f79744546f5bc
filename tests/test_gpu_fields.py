"""Headless field outputs (ausm_field) against the reference's own visualization shader.

The reference computes density, temperature, pressure, Mach number and entropy per
cell in visualizationShaderCode (src/shaders/ausm.js:612-695) and then colour-maps them
into an 8-bit texture; the field probe of oracle/wgsl_ref/translate.py is that shader
with only the final colour-mapped store replaced by a store of the raw value, so the
comparison is against the reference's arithmetic.  The wave speed is the shader's own
f32 buffer (ausm.js:617-624).  The same state is injected into the reference build
(after a few of its own frames) and into the library.

Tolerances: density, pressure, temperature and Mach use IEEE operations in the same
order on both sides (the library is compiled with -fmad=false, the reference build
with -ffp-contract=off): bit for bit.  Entropy log(p / rho^gamma) goes through CUDA's
logf / powf and the host's libm: 2e-6 of max(1, |s|).  Wave speed: the library
recomputes the face lengths and area from the vertices in the reference's formulas,
bit for bit as well.
"""
import numpy as np
import pytest

from golden_cases import grid_of, kwargs_of, params_of
from oracle.oracle import RefWGSL, ref_available
from test_gpu_parity import lib_kwargs

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref_available(), reason="reference shader build not present")]

CASES = ["run_slau2_m08_a4_odd", "run_ausmup_m8_a0_fs", "run_slau_m6_odd"]
FIELDS = ["density", "pressure", "temperature", "mach", "entropy"]


def reference_state(golden, name, frames=3):
    gname, M, N, grid = grid_of(golden, name)
    r = RefWGSL(M, N)
    r.set_uniforms(params_of(golden, name))
    r.set_grid(grid)
    r.prepare_state(1)
    r.frame(frames)
    q = r.texture("state2")
    r.set_state(q)  # the visualization pass of main.js:649-652 on this state
    return r, q, grid, M, N


@pytest.mark.parametrize("engine", ["fused", "reference"])
@pytest.mark.parametrize("name", CASES)
def test_fields_match_reference_shader(golden, name, engine):
    import ausm
    r, q, grid, M, N = reference_state(golden, name)
    s = ausm.Solver(M, N, engine=engine)
    s.set_vertices(grid)
    s.set_params(**lib_kwargs(kwargs_of(golden, name)))
    s.set_state(q)
    for f in FIELDS:
        ours = s.field(f)
        ref = r.field(f)
        assert ours.shape == ref.shape == (N, M)
        assert np.all(np.isfinite(ref))
        if f == "entropy":
            err = np.abs(ours.astype(np.float64) - ref) / np.maximum(1.0, np.abs(ref))
            assert err.max() <= 2e-6, f"{f}: {err.max():.3e}"
        else:
            assert np.array_equal(ours, ref), f"{f}: max diff {np.abs(ours - ref).max():.3e}"
    assert np.array_equal(s.field("wave_speed"), r.wave_speeds())
    s.close()
    r.close()
