"""Edge sizes on the GPU: the smallest grids (M = 4, N = 2), odd M, M below one tile
width, N below one tile height, and M / N that leave partial tiles, for every tile
height of the TMA stage kernel and for the batched kernel.  The fused engine is
checked against the reference-shaped engine (the reference's arithmetic, bit-exact
with the oracle) on the same analytic annulus grid: within the fused-engine bound of
1e-5 normwise after one step, and finite after a short run."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(4, 2), (5, 3), (7, 2), (33, 17), (100, 3), (31, 40), (64, 16)]


def annulus(M, N, r0=0.5, r1=4.0):
    """Vertices of an O-grid between circles r0 and r1: row 0 the body, CCW from theta=0,
    radii growing geometrically."""
    th = 2 * math.pi * np.arange(M) / M
    r = r0 * (r1 / r0) ** (np.arange(N + 1) / N)
    v = np.zeros((N + 1, M, 2), np.float32)
    v[..., 0] = r[:, None] * np.cos(th)[None, :]
    v[..., 1] = r[:, None] * np.sin(th)[None, :]
    return v


PARAMS = dict(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=0.6, aoa_deg=3.0, K_p=0.0, K_u=0.75, cfl=0.5,
              maxdt=math.inf, muscl=1, scheme="SLAU2", ramp=0.0)


def solver(M, N, engine="fused", **kw):
    from ausm import Solver
    s = Solver(M, N, engine=engine)
    s.set_vertices(annulus(M, N))
    s.set_params(**dict(PARAMS, **kw))
    s.prepare_state("freestream")
    return s


def normwise(a, b):
    a = np.asarray(a, np.float64).reshape(-1, 4)
    b = np.asarray(b, np.float64).reshape(-1, 4)
    m = np.abs(b).max(axis=0)
    mom = max(m[1], m[2], 1.0)
    return (np.abs(a - b).max(axis=0) / np.array([m[0], mom, mom, m[3]])).max()


@pytest.mark.parametrize("M,N", SIZES)
@pytest.mark.parametrize("scheme", ["SLAU2", "AUSM+-up"])
def test_edge_sizes_fused_vs_reference(M, N, scheme, monkeypatch):
    ref = solver(M, N, "reference", scheme=scheme)
    ref.step(1)
    q_ref = ref.state()[1:N + 1]
    ref.step(20)
    q_ref20 = ref.state()[1:N + 1]
    ref.close()
    for rows in ("8", "16", "32"):
        monkeypatch.setenv("AUSM_TILE_ROWS", rows)
        s = solver(M, N, scheme=scheme)
        s.step(1)
        d = normwise(s.state()[1:N + 1], q_ref)
        assert d <= 1e-5, f"{M}x{N} rows {rows}: {d:.3e}"
        s.step(20)
        q = s.state()[1:N + 1]
        assert np.all(np.isfinite(q))
        assert normwise(q, q_ref20) <= 1e-4
        assert math.isfinite(s.residual_l2()) and math.isfinite(s.forces()["Cl"])
        s.close()


def test_edge_sizes_in_one_batch():
    """All edge sizes in one batch: each member equals its own single-solve run to 1e-6."""
    from ausm import Batch
    sol = [solver(M, N) for M, N in SIZES]
    ref = [solver(M, N) for M, N in SIZES]
    with Batch() as b:
        for s in sol:
            b.add(s)
        out = b.step(5)
        assert np.all(np.isfinite(out))
        for s, r in zip(sol, ref):
            r.step(5)
            assert normwise(s.state()[1:s.N + 1], r.state()[1:r.N + 1]) <= 1e-6
        assert np.all(np.isfinite(b.residual_l2()))
    for s in sol + ref:
        s.close()
