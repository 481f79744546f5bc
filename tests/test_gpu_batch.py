"""Batched stepping (ausm_batch_*) against the same solves stepped alone.

Each solve's arithmetic in the batched kernel depends only on its own grid, state,
parameters and dt, so a member's state after n steps must be bit-identical alone (a
batch of one) and in any mix, with graphs on or off, across membership changes.  The
single-solve path (ausm_step, its own kernels) computes the same tile arithmetic; it is
checked to 1e-6 normwise relative (the fused-engine tolerance scale of
test_gpu_parity.py, tightened)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (M, N, naca, mach, aoa, scheme, ramp): uneven sizes, odd M, M below one tile width,
# N not a multiple of the tile height, all three schemes, one ramped start
SPECS = [
    (128, 96, 2412, 0.8, 2.0, "SLAU2", 0.0),
    (131, 50, 12, 2.0, 0.0, "AUSM+-up", 0.0),
    (20, 9, 4415, 0.5, -3.0, "SLAU", 0.0),
    (256, 160, 6409, 3.0, 6.0, "SLAU2", 0.0),
    (64, 33, 2318, 1.2, 1.0, "SLAU", 50.0),
]


@pytest.fixture(scope="module")
def grids():
    from ausm import Solver
    out = []
    for M, N, naca, *_ in SPECS:
        with Solver(M, N) as s:
            s.set_body_naca4(naca, 0.5, 0.0)
            s.set_outer_circle(10.0)
            s.set_radial_stretch(2e-3)
            s.generate_grid(300, "multicolor")
            out.append(s.vertices())
    return out


def make(k, grids):
    from ausm import Solver
    M, N, naca, mach, aoa, scheme, ramp = SPECS[k]
    s = Solver(M, N)
    s.set_vertices(grids[k])
    s.set_params(mach=mach, aoa_deg=aoa, scheme=scheme, cfl=0.5, maxdt=math.inf, ramp=ramp)
    s.prepare_state("freestream")
    return s


def normwise(a, b):
    a = np.asarray(a, np.float64).reshape(-1, 4)
    b = np.asarray(b, np.float64).reshape(-1, 4)
    m = np.abs(b).max(axis=0)
    mom = max(m[1], m[2], 1.0)
    return (np.abs(a - b).max(axis=0) / np.array([m[0], mom, mom, m[3]])).max()


def run_alone(k, grids, frames):
    from ausm import Batch
    s = make(k, grids)
    with Batch() as b:
        b.add(s)
        dts = [b.step(n)[0].copy() for n in frames]
    q = s.state()
    s.close()
    return q, dts


FRAMES = (7, 5, 1)


def test_batch_same_alone_and_in_mix(grids):
    from ausm import Batch
    alone = [run_alone(k, grids, FRAMES) for k in range(len(SPECS))]
    sol = [make(k, grids) for k in range(len(SPECS))]
    with Batch() as b:
        for s in sol:
            b.add(s)
        for f, n in enumerate(FRAMES):
            out = b.step(n)
            for k in range(len(SPECS)):
                assert out[k, 0] == alone[k][1][f][0], f"dt of member {k}, frame {f}"
                assert out[k, 1] == alone[k][1][f][1], f"wave speed of member {k}, frame {f}"
        for k, s in enumerate(sol):
            np.testing.assert_array_equal(s.state(), alone[k][0], err_msg=f"member {k}")
    for s in sol:
        s.close()


def test_batch_graphs_off_identical(grids):
    from ausm import Batch
    qs = []
    for graphs in (True, False):
        sol = [make(k, grids) for k in range(len(SPECS))]
        with Batch(graphs=graphs) as b:
            for s in sol:
                b.add(s)
            for n in FRAMES:
                b.step(n, wait=False)
            b.synchronize()
        qs.append([s.state() for s in sol])
        for s in sol:
            s.close()
    for a, c in zip(*qs):
        np.testing.assert_array_equal(a, c)


def test_batch_matches_single_solve_path(grids):
    from ausm import Batch
    sol = [make(k, grids) for k in range(len(SPECS))]
    ref = [make(k, grids) for k in range(len(SPECS))]
    with Batch() as b:
        for s in sol:
            b.add(s)
        for n in FRAMES:
            b.step(n)
            for r in ref:
                r.step(n)
        for k in range(len(SPECS)):
            d = normwise(sol[k].state(), ref[k].state())
            assert d <= 1e-6, f"member {k}: {d:.3e}"
            assert sol[k].max_wave_speed() == pytest.approx(ref[k].max_wave_speed(), rel=1e-6)
    for s in sol + ref:
        s.close()


def test_batch_membership_changes(grids):
    """Members leave and join between step calls; every member still follows its
    alone trajectory, and a removed member keeps stepping on its own stream."""
    from ausm import Batch
    frames = (3, 4, 2)
    alone = [run_alone(k, grids, frames) for k in range(len(SPECS))]
    sol = [make(k, grids) for k in range(len(SPECS))]
    with Batch() as b:
        for s in sol[:3]:
            b.add(s)
        b.step(frames[0])
        b.remove(sol[1])
        b.add(sol[3])
        sol[1].step(frames[1])  # frame 1 of its own sequence, alone
        b.step(frames[1])
        b.add(sol[1])
        sol[3].close()  # destroying a member removes it from the batch
        assert len(b) == 3
        b.step(frames[2])
    # sol[0], sol[2]: all three frames in the batch
    for k in (0, 2):
        np.testing.assert_array_equal(sol[k].state(), alone[k][0])
    # sol[1]: frame 0 in the batch, frame 1 alone (ausm_step), frame 2 in the batch
    d = normwise(sol[1].state(), alone[1][0])
    assert d <= 1e-6, d
    for k in (0, 1, 2):
        sol[k].close()


def test_batch_residual_norms(grids):
    from ausm import Batch
    sol = [make(k, grids) for k in range(len(SPECS))]
    with Batch() as b:
        for s in sol:
            b.add(s)
        b.step(4)
        l2 = b.residual_l2()
        for k, s in enumerate(sol):
            assert l2[k] == pytest.approx(s.residual_l2(), rel=1e-9), k
            assert math.isfinite(l2[k]) and l2[k] > 0
    for s in sol:
        s.close()


def test_batch_errors(grids):
    from ausm import AusmError, Batch, Solver
    from ausm import _lib
    s = make(0, grids)
    t = make(1, grids)
    with Batch() as b, Batch() as b2:
        b.add(s)
        with pytest.raises(AusmError) as e:
            b.add(s)
        assert e.value.code == _lib.ERR_STATE
        with pytest.raises(AusmError) as e:
            b2.add(s)
        assert e.value.code == _lib.ERR_STATE
        with pytest.raises(AusmError) as e:
            b.remove(t)
        assert e.value.code == _lib.ERR_NOT_FOUND
        with pytest.raises(AusmError) as e:
            s.set_engine("reference")
        assert e.value.code == _lib.ERR_STATE
        with Solver(64, 32) as bare:  # no grid, no state
            with pytest.raises(AusmError) as e:
                b.add(bare)
            assert e.value.code == _lib.ERR_STATE
        t.set_engine("reference")
        with pytest.raises(AusmError) as e:
            b.add(t)
        assert e.value.code == _lib.ERR_STATE
    s.close()
    t.close()


def test_batch_tile_heights_bit_identical(grids, monkeypatch):
    """The batch laid out with 8-, 16- and 32-row tiles gives the same state bits, and the
    same residual norms (they are summed over fixed chunks of each solve's cells, not
    over the batch's tiles)."""
    from ausm import Batch
    out = {}
    for rows in ("8", "16", "32"):
        monkeypatch.setenv("AUSM_TILE_ROWS", rows)
        sol = [make(k, grids) for k in range(len(SPECS))]
        with Batch() as b:
            for s in sol:
                b.add(s)
            for n in FRAMES:
                b.step(n)
            l2 = b.residual_l2()
        out[rows] = ([s.state() for s in sol], l2)
        for s in sol:
            s.close()
    for rows in ("8", "32"):
        for a, c in zip(out[rows][0], out["16"][0]):
            np.testing.assert_array_equal(a, c)
        np.testing.assert_array_equal(out[rows][1], out["16"][1])
