"""Bounded device-side waits: a tile whose wait gives up is reported as AUSM_ERR_TIMEOUT
on every path through the C ABI, and the call after the report succeeds.

The waits are made to run out with the library's test hook ausm_debug_set_wait_polls(0):
the first wait of every TMA box then gives up at once, the tile sets the error flag and
writes nothing, and its copies still land (a second wait with the full bound) before the
CTA exits.  Nothing faults and no address is invalid; the hook is reset to the default
65536 polls in every test's teardown.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M, N = 64, 32
TIMEOUT = -7
KW = dict(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=0.8, aoa_deg=2.0, K_p=0.0, K_u=0.75, cfl=0.5,
          maxdt=math.inf, muscl=1, scheme="SLAU2", ramp=0.0)


@pytest.fixture
def polls():
    import ausm
    ausm.set_device(0)
    yield ausm.set_wait_polls
    ausm.set_wait_polls(65536)


def solver():
    import ausm
    s = ausm.Solver(M, N)
    s.set_body_naca4(12, 0.5, 0.0)
    s.set_outer_circle(10.0)
    s.generate_grid(100, "multicolor")
    s.set_params(**KW)
    s.prepare_state("freestream")
    s.autotune()  # tune before the hook, so the tile height is not chosen from failing launches
    return s


def expect_timeout(fn):
    import ausm
    with pytest.raises(ausm.AusmError) as e:
        fn()
    assert e.value.code == TIMEOUT, str(e.value)


def test_step_reports_timeout_then_recovers(polls):
    ref = solver()
    ref.step(3)
    q_ref = ref.state()
    ref.close()
    s = solver()
    polls(0)
    expect_timeout(lambda: s.step(1))
    polls(65536)
    s.prepare_state("freestream")
    s.step(3)
    assert np.array_equal(s.state(), q_ref)
    s.close()


@pytest.mark.parametrize("reader", ["synchronize", "state", "forces", "residual_l2", "max_wave_speed"])
def test_async_step_reports_at_next_wait(polls, reader):
    s = solver()
    polls(0)
    s.step(2, wait=False)  # does not wait: nothing to report yet
    polls(65536)
    fn = {"synchronize": s.synchronize, "state": s.state, "forces": lambda: s.forces(with_cp=True),
          "residual_l2": s.residual_l2, "max_wave_speed": s.max_wave_speed}[reader]
    expect_timeout(fn)
    s.prepare_state("freestream")  # the timed-out tiles left the state stale: reset it
    fn()  # the flag was read and cleared: the same call now succeeds
    assert math.isfinite(s.step(1))
    s.close()


def test_time_steps_reports_timeout(polls):
    s = solver()
    polls(0)
    expect_timeout(lambda: s.time_steps(1, 3))
    polls(65536)
    s.prepare_state("freestream")
    assert s.time_steps(1, 3) > 0.0
    s.close()


def test_batch_reports_timeout(polls):
    import ausm
    sols = [solver() for _ in range(2)]
    with ausm.Batch() as b:
        for s in sols:
            b.add(s)
        b.step(1)  # tunes the batch's tile height with the full bound
        polls(0)
        expect_timeout(lambda: b.step(1))
        b.step(1, wait=False)
        expect_timeout(b.synchronize)
        expect_timeout(lambda: b.time_steps(1, 2))
        polls(65536)
        for s in sols:
            s.prepare_state("freestream")
        out = b.step(2)
        assert np.all(np.isfinite(out))
        for s in list(b.members):
            b.remove(s)
    for s in sols:
        s.close()
