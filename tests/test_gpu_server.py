"""Continuous-batching server on the GPU.

The key property (results the same alone and in the mix): a request's result (steps,
stop reason, residual norms, forces, wall Cp) is bit-identical when it is served alone
and when it arrives while other requests of other sizes and schemes are on the device,
admitted in a different round, with slots and budget limiting admission.  The plain
one-solve-at-a-time server path computes the same arithmetic with the single-solve
kernels and is checked to 1e-6 relative in Cp."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CHUNK = 50


def req(k, **over):
    import ausm
    specs = [
        dict(M=96, N=64, naca4=12, mach=0.5, aoa_deg=2.0, scheme="SLAU2"),
        dict(M=130, N=72, naca4=2412, mach=1.6, aoa_deg=0.0, scheme="AUSM+-up"),
        dict(M=64, N=40, naca4=4415, mach=0.8, aoa_deg=-2.0, scheme="SLAU"),
        dict(M=160, N=120, naca4=6409, mach=3.0, aoa_deg=6.0, scheme="SLAU2"),
        dict(M=72, N=54, naca4=2318, mach=0.3, aoa_deg=4.0, scheme="SLAU"),
    ]
    sp = dict(specs[k])
    sp.update(over)
    M, N = sp.pop("M"), sp.pop("N")
    sp.setdefault("residual_drop", 1.5)
    sp.setdefault("max_steps", 600)
    return ausm.make_request(M, N, far_radius=10.0, first_spacing=2e-3, grid_iters=150, **sp)


def same(a, b):
    for k in ("state", "stop", "steps", "l2_first", "l2_last", "Fx", "Fy", "Cl", "Cd"):
        assert a[k] == b[k] or (a[k] != a[k] and b[k] != b[k]), (k, a[k], b[k])
    np.testing.assert_array_equal(a["Cp"], b["Cp"])


@pytest.fixture(scope="module")
def alone():
    import ausm
    out = {}
    for k in range(5):
        with ausm.Server(4e9, chunk_steps=CHUNK) as s:
            i = s.submit(req(k))
            s.drain()
            out[k] = s.poll(i)
    return out


def test_alone_results(alone):
    from ausm import _lib
    for k, d in alone.items():
        assert d["state"] == _lib.REQ_DONE, d
        assert d["stop"] in (_lib.STOP_CONVERGED, _lib.STOP_MAX_STEPS)
        assert d["steps"] % CHUNK == 0 and 0 < d["steps"] <= 600
        assert np.all(np.isfinite(d["Cp"])) and np.isfinite(d["Cl"])
        if d["stop"] == _lib.STOP_CONVERGED:
            assert d["l2_last"] <= d["l2_first"] * 10 ** -1.5
        assert d["latency_ms"] >= d["run_ms"] > 0


def test_same_alone_and_in_the_mix(alone):
    """Arrivals in three waves between rounds, two slots, a budget that holds only
    some of the requests at once."""
    import ausm
    budget = sum(ausm.request_bytes(req(k)) for k in (1, 3)) + 1.0
    with ausm.Server(budget, max_active=2, chunk_steps=CHUNK) as s:
        ids = {3: s.submit(req(3)), 1: s.submit(req(1))}
        s.pump()
        ids[0] = s.submit(req(0))
        s.pump()
        s.pump()
        ids[4] = s.submit(req(4))
        ids[2] = s.submit(req(2))
        peak_active = 0
        while True:
            left = s.pump()
            peak_active = max(peak_active, s.stats()["active"])
            if left == 0:
                break
        st = s.stats()
        assert st["finished"] == 5 and st["failed"] == 0 and st["peak_bytes"] <= budget
        assert peak_active <= 2
        for k, i in ids.items():
            same(s.poll(i), alone[k])


def test_worker_thread_same_results(alone):
    import ausm
    with ausm.Server(16e9, max_active=8, chunk_steps=CHUNK) as s:
        s.start()
        ids = {k: s.submit(req(k)) for k in (4, 0, 2, 1, 3)}
        s.drain(timeout_s=300)
        for k, i in ids.items():
            same(s.poll(i), alone[k])
        s.stop()


def test_divergent_request_is_isolated(alone):
    """A request that blows up (CFL 40) ends DIVERGED; the others are unaffected."""
    import ausm
    from ausm import _lib
    with ausm.Server(16e9, chunk_steps=CHUNK) as s:
        bad = s.submit(req(3, cfl=40.0))
        ids = {k: s.submit(req(k)) for k in (0, 1)}
        s.drain()
        d = s.poll(bad)
        assert d["state"] == _lib.ERR_DIVERGED and d["stop"] == _lib.STOP_DIVERGED
        for k, i in ids.items():
            same(s.poll(i), alone[k])
        assert s.stats()["failed"] == 1


def test_plain_path_matches(alone):
    import ausm
    from ausm import _lib
    with ausm.Server(16e9, chunk_steps=CHUNK, plain=True) as s:
        ids = {k: s.submit(req(k)) for k in range(5)}
        s.drain()
        for k, i in ids.items():
            d, a = s.poll(i), alone[k]
            assert d["state"] == _lib.REQ_DONE and d["steps"] == a["steps"] and d["stop"] == a["stop"]
            scale = np.abs(a["Cp"]).max()
            assert np.abs(d["Cp"] - a["Cp"]).max() <= 1e-6 * scale


def test_plain_worker_drain_waits_for_admissions():
    """One slot and a worker thread: every request is admitted while nothing else is
    active, so drain must not mistake a request in admission for an idle server."""
    import ausm
    from ausm import _lib
    with ausm.Server(16e9, chunk_steps=CHUNK, plain=True) as s:
        s.start()
        ids = [s.submit(req(k % 5, max_steps=100)) for k in range(8)]
        s.drain(timeout_s=300)
        for i in ids:
            d = s.poll(i)
            assert d["state"] == _lib.REQ_DONE and d["steps"] == 100, d
            assert d["latency_ms"] >= d["run_ms"] > 0
        s.stop()


def test_body_points_request_matches_naca_request():
    """A request with the body given as points (a .dat airfoil sampled on the host) is
    the same solve as the NACA request those points come from."""
    import ausm
    import numpy as np
    from ausm.solver import lib
    import ctypes as C
    M = 96
    xy = np.zeros((M, 2))
    # the NACA 0012 points the server builds for chord 1 centred at 0 (half chord 0.5)
    lib().ausm_naca4_points(M, 12, 0.5, 0.0, 1, xy.ctypes.data_as(C.POINTER(C.c_double)))
    with ausm.Server(4e9, chunk_steps=CHUNK) as s:
        a = s.submit(req(0))
        b = s.submit(req(0, body_xy=xy))
        s.drain()
        ra, rb = s.poll(a), s.poll(b)
    assert ra["state"] == 0 and rb["state"] == 0
    np.testing.assert_array_equal(ra["Cp"], rb["Cp"])
    assert ra["Cl_c"] == ra["Cl"]  # chord 1


def test_sharded_server_same_results(alone):
    """Two servers behind one ShardedServer (both on device 0 here: the placement and
    routing are what is tested; one server per GPU in production): every request lands
    on one of them and its result is the same as alone."""
    import ausm
    with ausm.ShardedServer([0, 0], 4e9, chunk_steps=CHUNK) as sh:
        sh.start()
        ids = [sh.submit(req(k)) for k in range(5)]
        sh.drain()
        res = [sh.poll(i) for i in ids]
    assert {i[0] for i in ids} == {0, 1}
    for k, d in enumerate(res):
        same(d, alone[k])


def test_failed_round_ends_only_its_members(alone):
    """A round whose batch step fails (here a bounded tile wait made to give up at once
    through the test hook, no fault) ends the requests of that round with its status;
    a request still queued behind them is served afterwards with its usual result."""
    import ausm
    from ausm import _lib
    with ausm.Server(4e9, max_active=1, chunk_steps=CHUNK) as s:
        a, b = s.submit(req(0)), s.submit(req(1))
        s.pump()  # admits a (one slot) and runs its first round
        ausm.set_wait_polls(0)
        try:
            with pytest.raises(ausm.AusmError) as e:
                s.pump()
            assert e.value.code == _lib.ERR_TIMEOUT
        finally:
            ausm.set_wait_polls(65536)
        assert s.poll(a)["state"] == _lib.ERR_TIMEOUT
        assert s.poll(b)["state"] == _lib.REQ_QUEUED
        s.drain()
        same(s.poll(b), alone[1])
