"""Serving host logic that needs no GPU: request validation and rejection, budget
rejection, the per-request byte estimate, result polling of queued requests and the
counters.  The server makes no CUDA call until its first round."""
import math

import numpy as np
import pytest


@pytest.fixture
def ausm_mod():
    import ausm
    return ausm


def test_request_bytes(ausm_mod):
    r = ausm_mod.make_request(256, 128)
    M, N = 256, 128
    assert ausm_mod.request_bytes(r) == 40 * M * (N + 1) + 16 * M * N + 48 * M * N + 8 * M + 65536


BAD = [
    (dict(M=3), "grid"),
    (dict(N=1), "grid"),
    (dict(mach=float("nan")), "non-finite"),
    (dict(mach=0.0), "mach > 0"),
    (dict(cfl=-1.0), "cfl > 0"),
    (dict(gamma=1.0), "gamma > 1"),
    (dict(scheme=7), "scheme"),
    (dict(naca4=0), "NACA"),
    (dict(naca4=2400), "NACA"),
    (dict(far_radius=0.5), "far_radius"),
    (dict(first_spacing=-1.0), "first_spacing"),
    (dict(max_steps=0), "max_steps"),
    (dict(residual_drop=float("inf")), "residual_drop"),
    (dict(ramp=10.0), "ramp"),
]


@pytest.mark.parametrize("kw,word", BAD)
def test_submit_rejects_poisoned_requests(ausm_mod, kw, word):
    from ausm import _lib
    base = dict(M=64, N=32)
    base.update(kw)
    M, N = base.pop("M"), base.pop("N")
    r = ausm_mod.make_request(M, N, **base)
    with ausm_mod.Server(1e9) as s:
        with pytest.raises(ausm_mod.AusmError) as e:
            s.submit(r)
        assert e.value.code == _lib.ERR_INVALID
        assert word in str(e.value)
        st = s.stats()
        assert st["rejected"] == 1 and st["submitted"] == 0 and st["pending"] == 0


def test_submit_rejects_non_finite_body(ausm_mod):
    from ausm import _lib
    xy = np.zeros((64, 2))
    xy[5, 1] = np.nan
    r = ausm_mod.make_request(64, 32, body_xy=xy)
    with ausm_mod.Server(1e9) as s:
        with pytest.raises(ausm_mod.AusmError) as e:
            s.submit(r)
        assert e.value.code == _lib.ERR_INVALID


def test_budget_rejection_and_queueing(ausm_mod):
    from ausm import _lib
    small = ausm_mod.make_request(64, 32)
    big = ausm_mod.make_request(1024, 768)
    budget = ausm_mod.request_bytes(small) * 3
    with ausm_mod.Server(budget) as s:
        with pytest.raises(ausm_mod.AusmError) as e:
            s.submit(big)
        assert e.value.code == _lib.ERR_BUDGET
        ids = [s.submit(small) for _ in range(5)]
        assert ids == sorted(ids) and len(set(ids)) == 5
        for i in ids:
            d = s.poll(i)
            assert d["state"] == _lib.REQ_QUEUED
            assert math.isnan(d["latency_ms"]) and math.isnan(d["Cl"])
        st = s.stats()
        assert st["submitted"] == 5 and st["rejected"] == 1 and st["pending"] == 5 and st["active"] == 0
        with pytest.raises(ausm_mod.AusmError) as e:
            s.poll(12345)
        assert e.value.code == _lib.ERR_NOT_FOUND


def test_server_create_validation(ausm_mod):
    from ausm import _lib
    for args in ((0.0, 4, 10), (1e9, 0, 10), (1e9, 4, 0)):
        with pytest.raises(ausm_mod.AusmError) as e:
            ausm_mod.Server(*args)
        assert e.value.code == _lib.ERR_INVALID
