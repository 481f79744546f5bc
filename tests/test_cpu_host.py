"""Host-side checks that need no GPU: the C ABI library loads and exports every entry
point of include/ausm.h, host geometry generators, argument validation, the .dat
front end, and the multi-rank timing reduction of bench.py."""
import ctypes as C
import math
import os
import re
from pathlib import Path

import numpy as np
import pytest

from ausm import _lib, geometry
from oracle.geometry_ref import circular_outer, naca4_boundary, rectangular_outer

from oracle.build import REF_SRC as REF  # the reference tree, where the oracle's build recipe finds it


def test_library_exports_every_header_function():
    L = _lib.lib()
    names = _lib.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_default_params_are_the_reference_defaults():
    from ausm import default_params
    p = default_params()
    # util.js:78-96, main.js:877-885
    assert (p.gamma, p.in_rho, p.cfl, p.maxdt, p.K_p, p.K_u, p.muscl, p.scheme) == (1.4, 1.0, 1.5, 1e-4, 0.0, 0.75, 1, 0)
    assert p.in_pressure == 1.0 / 1.4 and p.mach == 3.8


@pytest.mark.parametrize("digits", [12, 2412, 4412, 24, 6409])
@pytest.mark.parametrize("M", [64, 33, 510])
def test_naca4_matches_reference_formula(digits, M):
    a = geometry.naca4(M, digits, 0.3, -0.7)
    b = naca4_boundary(M, digits, 0.3, -0.7)
    assert np.abs(a - b).max() < 1e-14
    assert np.array_equal(a.astype(np.float32), b.astype(np.float32)) or np.abs(a - b).max() < 1e-15


def test_naca4_closed_trailing_edge():
    """-0.1036 closes the trailing edge: first (TE) point at y = 0, x = chord end."""
    a = geometry.naca4(256, 12, 0.5, 0.0, closed_te=True)
    assert abs(a[0, 1]) < 1e-12 and abs(a[0, 0] - 0.5) < 1e-12
    b = geometry.naca4(256, 12, 0.5, 0.0, closed_te=False)
    assert abs(b[1, 1] - a[1, 1]) > 0  # open-TE coefficient differs


def test_outer_boundaries():
    assert np.array_equal(geometry.outer(96, "rect", 1.5), rectangular_outer(96, 1.5))
    assert np.abs(geometry.outer(96, "circle", 20.0) - circular_outer(96, 20.0)).max() < 1e-12


def test_host_argument_validation():
    L = _lib.lib()
    xy = np.zeros((8, 2))
    p = xy.ctypes.data_as(C.POINTER(C.c_double))
    assert L.ausm_naca4_points(2, 12, 0.3, 0.0, 1, p) == _lib.ERR_INVALID
    assert L.ausm_naca4_points(8, 0, 0.3, 0.0, 1, p) == _lib.ERR_INVALID
    assert L.ausm_naca4_points(8, 2400, 0.3, 0.0, 1, p) == _lib.ERR_INVALID  # zero thickness
    assert L.ausm_naca4_points(8, 2012, 0.3, 0.0, 1, p) == _lib.ERR_INVALID  # camber without position
    assert b"thickness" in L.ausm_last_error(None) or b"camber" in L.ausm_last_error(None)
    assert L.ausm_outer_points(8, 7, 1.0, 0, 0, p) == _lib.ERR_INVALID
    assert L.ausm_outer_points(8, 0, -1.0, 0, 0, p) == _lib.ERR_INVALID
    assert L.ausm_default_params(None) == _lib.ERR_INVALID
    with pytest.raises(_lib.AusmError):
        geometry.naca4(8, 0)
    # grid sizes are checked before any device call
    h = C.c_void_p()
    assert L.ausm_create(3, 8, C.byref(h)) == _lib.ERR_INVALID and not h.value
    assert L.ausm_create(8, 1, C.byref(h)) == _lib.ERR_INVALID
    assert L.ausm_create(100000, 30000, C.byref(h)) == _lib.ERR_INVALID  # M (N+3) above 2e9
    assert b"too large" in L.ausm_last_error(None)


def _airfoil_texts():
    out = {}
    d = REF / "dat" / "supercritical"
    if d.exists():
        for f in sorted(d.glob("*.dat")):
            out[f.name] = f.read_text()
    js = REF / "src" / "airfoilData.js"
    if js.exists():
        for name, body in re.findall(r"const\s+(\w+)\s*=\s*`([^`]*)`", js.read_text()):
            out[name] = body
    return out


AIRFOILS = _airfoil_texts()


@pytest.mark.skipif(not AIRFOILS, reason="reference airfoil inputs not present")
@pytest.mark.parametrize("name", sorted(AIRFOILS))
def test_dat_loader_all_reference_airfoils(name):
    text = AIRFOILS[name]
    upper, lower, fmt = geometry.parse_dat(text)
    assert fmt in ("selig", "lednicer")
    # upper runs TE -> LE, lower LE -> TE (airfoilDatParser.js:14-16)
    assert upper[0][0] > 0.9 and upper[-1][0] < 0.1 and lower[0][0] < 0.1 and lower[-1][0] > 0.9
    pts = geometry.sample_airfoil(text, 510, 0.3, -0.7)
    assert pts.shape == (510, 2) and np.all(np.isfinite(pts))
    # chord maps to [-0.7 - 0.3, -0.7 + 0.3] (scale 2*0.3 on [0,1] centred at 0.5)
    assert pts[:, 0].min() > -1.0 - 1e-3 and pts[:, 0].max() < -0.4 + 1e-3
    # counter-clockwise contour: positive signed area
    x, y = pts[:, 0], pts[:, 1]
    area = 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)
    assert area > 0
    # the spline passes through its control points: sampling the contour parameter at a
    # control point returns it
    sample = geometry.parse_airfoil(text)
    p0 = sample(0.0)
    assert abs(p0[0] - upper[0][0]) < 1e-12 and abs(p0[1] - upper[0][1]) < 1e-12


def test_dat_loader_formats_and_errors():
    selig = "NAME\n1.0 0.0\n0.5 0.05\n0.0 0.0\n0.5 -0.05\n1.0 0.0\n"
    u, l, fmt = geometry.parse_dat(selig)
    assert fmt == "selig" and u[-1] == (0.0, 0.0) and l[0] == (0.0, 0.0)
    led = "NAME\n 3.  3.\n\n0.0 0.0\n0.5 0.05\n1.0 0.0\n\n0.0 0.0\n0.5 -0.05\n1.0 0.0\n"
    u, l, fmt = geometry.parse_dat(led)
    assert fmt == "lednicer" and u[0] == (1.0, 0.0) and l[-1] == (1.0, 0.0)
    with pytest.raises(ValueError):
        geometry.parse_dat("no numbers here\n")
    with pytest.raises(ValueError):
        geometry.parse_dat("1 0\n0 0\n")
    assert geometry._parse_float(".0075") == 0.0075 and math.isnan(geometry._parse_float("SC(2)"))
    assert geometry._parse_float("103.") == 103.0


def _max_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    q.put((rank, bench.max_over_ranks(1.0 + rank, dist)))
    dist.destroy_process_group()


def test_bench_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_max_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, 2.0), (1, 2.0)]
