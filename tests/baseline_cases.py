"""Inputs of the benchmark configurations that the parity tests run (the O-grids, flows
and step counts), shared by the tests and by tests/golden/make_baseline_golden.py.

Configuration 1 ("plain method, small"): NACA 0012 (closed trailing edge), O-grid of
256 x 128 cells, circular far field at 20 chords, geometric radial stretching with a
first cell of 1e-3 chord, 2000 elliptic (TTM, P = Q = 0) sweeps; M 0.5, AoA 0, gamma
1.4, uniform freestream start, SLAU2 + MUSCL, TVD-RK3, CFL 0.5, FP32, 2000 steps.
Configuration 2 ("README scale"): NACA 2412 O-grid of 512 x 384 cells, far field at
20 chords, the same grid generator; (M 0.8, AoA 2, SLAU2), (M 2, AoA 0, AUSM+-up),
(M 8, AoA 0, SLAU) from a uniform freestream start at CFL 0.5.

The grids come from the oracle (test infrastructure): the stretched initial guess of
oracle/geometry_ref.py (the library's geometric radial stretching restated in double:
per column a geometric progression from the body to the far-field point whose first
step is first_spacing), rounded to float32, then the reference's own Jacobi TTM sweeps
in float32 (the oracle reproduces the reference's grid shader bit for bit).  Chord 1
centred at the origin.
"""
import math

import numpy as np

CONFIG1 = dict(M=256, N=128, naca=12, far=20.0, first=1e-3, iters=2000, mach=0.5, aoa_deg=0.0, scheme="SLAU2",
               cfl=0.5, steps=2000, frame=100, converged_frame=500, max_steps=50000, drop=4.0)
CONFIG2 = dict(M=512, N=384, naca=2412, far=20.0, first=1e-3, iters=2000, cfl=0.5,
               runs=[dict(mach=0.8, aoa_deg=2.0, scheme="SLAU2"), dict(mach=2.0, aoa_deg=0.0, scheme="AUSM+-up"),
                     dict(mach=8.0, aoa_deg=0.0, scheme="SLAU")])


def make_grid(cfg):
    """float32 (N+1, M, 2) vertices of a configuration's O-grid."""
    from oracle.geometry_ref import circular_outer, naca4_boundary, stretched_guess
    from oracle.oracle import Oracle
    M, N = cfg["M"], cfg["N"]
    body = naca4_boundary(M, cfg["naca"], 0.5, 0.0)
    outer = circular_outer(M, cfg["far"])
    o = Oracle(M, N, "f32")
    o.set_vertices(stretched_guess(body, outer, N, cfg["first"]).astype(np.float32))
    o.grid_jacobi(cfg["iters"])
    v = o.vertices()
    o.close()
    return v


def flow_kwargs(run, cfl):
    """Solver parameters (library names) of a run."""
    return dict(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=run["mach"], aoa_deg=run["aoa_deg"], K_p=0.0,
                K_u=0.75, cfl=cfl, maxdt=math.inf, muscl=1, scheme=run["scheme"], ramp=0.0)


def wall_cp(q_row1, mach, gamma=1.4):
    """Wall Cp of a state's first interior row as the library computes it: float32
    pressure of the cell (graphs.js:26-29), (p - p_inf) / q_inf in double."""
    w = np.asarray(q_row1, np.float32)
    g = np.float32(gamma)
    rho, u, v = w[:, 0], w[:, 1] / w[:, 0], w[:, 2] / w[:, 0]
    p = ((w[:, 3] - np.float32(0.5) * rho * (u * u + v * v)) * (g - np.float32(1.0))).astype(np.float64)
    speed = mach * math.sqrt(gamma * (1.0 / gamma) / 1.0)
    return (p - 1.0 / gamma) / (0.5 * speed * speed)


def density_l2_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


# Configuration 5 ("large precision study": NACA 0024, far field at 40 chords, M 6, AoA 4,
# SLAU2 + MUSCL, CFL 0.5) on the 1024 x 768 sub-grid where the FP64 oracle runs on the
# host cores: the grid of the 4096 x 3072 workload's generator at that size (geometric
# stretch with a 1e-3 chord first cell, 200 multicolour TTM sweeps in double, rounded to
# float32), dt recomputed every 1000 steps as in the full-size precision study.
CONFIG5_SUB = dict(M=1024, N=768, naca=24, far=40.0, first=1e-3, iters=200, mach=6.0, aoa_deg=4.0, scheme="SLAU2",
                   cfl=0.5, chunk=1000, checkpoints=(2000, 20000, 100000), sub=8)


def make_grid_multicolor(cfg):
    """float32 (N+1, M, 2) vertices: the stretched guess, then cfg['iters'] multicolour
    sweeps of the oracle's FP64 restatement of the library's generator."""
    from oracle.geometry_ref import circular_outer, naca4_boundary, stretched_guess
    from oracle.oracle import Oracle
    M, N = cfg["M"], cfg["N"]
    body = naca4_boundary(M, cfg["naca"], 0.5, 0.0)
    outer = circular_outer(M, cfg["far"])
    o = Oracle(M, N, "f64")
    o.set_vertices(stretched_guess(body, outer, N, cfg["first"]))
    o.grid_multicolor(cfg["iters"], 0.0)
    v = o.vertices().astype(np.float32)
    o.close()
    return v


def primitives(q, gamma=1.4):
    """density and pressure (float64) of conserved states (..., 4)"""
    q = np.asarray(q, np.float64)
    rho = q[..., 0]
    p = (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / rho) * (gamma - 1.0)
    return rho, p
