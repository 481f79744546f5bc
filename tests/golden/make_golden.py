"""Generate the golden fixtures from the reference's own compute shaders.

Runs the reference's WGSL compute shaders compiled for the CPU (oracle/wgsl_ref/,
built by oracle/build.py from the reference tree) in main.js's dispatch order and
stores inputs and outputs as tests/golden/ref_cases.npz.  Run it where the reference
tree is present:

    python tests/golden/make_golden.py

Cases (float32 throughout, as the reference's textures):
  grid_*   prepareGrid: linear initial guess + Jacobi TTM sweeps + finalize
           (both ping-pong iterates, area, face lengths)
  run_*    prepareState (rest or uniform freestream) then frames of step(n) on an
           injected grid: state2, dt of each frame, max wave speed, forces
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.geometry_ref import naca4_boundary, rectangular_outer  # noqa: E402
from oracle.oracle import RefWGSL, make_params  # noqa: E402

GRIDS = {
    # name: (M, N, naca, size, xoff, outer_ratio, iters)
    "grid_64x32": (64, 32, 12, 0.3, -0.7, 1.5, 400),
    "grid_33x17": (33, 17, 2412, 0.3, -0.7, 1.5, 150),
    "grid_48x20": (48, 20, 4412, 0.2, -0.7, 1.5, 1000),
}

# name: (grid, params kwargs, init mode, frames[list of steps per frame])
RUNS = {
    "run_slau2_m05_a2_fs": ("grid_64x32", dict(mach=0.5, aoa_deg=2.0, scheme="SLAU2", cfl=0.5), 1, [1, 4]),
    "run_slau_m2_a0_fs": ("grid_64x32", dict(mach=2.0, aoa_deg=0.0, scheme="SLAU", cfl=0.5), 1, [1, 4]),
    "run_ausmup_m8_a0_fs": ("grid_64x32", dict(mach=8.0, aoa_deg=0.0, scheme="AUSM+-up", cfl=0.5), 1, [1, 4]),
    "run_ausmup_m03_kp_fs": ("grid_64x32", dict(mach=0.3, aoa_deg=-3.0, scheme="AUSM+-up", K_p=0.25, cfl=0.8), 1, [1, 3]),
    "run_slau2_m05_rest": ("grid_64x32", dict(mach=0.5, aoa_deg=0.0, scheme="SLAU2", cfl=0.5), 0, [1, 4]),
    "run_slau2_nomuscl_m15": ("grid_64x32", dict(mach=1.5, aoa_deg=5.0, scheme="SLAU2", muscl=0, cfl=0.5), 1, [1, 4]),
    "run_defaults_m38": ("grid_64x32", dict(mach=3.8, aoa_deg=0.0, scheme="SLAU2", cfl=1.5, maxdt=1e-4), 1, [2, 2]),
    "run_slau2_m08_a4_odd": ("grid_33x17", dict(mach=0.8, aoa_deg=4.0, scheme="SLAU2", cfl=0.5), 1, [1, 9]),
    "run_slau_m6_odd": ("grid_33x17", dict(mach=6.0, aoa_deg=4.0, scheme="SLAU", cfl=0.5), 1, [2, 6]),
    "run_ausmup_m2_a3_4412": ("grid_48x20", dict(mach=2.0, aoa_deg=3.0, scheme="AUSM+-up", cfl=0.5), 1, [1, 6]),
    "run_slau2_long": ("grid_48x20", dict(mach=0.5, aoa_deg=2.0, scheme="SLAU2", cfl=0.5), 1, [50, 50, 50, 50]),
}


def make():
    out = {}
    grids = {}
    for name, (M, N, naca, size, xoff, ratio, iters) in GRIDS.items():
        body = naca4_boundary(M, naca, size, xoff).astype(np.float32)
        outer = rectangular_outer(M, ratio).astype(np.float32)
        r = RefWGSL(M, N)
        r.set_uniforms(make_params())
        r.set_boundaries(body, outer)
        r.prepare_grid(iters)
        gp1 = r.texture("gridPoints1")
        grids[name] = gp1
        out[f"{name}/meta"] = np.array([M, N, naca, iters], dtype=np.int64)
        out[f"{name}/body"] = body
        out[f"{name}/outer"] = outer
        out[f"{name}/gridPoints0"] = r.texture("gridPoints0")
        out[f"{name}/gridPoints1"] = gp1
        out[f"{name}/area"] = r.texture("gridArea")
        out[f"{name}/faceLengths"] = r.texture("faceLengths")
        r.close()
    for name, (gname, kw, mode, frames) in RUNS.items():
        M, N = GRIDS[gname][0], GRIDS[gname][1]
        p = make_params(**kw)
        r = RefWGSL(M, N)
        r.set_uniforms(p)
        r.set_grid(grids[gname])
        r.prepare_state(mode)
        out[f"{name}/grid"] = np.array([gname])
        out[f"{name}/params"] = np.array([p.gamma, p.in_rho, p.in_pressure, p.inflow[0], p.inflow[1],
                                          *p.in_state, p.K_p, p.K_u, p.cfl, p.maxdt, p.muscl, p.scheme],
                                         dtype=np.float64)
        out[f"{name}/kw"] = np.array([json.dumps(kw)])
        out[f"{name}/mode"] = np.array([mode])
        out[f"{name}/frames"] = np.array(frames)
        out[f"{name}/maxwave0"] = np.array([r.max_wave()], dtype=np.float32)
        for k, n in enumerate(frames):
            dt = r.frame(n)
            out[f"{name}/dt{k}"] = np.array([dt], dtype=np.float32)
            out[f"{name}/state{k}"] = r.texture("state2")
            out[f"{name}/maxwave{k + 1}"] = np.array([r.max_wave()], dtype=np.float32)
        out[f"{name}/forces"] = r.forces().astype(np.float32)
        r.eval_residual()
        out[f"{name}/residual"] = r.texture("residual")
        r.close()
    path = Path(__file__).resolve().parent / "ref_cases.npz"
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    p = make()
    print(p, p.stat().st_size, "bytes")
