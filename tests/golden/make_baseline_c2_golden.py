"""Generate tests/golden/baseline_c2.npz: the float32 oracle (the restatement, which
reproduces the reference's own shaders bit for bit on every golden run and is about three
times faster on the host) on benchmark configuration 2 as written (tests/baseline_cases.py
CONFIG2: NACA 2412, 512 x 384; M 0.8 SLAU2, M 2 AUSM+-up, M 8 SLAU; 20000 RK3 steps in
frames of 100 from a uniform freestream start), and the same with the oracle compiled with
fused multiply-add contraction (the float32 spread of the reference's arithmetic).  Per run:

  k/cp, k/cp_fma           wall Cp after 20000 steps (M values)
  k/rho_sub, k/rho_sub_fma interior density on every 4th cell in i and j (N/4 x M/4)
  k/forces                 Fx, Fy, |F|, Cl, Cd, Cl/Cd of the oracle
  grid_sha256              checksum of the float32 grid

Run from the repository root (about an hour on 8 cores):

    python tests/golden/make_baseline_c2_golden.py
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]

from baseline_cases import CONFIG2, make_grid, wall_cp  # noqa: E402

STEPS, FRAME, SUB = 20000, 100, 4


def run(grid, run_cfg, lib=None):
    import oracle.oracle as oo
    from oracle.oracle import Oracle, make_params
    if lib is not None:
        oo.ORACLE_SO, oo._olib = lib, None
    M, N = CONFIG2["M"], CONFIG2["N"]
    o = Oracle(M, N, "f32")
    o.set_params(make_params(mach=run_cfg["mach"], aoa_deg=run_cfg["aoa_deg"], scheme=run_cfg["scheme"],
                             cfl=CONFIG2["cfl"]))
    o.set_vertices(grid)
    o.metrics()
    o.init_state(1)
    for _ in range(STEPS // FRAME):
        o.step(FRAME)
    q = o.state()
    out = {"cp": wall_cp(q[1], run_cfg["mach"]), "rho_sub": q[1:N + 1:SUB, ::SUB, 0].copy(), "forces": o.forces()}
    o.close()
    return out


def make():
    from oracle.build import build_oracle
    grid = make_grid(CONFIG2)
    out = {"grid_sha256": np.array([hashlib.sha256(grid.tobytes()).hexdigest()])}
    plain_lib, fma_lib = build_oracle(), build_oracle(contract=True)
    for k, rc in enumerate(CONFIG2["runs"]):
        a = run(grid, rc, plain_lib)
        b = run(grid, rc, fma_lib)
        out[f"{k}/cp"], out[f"{k}/rho_sub"], out[f"{k}/forces"] = a["cp"], a["rho_sub"], a["forces"]
        out[f"{k}/cp_fma"], out[f"{k}/rho_sub_fma"] = b["cp"], b["rho_sub"]
        print(k, rc, "spread Cp", np.abs(a["cp"] - b["cp"]).max() / np.abs(a["cp"]).max(), flush=True)
    path = Path(__file__).resolve().parent / "baseline_c2.npz"
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    p = make()
    print(p, p.stat().st_size, "bytes")
