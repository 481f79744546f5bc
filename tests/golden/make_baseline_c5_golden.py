"""Generate tests/golden/baseline_c5sub.npz: the FP64 oracle (the restatement of the
reference's shaders in double) on benchmark configuration 5's flow on the 1024 x 768
sub-grid (tests/baseline_cases.py CONFIG5_SUB: NACA 0024, far field at 40 chords, M 6,
AoA 4, SLAU2 + MUSCL, CFL 0.5), from the uniform freestream in double, dt recomputed every
1000 steps.  At each checkpoint s (steps):

  s/rho_sub, s/p_sub   interior density and pressure on every 8th cell in i and j (float64)
  s/cp                 wall Cp of the first interior row, in double: (p - p_inf) / (M^2 / 2)
  s/forces             Fx, Fy, |F|, Cl, Cd, Cl/Cd of the oracle
  s/residual_l2        the oracle's density-residual norm
  s/state_sha256       checksum of the whole float64 interior state
  grid_sha256          checksum of the float32 grid

The file is rewritten after every checkpoint, so a run stopped early leaves the earlier
checkpoints.  Run from the repository root (about 0.13 s per step on 8 host cores: 4 min
to 2000 steps, 45 min to 20000, 3.5 h to 100000):

    python tests/golden/make_baseline_c5_golden.py [last checkpoint]
"""
from __future__ import annotations

import hashlib
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]

from baseline_cases import CONFIG5_SUB, make_grid_multicolor, primitives  # noqa: E402

PATH = Path(__file__).resolve().parent / "baseline_c5sub.npz"


def make(last=None):
    from oracle.oracle import Oracle, make_params
    cfg = CONFIG5_SUB
    M, N, sub = cfg["M"], cfg["N"], cfg["sub"]
    grid = make_grid_multicolor(cfg)
    out = {"grid_sha256": np.array([hashlib.sha256(grid.tobytes()).hexdigest()])}
    o = Oracle(M, N, "f64")
    o.set_params(make_params(mach=cfg["mach"], aoa_deg=cfg["aoa_deg"], scheme=cfg["scheme"], cfl=cfg["cfl"]))
    o.set_vertices(grid.astype(np.float64))
    o.metrics()
    o.init_state(1)
    done, t0 = 0, time.time()
    for cp_steps in cfg["checkpoints"]:
        if last is not None and cp_steps > last:
            break
        while done < cp_steps:
            n = min(cfg["chunk"], cp_steps - done)
            o.step(n)
            done += n
        q = o.state()[1:N + 1]
        rho, p = primitives(q)
        k = str(cp_steps)
        out[k + "/rho_sub"] = rho[::sub, ::sub].copy()
        out[k + "/p_sub"] = p[::sub, ::sub].copy()
        out[k + "/cp"] = (p[0] - 1.0 / 1.4) / (0.5 * cfg["mach"] ** 2)
        out[k + "/forces"] = np.asarray(o.forces(), np.float64)
        out[k + "/residual_l2"] = np.array([o.residual_l2()])
        out[k + "/state_sha256"] = np.array([hashlib.sha256(np.ascontiguousarray(q, np.float64).tobytes()).hexdigest()])
        np.savez_compressed(PATH, **out)
        print(f"{cp_steps} steps after {time.time() - t0:.0f} s: Cl {out[k + '/forces'][3]:.6f}, "
              f"residual {out[k + '/residual_l2'][0]:.3e}", flush=True)
    o.close()
    return PATH


if __name__ == "__main__":
    p = make(int(sys.argv[1]) if len(sys.argv) > 1 else None)
    print(p, p.stat().st_size, "bytes")
