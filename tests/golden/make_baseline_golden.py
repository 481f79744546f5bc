"""Generate tests/golden/baseline_c1.npz: the reference's own compute shaders (compiled
for the CPU by oracle/build.py from the reference tree) on benchmark configuration 1
(tests/baseline_cases.py CONFIG1), for the parity gates that the oracle cannot run
within a test's time:

  rho_2000, cp_2000   interior density and wall Cp after the configuration's 2000 steps
                      (frames of 100 steps, dt held per frame as step(n) does)
  rho_end, cp_end     the same at the end of the converged run: then frames of 500 steps
                      until the density-residual L2 has dropped `drop` decades below its
                      value at the start, or max_steps steps (the served configuration's
                      stopping rule)
  steps_end, l2       step count of the end, residual norms after each frame
  rho_end_fma,        the same end state from the reference's shaders compiled with fused
  cp_end_fma          multiply-add contraction (oracle/build.py build_ref(contract=True)): a
                      second float32 rounding of the reference's own arithmetic, whose
                      distance from rho_end / cp_end is the float32 reproducibility floor of
                      this slowly converging subsonic run
  grid_sha256         checksum of the float32 grid (the tests rebuild the grid and check it)

Run where the reference tree is present:

    python tests/golden/make_baseline_golden.py
"""
from __future__ import annotations

import hashlib
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]

from baseline_cases import CONFIG1, make_grid, wall_cp  # noqa: E402
from oracle.oracle import RefWGSL, make_params  # noqa: E402


def residual_l2(r, N):
    r.eval_residual()
    res = r.texture("residual")[..., 0].astype(np.float64)
    return float(np.sqrt(np.mean(res ** 2)))


def run(grid, lib=None):
    """The configuration's run on the reference build at `lib` (default: oracle/_ref)."""
    import oracle.oracle as oo
    c = CONFIG1
    M, N = c["M"], c["N"]
    if lib is not None:
        oo.REF_SO, oo._rlib = lib, None
    r = RefWGSL(M, N)
    r.set_uniforms(make_params(mach=c["mach"], aoa_deg=c["aoa_deg"], scheme=c["scheme"], cfl=c["cfl"]))
    r.set_grid(grid)
    r.prepare_state(1)
    l2 = [residual_l2(r, N)]
    out = {}
    steps = 0
    t0 = time.time()
    while steps < c["steps"]:
        r.frame(c["frame"])
        steps += c["frame"]
        l2.append(residual_l2(r, N))
    q = r.texture("state2")
    out["rho_2000"] = q[1:N + 1, :, 0].copy()
    out["cp_2000"] = wall_cp(q[1], c["mach"])
    target = l2[0] * 10.0 ** (-c["drop"])
    while steps < c["max_steps"] and l2[-1] > target:
        r.frame(c["converged_frame"])
        steps += c["converged_frame"]
        l2.append(residual_l2(r, N))
        if steps % 5000 == 0:
            print(f"{steps} steps, residual {l2[-1] / l2[0]:.3e} of the start, {time.time() - t0:.0f} s", flush=True)
    q = r.texture("state2")
    out["rho_end"] = q[1:N + 1, :, 0].copy()
    out["cp_end"] = wall_cp(q[1], c["mach"])
    out["steps_end"] = np.array([steps])
    out["l2"] = np.array(l2)
    r.close()
    return out


def make():
    from oracle.build import build_ref
    grid = make_grid(CONFIG1)
    out = run(grid)
    fma = run(grid, build_ref(contract=True))
    out["rho_end_fma"], out["cp_end_fma"] = fma["rho_end"], fma["cp_end"]
    out["grid_sha256"] = np.array([hashlib.sha256(grid.tobytes()).hexdigest()])
    path = Path(__file__).resolve().parent / "baseline_c1.npz"
    np.savez_compressed(path, **out)
    return path


if __name__ == "__main__":
    p = make()
    print(p, p.stat().st_size, "bytes")
