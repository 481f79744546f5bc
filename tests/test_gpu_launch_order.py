"""Programmatic dependent launch changes when a stage kernel's CTAs start, never what
they compute: a stage kernel issues its face-record loads before its grid-dependency
wait and reads the previous stage's state only after it.  The same solves, stepped in
two processes with the launch attribute on (the default) and off (AUSM_PDL=0), give
bit-identical states: one grid alone (several tile heights) and a mixed batch."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

CHILD = r'''
import math, sys
import numpy as np
sys.path.insert(0, {root!r}); sys.path.insert(0, {pkg!r})
from ausm import Solver, Batch

def annulus(M, N, r0=0.5, r1=4.0):
    th = 2 * math.pi * np.arange(M) / M
    r = r0 * (r1 / r0) ** (np.arange(N + 1) / N)
    v = np.zeros((N + 1, M, 2), np.float32)
    v[..., 0] = r[:, None] * np.cos(th)[None, :]
    v[..., 1] = r[:, None] * np.sin(th)[None, :]
    return v

def make(M, N, scheme, mach):
    s = Solver(M, N)
    s.set_vertices(annulus(M, N))
    s.set_params(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=mach, aoa_deg=3.0, K_p=0.0, K_u=0.75,
                 cfl=0.5, maxdt=math.inf, muscl=1, scheme=scheme, ramp=0.0)
    s.prepare_state("freestream")
    return s

out = {{}}
s = make(200, 96, "SLAU2", 2.0)
for k in range(3):
    s.step(7)
out["single"] = s.state()
s.close()
sols = [make(100, 40, "SLAU2", 0.8), make(67, 33, "AUSM+-up", 3.0), make(150, 75, "SLAU", 1.5)]
b = Batch()
for x in sols:
    b.add(x)
for k in range(4):
    b.step(5)
for i, x in enumerate(sols):
    out["batch%d" % i] = x.state()
b.close()
for x in sols:
    x.close()
np.savez({path!r}, **out)
'''


def run_child(tmp_path, pdl, rows):
    path = str(tmp_path / f"pdl{pdl}_rows{rows}.npz")
    code = CHILD.format(root=str(ROOT), pkg=str(ROOT / "ausm-webgpu_b200"), path=path)
    env = dict(os.environ, AUSM_PDL=pdl, AUSM_TILE_ROWS=rows)
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(path)


@pytest.mark.parametrize("rows", ["8", "16"])
def test_pdl_on_and_off_bit_identical(tmp_path, rows):
    on = run_child(tmp_path, "1", rows)
    off = run_child(tmp_path, "0", rows)
    assert set(on.files) == set(off.files)
    for k in on.files:
        assert np.all(np.isfinite(on[k])), k
        np.testing.assert_array_equal(on[k], off[k], err_msg=k)
