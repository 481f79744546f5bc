"""Parity on the benchmark configurations themselves, against the oracle and the
reference's own shaders, through the C ABI (tests/baseline_cases.py has the inputs).

Configuration 1 (NACA 0012, 256 x 128, M 0.5, SLAU2):
  - one step: the fused engine against the float32 oracle, normwise <= 1e-5 (as the
    golden-case gate); the reference-shaped engine bit for bit;
  - the configuration's 2000 steps (frames of 100): against the reference's own shaders
    (tests/golden/baseline_c1.npz), density relative L2 and wall Cp (max difference over
    max |Cp|) <= 1e-4 for the fused engine, bit for bit for the reference-shaped engine;
  - the converged run (frames of 500 after that, to a 4-decade density-residual drop or
    the served configuration's 50000-step limit, whichever comes first; the reference
    stops at the limit, 3.2 decades down): density relative L2 <= 1e-4, and wall Cp
    within max(1e-4, the spread of the reference itself): the fixture also holds the
    end state of the reference's shaders compiled with fused multiply-add contraction,
    and the two float32 builds of the reference differ by 4.2e-4 of max |Cp| there (a
    slowly converging subsonic mode amplifies round-off), so no float32 code can be held
    to 1e-4 in Cp at that point; in density they agree to 4.5e-5.
Configuration 2 (NACA 2412, 512 x 384; M 0.8 SLAU2, M 2 AUSM+-up, M 8 SLAU): one step
  at 1e-5 and 300 steps (frames of 100) at 1e-4 normwise against the float32 oracle run
  on the host cores in the test; as written (20000 steps) against the float32 oracle's
  run (tests/golden/baseline_c2.npz).
Configuration 5 (NACA 0024, M 6, AoA 4, SLAU2) on its 1024 x 768 sub-grid against the
  FP64 oracle (tests/golden/baseline_c5sub.npz, up to 100000 steps): the full-FP64
  engine bit for bit, the FP32 engines against the reference's own float32 error.
"""
import hashlib
import math
from pathlib import Path

import numpy as np
import pytest

from baseline_cases import (CONFIG1, CONFIG2, CONFIG5_SUB, density_l2_rel, flow_kwargs, make_grid, make_grid_multicolor,
                            primitives, wall_cp)
from test_gpu_parity import normwise

pytestmark = pytest.mark.gpu

TOL_STEP1 = 1e-5
TOL_RUN = 1e-4
GOLDEN = Path(__file__).resolve().parent / "golden" / "baseline_c1.npz"

_grids = {}


def grid(cfg):
    key = (cfg["M"], cfg["N"], cfg["naca"])
    if key not in _grids:
        _grids[key] = make_grid(cfg)
    return _grids[key]


@pytest.fixture(scope="module")
def c1():
    g = dict(np.load(GOLDEN))
    v = grid(CONFIG1)
    assert hashlib.sha256(v.tobytes()).hexdigest() == str(g["grid_sha256"][0]), "grid differs from the fixture's"
    return g, v


def solver(cfg, v, run, engine="fused"):
    from ausm import Solver
    s = Solver(cfg["M"], cfg["N"], engine=engine)
    s.set_vertices(v)
    s.set_params(**flow_kwargs(run, cfg["cfl"]))
    s.prepare_state("freestream")
    return s


def oracle(cfg, v, run):
    from oracle.oracle import Oracle, make_params
    o = Oracle(cfg["M"], cfg["N"], "f32")
    o.set_params(make_params(mach=run["mach"], aoa_deg=run["aoa_deg"], scheme=run["scheme"], cfl=cfg["cfl"]))
    o.set_vertices(v)
    o.metrics()
    o.init_state(1)
    return o


def advance(s, steps, frame):
    done = 0
    while done < steps:
        n = min(frame, steps - done)
        s.step(n)
        done += n


def test_config1_one_step(c1):
    _, v = c1
    N = CONFIG1["N"]
    o = oracle(CONFIG1, v, CONFIG1)
    dt_ref = o.step(1)
    ref = o.state()[1:N + 1]
    o.close()
    for engine in ("fused", "reference"):
        s = solver(CONFIG1, v, CONFIG1, engine)
        dt = s.step(1)
        q = s.state()[1:N + 1]
        s.close()
        if engine == "reference":
            assert np.array_equal(q, ref) and np.float32(dt) == np.float32(dt_ref)
        else:
            err = normwise(q, ref)
            assert err <= TOL_STEP1, f"normwise {err:.3e}"
            assert abs(dt - dt_ref) <= 1e-5 * dt_ref


@pytest.mark.parametrize("engine", ["fused", "reference"])
def test_config1_2000_steps(c1, engine):
    g, v = c1
    N = CONFIG1["N"]
    s = solver(CONFIG1, v, CONFIG1, engine)
    advance(s, CONFIG1["steps"], CONFIG1["frame"])
    q = s.state()
    f = s.forces(with_cp=True)
    s.close()
    rho = q[1:N + 1, :, 0]
    if engine == "reference":
        assert np.array_equal(rho, g["rho_2000"])
        assert np.array_equal(wall_cp(q[1], CONFIG1["mach"]), g["cp_2000"])
        return
    d_rho = density_l2_rel(rho, g["rho_2000"])
    d_cp = np.abs(f["Cp"] - g["cp_2000"]).max() / np.abs(g["cp_2000"]).max()
    assert d_rho <= TOL_RUN, f"density relative L2 {d_rho:.3e}"
    assert d_cp <= TOL_RUN, f"wall Cp {d_cp:.3e} of max |Cp|"


def test_config1_converged(c1):
    g, v = c1
    N = CONFIG1["N"]
    s = solver(CONFIG1, v, CONFIG1)
    advance(s, CONFIG1["steps"], CONFIG1["frame"])
    advance(s, int(g["steps_end"][0]) - CONFIG1["steps"], CONFIG1["converged_frame"])
    q = s.state()
    f = s.forces(with_cp=True)
    s.close()
    d_rho = density_l2_rel(q[1:N + 1, :, 0], g["rho_end"])
    cmax = np.abs(g["cp_end"]).max()
    d_cp = np.abs(f["Cp"] - g["cp_end"]).max() / cmax
    spread = np.abs(g["cp_end_fma"] - g["cp_end"]).max() / cmax  # the reference against itself
    assert d_rho <= TOL_RUN, f"density relative L2 {d_rho:.3e} after {int(g['steps_end'][0])} steps"
    assert d_cp <= max(TOL_RUN, spread), \
        f"wall Cp {d_cp:.3e} of max |Cp| after {int(g['steps_end'][0])} steps (reference spread {spread:.3e})"


@pytest.mark.parametrize("k", range(len(CONFIG2["runs"])), ids=lambda k: CONFIG2["runs"][k]["scheme"])
def test_config2_runs(k):
    run = CONFIG2["runs"][k]
    v = grid(CONFIG2)
    N = CONFIG2["N"]
    o = oracle(CONFIG2, v, run)
    s = solver(CONFIG2, v, run)
    o.step(1)
    s.step(1)
    err1 = normwise(s.state()[1:N + 1], o.state()[1:N + 1])
    assert err1 <= TOL_STEP1, f"after one step: normwise {err1:.3e}"
    advance(o, 299, 100)
    advance(s, 299, 100)
    ref = o.state()[1:N + 1]
    q = s.state()[1:N + 1]
    o.close()
    s.close()
    assert np.all(np.isfinite(q))
    err = normwise(q, ref)
    assert err <= TOL_RUN, f"after 300 steps: normwise {err:.3e}"


GOLDEN_C2 = Path(__file__).resolve().parent / "golden" / "baseline_c2.npz"


@pytest.mark.skipif(not GOLDEN_C2.exists(), reason="configuration-2 fixture not generated")
@pytest.mark.parametrize("engine", ["fused", "reference"])
@pytest.mark.parametrize("k", range(len(CONFIG2["runs"])), ids=lambda k: CONFIG2["runs"][k]["scheme"])
def test_config2_as_written(k, engine):
    """Configuration 2 as written: 20000 RK3 steps in frames of 100 against the float32
    oracle, which reproduces the reference's shaders bit for bit (tests/golden/
    baseline_c2.npz).  Density (relative L2 over every 4th cell in i and j) and wall Cp
    (max over max |Cp|) within max(1e-4, the spread between the oracle and the same
    oracle compiled with FMA contraction) for the fused engine; the reference-shaped
    engine bit for bit."""
    g = dict(np.load(GOLDEN_C2))
    run = CONFIG2["runs"][k]
    v = grid(CONFIG2)
    assert hashlib.sha256(v.tobytes()).hexdigest() == str(g["grid_sha256"][0])
    N = CONFIG2["N"]
    s = solver(CONFIG2, v, run, engine)
    advance(s, 20000, 100)
    q = s.state()
    f = s.forces(with_cp=True)
    s.close()
    assert np.all(np.isfinite(q))
    rho = q[1:N + 1:4, ::4, 0]
    ref_rho, ref_cp = g[f"{k}/rho_sub"], g[f"{k}/cp"]
    if engine == "reference":
        assert np.array_equal(rho, ref_rho)
        assert np.array_equal(f["Cp"], ref_cp)
        return
    d_rho = density_l2_rel(rho, ref_rho)
    s_rho = density_l2_rel(g[f"{k}/rho_sub_fma"], ref_rho)
    cmax = np.abs(ref_cp).max()
    d_cp = np.abs(f["Cp"] - ref_cp).max() / cmax
    s_cp = np.abs(g[f"{k}/cp_fma"] - ref_cp).max() / cmax
    assert d_rho <= max(TOL_RUN, s_rho), f"density relative L2 {d_rho:.3e} (reference spread {s_rho:.3e})"
    assert d_cp <= max(TOL_RUN, s_cp), f"wall Cp {d_cp:.3e} of max |Cp| (reference spread {s_cp:.3e})"


GOLDEN_C5 = Path(__file__).resolve().parent / "golden" / "baseline_c5sub.npz"
TOL_C5_F64 = 1e-9  # FP64 engine vs FP64 oracle, relative to the field's max
C5_ENGINES = {}


def c5_run(v, engine):
    """Configuration 5's flow on the 1024 x 768 sub-grid by one engine, dt recomputed every
    1000 steps, observed at the fixture's checkpoints, with the lift and drag after every
    1000 steps (run once per engine per module)."""
    from ausm import Solver
    if engine in C5_ENGINES:
        return C5_ENGINES[engine]
    cfg = CONFIG5_SUB
    M, N, sub, chunk = cfg["M"], cfg["N"], cfg["sub"], cfg["chunk"]
    g = dict(np.load(GOLDEN_C5))
    checkpoints = sorted(int(k.split("/")[0]) for k in g if k.endswith("/cp"))
    s = Solver(M, N, engine=engine)
    s.set_vertices(v)
    s.set_params(**flow_kwargs(cfg, cfg["cfl"]))
    s.prepare_state("freestream")  # in double for the FP64 engine, as the oracle's
    out, forces, done = {}, [], 0
    for c in checkpoints:
        while done < c:
            n = min(chunk, c - done)
            s.step(n)
            done += n
            f = s.forces()
            forces.append((f["Cl"], f["Cd"]))
        q = s.state_f64()[1:N + 1]
        rho, p = primitives(q)
        out[c] = {"rho_sub": rho[::sub, ::sub], "p_sub": p[::sub, ::sub],
                  "cp": (p[0] - 1.0 / 1.4) / (0.5 * cfg["mach"] ** 2), "Cl": forces[-1][0], "Cd": forces[-1][1],
                  "chunks": len(forces),
                  "sha": hashlib.sha256(np.ascontiguousarray(q, np.float64).tobytes()).hexdigest(),
                  "finite": bool(np.all(np.isfinite(q)))}
    s.close()
    C5_ENGINES[engine] = (g, checkpoints, out, np.array(forces))
    return C5_ENGINES[engine]


def c5_errors(r, g, c):
    """errors of one engine's checkpoint against the FP64 oracle's"""
    k = str(c)
    e = {}
    for name in ("rho_sub", "p_sub", "cp"):
        a, b = r[name], g[f"{k}/{name}"]
        e[name] = float(np.abs(a - b).max() / np.abs(b).max())
        e[name + "_l2"] = float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))
    F = g[f"{k}/forces"]
    e["Cl"] = abs(r["Cl"] - F[3]) / abs(F[3])
    e["Cd"] = abs(r["Cd"] - F[4]) / abs(F[4])
    return e


@pytest.fixture(scope="module")
def c5():
    if not GOLDEN_C5.exists():
        pytest.skip("configuration-5 sub-grid fixture not generated")
    v = make_grid_multicolor(CONFIG5_SUB)
    g = np.load(GOLDEN_C5)
    assert hashlib.sha256(v.tobytes()).hexdigest() == str(g["grid_sha256"][0]), "grid differs from the fixture's"
    return v


def test_config5_subgrid_f64_engine(c5):
    """The full-FP64 GPU engine, which the 4096 x 3072 precision study takes as its FP64
    solution, against the FP64 oracle on configuration 5's flow at 1024 x 768: the whole
    float64 state bit for bit at every checkpoint (up to 100000 steps; both evaluate the
    same operations in the same order, correctly rounded, with no contraction), and the
    sampled fields within 1e-9 of their max as a readable second statement."""
    g, checkpoints, out, _ = c5_run(c5, "f64")
    for c in checkpoints:
        r = out[c]
        assert r["finite"]
        e = c5_errors(r, g, c)
        same = r["sha"] == str(g[f"{c}/state_sha256"][0])
        print(f"{c} steps: FP64 engine vs FP64 oracle {e} bit-identical state: {same}")
        for name in ("rho_sub", "p_sub", "cp"):
            assert e[name] <= TOL_C5_F64, f"{name} after {c} steps: {e[name]:.3e}"
        assert same, f"state after {c} steps differs from the FP64 oracle's"


def test_config5_subgrid_fp32_error(c5):
    """The FP32 engines' error against the FP64 oracle on configuration 5's flow at
    1024 x 768 (the precision study's comparison at a size the oracle runs on the host
    cores).  The reference-shaped engine is the reference's own float32 arithmetic (bit
    for bit its shaders), so its error is what a float32 code of this solver incurs on
    this flow.  At every checkpoint the fused engine's density, pressure and wall Cp
    (max and L2 over max and norm) are within max(2 x the reference's, 1e-4).  Lift and
    drag: the M 6 leading-edge region amplifies round-off-sized differences by about 1e5
    over 20000 steps, after which every float32 run's lift error wanders from one
    1000-step chunk to the next (1e-5 to 2.4e-3 for the reference's arithmetic from four
    start states one rounding apart); the fused engine's Cl and Cd are held to twice the
    largest error the reference-shaped engine showed in any chunk up to that checkpoint
    (against the FP64 engine, which is the oracle bit for bit), or 1e-4."""
    g, checkpoints, fused, _ = c5_run(c5, "fused")
    _, _, ref, ref_forces = c5_run(c5, "reference")
    _, _, _, f64_forces = c5_run(c5, "f64")
    ref_force_err = np.abs(ref_forces - f64_forces) / np.abs(f64_forces)  # per chunk: Cl, Cd
    for c in checkpoints:
        assert fused[c]["finite"] and ref[c]["finite"]
        ef, er = c5_errors(fused[c], g, c), c5_errors(ref[c], g, c)
        envelope = ref_force_err[:ref[c]["chunks"]].max(axis=0)
        print(f"{c} steps vs the FP64 oracle: fused {ef}")
        print(f"{c} steps vs the FP64 oracle: reference {er}; its largest Cl, Cd errors so far {envelope}")
        for name in ("rho_sub", "rho_sub_l2", "p_sub", "p_sub_l2", "cp", "cp_l2"):
            assert ef[name] <= max(2.0 * er[name], 1e-4), \
                f"{name} after {c} steps: fused {ef[name]:.3e}, reference's own float32 {er[name]:.3e}"
        for k, name in enumerate(("Cl", "Cd")):
            assert ef[name] <= max(2.0 * envelope[k], 1e-4), \
                f"{name} after {c} steps: fused {ef[name]:.3e}, reference's largest so far {envelope[k]:.3e}"
