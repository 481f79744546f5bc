"""Benchmark of the explicit TVD-RK3 O-grid time step (Mcell-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one GPU): NACA 0024 O-grid of 4096 x 3072 cells (12.58 M), circular far field
at 40 chords, geometric radial stretching with a first cell of 1e-3 chord, M = 6,
AoA = 4 deg, SLAU2 + MUSCL, TVD-RK3, CFL 0.5, FP32 state, uniform freestream start
(the large precision-study configuration).  Synthetic: the grid and flow are generated
here, there is no dataset.  One timed step = one TVD-RK3 step (three fused stage
launches) of the whole grid; the 201 MB state buffers and 403 MB of face records are
larger than the 126 MB L2, so every step streams them from HBM.  The timed region is
one reference frame of K steps (step(K): dt from the state at the frame's start, one CFL
reduction at its end, main.js:744-791), CUDA events on the solver's stream, synchronised
on both sides; it is repeated for about 1.5 s and the median region is reported (regions
of K separate step(1) calls, dt every step, alternate with them and are reported
beside as ms_per_step_dt_every_step), with the SM clock sampled by nvidia-smi
every 50 ms from before the warm-up to the end.  The default line also carries the
batched configuration (64 uneven grids) and a bounded sample of the served stream.

Multi-GPU (torchrun): every rank advances its own replica of the grid (solves are
independent; there is no data-path collective), value = all ranks' cell-updates / the
max over ranks of the device-timed region; scaling is weak.  Host-side timing
reductions use torch.distributed with the gloo backend.

--impl reference times the reference's own step on the host cores: the reference's
WGSL compute shaders compiled for the CPU (oracle/_ref, built from the reference
tree) when present, else the oracle restatement; each step is one RK3 step of a
sub-grid of the same flow sized so the run ends within a few minutes.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "ausm-webgpu_b200"))

WORKLOAD = dict(name="naca0024_4096x3072_m6_aoa4_slau2", naca=24, M=4096, N=3072, far_chords=40.0,
                first_spacing=1e-3, mach=6.0, aoa_deg=4.0, scheme="SLAU2", cfl=0.5, grid_iters=200)
ALG_BYTES_PER_CELL_STEP = 152  # 3 stages x (16 in + 16 out) + 2 x 16 Qn + 3 x 8 vertex
TIMED_S = 1.5  # seconds of repeated timed regions (the median region is reported)
METRIC = "Mcell-updates/s per RK3 step"

# 64 independent O-grids, cells log-uniform from 128x96 to 1024x768 (aspect 4:3), random
# NACA 4-digit bodies (camber 0-6 %, position 0.2-0.6, thickness 8-18 %), Mach U[0.1, 3],
# AoA U[-4, 8] deg, scheme uniform over SLAU2 / SLAU / AUSM+-up, 5000 RK3 steps each from
# a uniform freestream start, CFL 0.5; seeded.
BATCH = dict(name="batch64_uneven_128x96-1024x768", count=64, seed=20261203, cells_lo=128 * 96,
             cells_hi=1024 * 768, steps=5000, chunk=100, far_chords=20.0, first_spacing=1e-3, cfl=0.5,
             grid_iters=200, ref_steps=500)


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def max_over_ranks(x: float, dist=None) -> float:
    """Max of a host scalar over all ranks (device times are taken as the slowest rank)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, dist=None) -> float:
    """Sum of a host scalar over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(cells: int):
    """Per-launch DRAM bytes of the fused stage kernel from the committed ncu summary."""
    p = ROOT / "profiles" / "fused_stage_4096x3072.md"
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_cell_launch:\s*([0-9.eE+-]+)", p.read_text())
    if not m:
        return None
    return float(m.group(1)) * cells


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, interval_ms: int = 50):
        self.idx = gpu_index
        self.ms = interval_ms
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", str(self.ms)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return None
        try:
            rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
            os.unlink(self.f.name)
        except OSError:
            return None
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_solver(ausm, wl, engine="fused", M=None, N=None):
    M = M or wl["M"]
    N = N or wl["N"]
    s = ausm.Solver(M, N, engine=engine)
    size = 0.5  # half chord: chord 1 centred at the origin
    s.set_body_naca4(wl["naca"], size, 0.0)
    s.set_outer_circle(wl["far_chords"] * 2 * size)
    s.set_radial_stretch(wl["first_spacing"] * 2 * size)
    s.generate_grid(wl["grid_iters"], "multicolor")
    s.set_params(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=wl["mach"], aoa_deg=wl["aoa_deg"], K_p=0.0,
                 K_u=0.75, cfl=wl["cfl"], maxdt=math.inf, muscl=1, scheme=wl["scheme"], ramp=0.0)
    s.prepare_state("freestream")
    return s


# Served stream: Poisson arrivals at `rate` req/s; each request a random NACA 4-digit
# airfoil (as in BATCH), grid cells log-uniform 16k-1M (aspect 4:3), Mach U[0.3, 6],
# AoA U[-4, 8] deg, scheme uniform; stop at a 4-decade density-residual drop or 50000
# steps; admission by a 160 GB HBM budget.  The stream is a bounded sample of
# `requests` arrivals (the full 10000-request stream is hours of GPU time) served with
# `slots` concurrent solves, fewer than the requests, so that requests wait for slots
# and are admitted as others retire.
SERVE = dict(name="served_poisson", seed=20261203, requests=48, rate=200.0, cells_lo=16384, cells_hi=1 << 20,
             residual_drop=4.0, max_steps=50000, chunk=100, budget=160e9, slots=16, far_chords=20.0,
             first_spacing=1e-3, grid_iters=200)


def serve_stream(cfg):
    import numpy as np
    rng = np.random.default_rng(cfg["seed"] + 1)
    n = cfg["requests"]
    arrivals = np.cumsum(rng.exponential(1.0 / cfg["rate"], n))
    lo, hi = math.log(cfg["cells_lo"]), math.log(cfg["cells_hi"])
    out = []
    for k in range(n):
        cells = math.exp(rng.uniform(lo, hi))
        M = max(16, int(round(math.sqrt(cells * 4.0 / 3.0) / 2)) * 2)
        N = max(12, int(round(M * 0.75)))
        m, pos, t = int(rng.integers(0, 7)), int(rng.integers(2, 7)), int(rng.integers(8, 19))
        out.append(dict(t=float(arrivals[k]), M=M, N=N, naca=m * 1000 + (pos * 100 if m else 0) + t,
                        mach=float(rng.uniform(0.3, 6.0)), aoa=float(rng.uniform(-4.0, 8.0)),
                        scheme=int(rng.integers(0, 3))))
    return out


def placed_stream(ausm, cfg, rank, world):
    """The requests of the stream this rank serves: whole requests placed on devices by
    budget and work (ausm.place_requests; every rank computes the same placement)."""
    stream = serve_stream(cfg)
    if world == 1:
        return stream
    reqs = [ausm.make_request(sp["M"], sp["N"], naca4=sp["naca"], max_steps=cfg["max_steps"]) for sp in stream]
    dev = ausm.place_requests([ausm.request_bytes(r) for r in reqs],
                              [float(r.M) * r.N * r.max_steps for r in reqs], world, cfg["budget"])
    return [sp for sp, d in zip(stream, dev) if d == rank]


def run_served(ausm, cfg, plain, rank=0, world=1):
    """Submits the stream (this rank's share of it) at its arrival times to a server
    (worker thread) and waits for every result; latency = submit -> result ready."""
    import numpy as np
    stream = placed_stream(ausm, cfg, rank, world)
    srv = ausm.Server(cfg["budget"], cfg["slots"], cfg["chunk"], plain=plain)
    srv.start()
    ids = []
    t0 = time.perf_counter()
    for sp in stream:
        delay = sp["t"] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        r = ausm.make_request(sp["M"], sp["N"], naca4=sp["naca"], chord=1.0, far_radius=cfg["far_chords"],
                              first_spacing=cfg["first_spacing"], grid_iters=cfg["grid_iters"],
                              residual_drop=cfg["residual_drop"], max_steps=cfg["max_steps"], mach=sp["mach"],
                              aoa_deg=sp["aoa"], scheme=sp["scheme"])
        ids.append(srv.submit(r))
    srv.drain()
    wall = time.perf_counter() - t0
    res = [srv.poll(i) for i in ids]
    st = srv.stats()
    srv.stop()
    srv.close()
    lat = np.array([r["latency_ms"] for r in res])
    queued = np.array([r["queue_ms"] for r in res])
    done = [r for r in res if r["state"] == 0]
    return {"solves_per_s": len(done) / wall, "wall_s": wall, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "queue_ms_p50": float(np.percentile(queued, 50)),
            "queue_ms_max": float(queued.max()), "slots": cfg["slots"] if not plain else 1,
            "finished": len(done), "failed": len(res) - len(done),
            "converged": sum(1 for r in done if r["stop"] == 1), "max_steps": sum(1 for r in done if r["stop"] == 2),
            "steps_mean": float(np.mean([r["steps"] for r in res])), "rounds": st["rounds"],
            "mcell_updates_per_s": st["cell_updates"] / wall / 1e6, "peak_gb": st["peak_bytes"] / 1e9}, res


def run_serve_mode(ausm, cfg, rank=0, world=1, dist=None):
    served, rs = run_served(ausm, cfg, plain=False, rank=rank, world=world)
    plain, rp = run_served(ausm, cfg, plain=True, rank=rank, world=world)
    if world > 1:  # whole-job rate: all ranks' solves over the slowest rank's wall time
        for d in (served, plain):
            d["rank_wall_s"] = d["wall_s"]
            d["wall_s"] = max_over_ranks(d["wall_s"], dist)
            d["finished_rank"] = d["finished"]
            d["finished"] = int(round(sum_over_ranks(d["finished"], dist)))
            d["solves_per_s"] = d["finished"] / d["wall_s"]
    err = 0.0
    for a, b in zip(rs, rp):
        if a["state"] == 0 and b["state"] == 0:
            err = max(err, float(abs(a["Cp"] - b["Cp"]).max() / max(abs(b["Cp"]).max(), 1e-30)))
    return {"metric": "served solves/s", "value": served["solves_per_s"], "unit": "solves/s",
            "workload": cfg["name"], "requests": cfg["requests"], "rate_per_s": cfg["rate"],
            "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"], "served": served,
            "plain_one_solve_at_a_time": plain, "speedup_vs_plain": served["solves_per_s"] / plain["solves_per_s"],
            "cp_max_rel_diff_vs_plain": err,
            "config": {k: cfg[k] for k in ("seed", "requests", "rate", "residual_drop", "max_steps", "chunk",
                                           "budget", "slots")}}


def run_precision(ausm, steps, chunk=1000, sensitivity=False, reference=False, noise=False):
    """The 4096 x 3072 workload advanced `steps` RK3 steps by the FP32 fused engine
    (FP64 metrics, residual norm and forces) and by the full-FP64 engine from the same
    grid and initial state, dt recomputed every `chunk` steps in both; errors of the
    FP32 run against the FP64 run (both start from the float32 freestream, the FP64 engine
    from it widened).  sensitivity: a second FP64 run from the freestream in double (1e-8
    away from the float32 one): how far two FP64 runs drift apart from that alone, the
    floor for any float32 run of this flow.  reference: the reference-shaped FP32 engine
    (the reference's arithmetic bit for bit, FP32 metrics) against the FP64 run too.
    noise: an FP64 run from the float32 start with each cell's state changed by about one
    float32 rounding (relative N(0, 1e-7), seeded): how far round-off-sized per-cell noise
    alone takes an FP64 run."""
    import numpy as np
    wl = dict(WORKLOAD)
    out = {"metric": "precision study", "workload": wl["name"], "steps": steps, "chunk": chunk}
    runs = {}
    centres = None
    for engine in (("fused", "f64") + (("f64_exact_start",) if sensitivity else ())
                   + (("reference",) if reference else ()) + (("f64_noisy_start",) if noise else ())):
        s = build_solver(ausm, wl)
        if centres is None:
            v = s.vertices().astype(np.float64)
            centres = 0.25 * (v[:-1] + np.roll(v[:-1], -1, axis=1) + v[1:] + np.roll(v[1:], -1, axis=1))
        if engine == "reference":
            s.set_engine("reference")
        elif engine != "fused":
            s.set_engine("f64")  # carries the float32 freestream over, widened
            if engine == "f64_exact_start":
                s.prepare_state("freestream")  # the freestream in double
            if engine == "f64_noisy_start":
                q = s.state()
                rng = np.random.default_rng(7)
                q[1:s.N + 1] *= (1.0 + 1e-7 * rng.standard_normal(q[1:s.N + 1].shape)).astype(np.float32)
                s.set_state(q)
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            n = min(chunk, steps - done)
            s.step(n)
            done += n
        runs[engine] = {"seconds": time.perf_counter() - t0, "q": s.state_f64()[1:s.N + 1],
                        "F": s.forces(with_cp=True), "l2": s.residual_l2()}
        s.close()
    g = 1.4
    def prim(q):
        rho = q[..., 0]
        p = (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / rho) * (g - 1.0)
        return rho, p
    r32, p32 = prim(runs["fused"]["q"])
    r64, p64 = prim(runs["f64"]["q"])
    # where the density differs by more than 1e-2 of its max: downstream of the trailing
    # edge (x > 0.5 chord) or not, and the radius of those cells
    big = np.abs(r32 - r64) > 1e-2 * np.abs(r64).max()
    rad = np.hypot(centres[..., 0], centres[..., 1])
    out["rho_1e-2_cells"] = {"count": int(big.sum()), "downstream_fraction": float((centres[..., 0][big] > 0.5).mean())
                             if big.any() else None, "radius_median": float(np.median(rad[big])) if big.any() else None,
                             "x_range": [float(centres[..., 0][big].min()), float(centres[..., 0][big].max())]
                             if big.any() else None,
                             "j_range": [int(np.nonzero(big)[0].min()), int(np.nonzero(big)[0].max())] if big.any() else None}
    def errs(a, b):
        out = {"max_rel": float(np.abs(a - b).max() / np.abs(b).max()),
               "l2_rel": float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))}
        if a.ndim == 2:
            # the same allowing each cell a one-cell shift (periodic in i, clamped in j):
            # a shock or expansion that sits one cell apart in the two runs counts as zero
            bp = np.pad(b, ((1, 1), (0, 0)), mode="edge")
            best = np.full(a.shape, np.inf)
            for dj in (-1, 0, 1):
                for di in (-1, 0, 1):
                    best = np.minimum(best, np.abs(a - np.roll(bp[1 + dj:1 + dj + a.shape[0]], di, axis=1)))
            out["max_rel_one_cell_shift"] = float(best.max() / np.abs(b).max())
            out["cells_above_1e-3_rel"] = int(np.count_nonzero(np.abs(a - b) > 1e-3 * np.abs(b).max()))
        return out
    cp32, cp64 = runs["fused"]["F"]["Cp"], runs["f64"]["F"]["Cp"]
    F32, F64 = runs["fused"]["F"], runs["f64"]["F"]
    out.update({"rho": errs(r32, r64), "p": errs(p32, p64), "cp": errs(cp32, cp64),
                "cl": {"f32": F32["Cl"], "f64": F64["Cl"], "rel": abs(F32["Cl"] - F64["Cl"]) / abs(F64["Cl"])},
                "cd": {"f32": F32["Cd"], "f64": F64["Cd"], "rel": abs(F32["Cd"] - F64["Cd"]) / abs(F64["Cd"])},
                "residual_l2": {"f32": runs["fused"]["l2"], "f64": runs["f64"]["l2"]},
                "seconds": {"f32": runs["fused"]["seconds"], "f64": runs["f64"]["seconds"]}})
    if reference:
        rr, pr = prim(runs["reference"]["q"])
        Fr = runs["reference"]["F"]
        big = np.abs(rr - r64) > 1e-2 * np.abs(r64).max()
        out["reference_vs_f64"] = {
            "rho": errs(rr, r64), "p": errs(pr, p64), "cp": errs(Fr["Cp"], cp64),
            "cl_rel": abs(Fr["Cl"] - F64["Cl"]) / abs(F64["Cl"]), "cd_rel": abs(Fr["Cd"] - F64["Cd"]) / abs(F64["Cd"]),
            "rho_1e-2_cells": int(big.sum()), "seconds": runs["reference"]["seconds"]}
    if noise:
        rn, pn = prim(runs["f64_noisy_start"]["q"])
        Fn = runs["f64_noisy_start"]["F"]
        out["f64_noisy_start_vs_f64"] = {
            "rho": errs(rn, r64), "p": errs(pn, p64), "cp": errs(Fn["Cp"], cp64),
            "cl_rel": abs(Fn["Cl"] - F64["Cl"]) / abs(F64["Cl"]), "cd_rel": abs(Fn["Cd"] - F64["Cd"]) / abs(F64["Cd"]),
            "rho_1e-2_cells": int(np.count_nonzero(np.abs(rn - r64) > 1e-2 * np.abs(r64).max()))}
    if sensitivity:
        rb, pb = prim(runs["f64_exact_start"]["q"])
        Fb = runs["f64_exact_start"]["F"]
        out["f64_exact_start_vs_f64"] = {
            "rho": errs(rb, r64), "p": errs(pb, p64), "cp": errs(Fb["Cp"], cp64),
            "cl_rel": abs(Fb["Cl"] - F64["Cl"]) / abs(F64["Cl"]), "cd_rel": abs(Fb["Cd"] - F64["Cd"]) / abs(F64["Cd"])}
    return out


def run_precision_ensemble(ausm, wl, steps, seeds, chunk=1000):
    """How large a float32 error the flow allows: the fused and the reference-shaped FP32
    engines (the latter is the reference's arithmetic bit for bit), each from the float32
    freestream (seed 0) and from seeds - 1 starts with every cell changed by about one
    float32 rounding (relative N(0, 1e-7), numpy seed k), against the FP64 engine from the
    freestream in double; dt recomputed every `chunk` steps in all.  Per run: density and
    pressure errors of the final state (max over max, relative L2), and the lift and drag
    errors at the end and at the worst chunk; per engine the range over the runs."""
    import numpy as np
    g = 1.4

    def run(engine, seed):
        s = build_solver(ausm, wl)
        N = s.N
        if engine == "f64":
            s.set_engine("f64")
            s.prepare_state("freestream")  # in double
        elif engine == "reference":
            s.set_engine("reference")
        if seed > 0:
            q = s.state()
            rng = np.random.default_rng(seed)
            q[1:N + 1] *= (1.0 + 1e-7 * rng.standard_normal(q[1:N + 1].shape)).astype(np.float32)
            s.set_state(q)
        done, forces = 0, []
        while done < steps:
            n = min(chunk, steps - done)
            s.step(n)
            done += n
            f = s.forces()
            forces.append((f["Cl"], f["Cd"]))
        q = s.state_f64()[1:N + 1]
        s.close()
        rho = q[..., 0]
        p = (q[..., 3] - 0.5 * (q[..., 1] ** 2 + q[..., 2] ** 2) / rho) * (g - 1.0)
        return rho, p, np.array(forces)

    r64, p64, f64 = run("f64", 0)
    out = {"metric": "precision ensemble", "workload": wl["name"], "grid": f"{wl['M']}x{wl['N']}", "steps": steps,
           "chunk": chunk, "seeds": seeds, "runs": {}, "range": {}}
    for engine in ("fused", "reference"):
        for seed in range(seeds):
            rho, p, f = run(engine, seed)
            ef = np.abs(f - f64) / np.abs(f64)
            out["runs"][f"{engine}/{seed}"] = {
                "rho_max": float(np.abs(rho - r64).max() / np.abs(r64).max()),
                "rho_l2": float(np.sqrt(np.mean((rho - r64) ** 2)) / np.sqrt(np.mean(r64 ** 2))),
                "p_max": float(np.abs(p - p64).max() / np.abs(p64).max()),
                "p_l2": float(np.sqrt(np.mean((p - p64) ** 2)) / np.sqrt(np.mean(p64 ** 2))),
                "cl_end": float(ef[-1, 0]), "cl_worst_chunk": float(ef[:, 0].max()),
                "cd_end": float(ef[-1, 1]), "cd_worst_chunk": float(ef[:, 1].max())}
        runs = [v for k, v in out["runs"].items() if k.startswith(engine + "/")]
        out["range"][engine] = {key: [min(r[key] for r in runs), max(r[key] for r in runs)] for key in runs[0]}
    return out


def batch_specs(cfg):
    import numpy as np
    rng = np.random.default_rng(cfg["seed"])
    out = []
    lo, hi = math.log(cfg["cells_lo"]), math.log(cfg["cells_hi"])
    for _ in range(cfg["count"]):
        cells = math.exp(rng.uniform(lo, hi))
        M = max(16, int(round(math.sqrt(cells * 4.0 / 3.0) / 2)) * 2)
        N = max(12, int(round(M * 0.75)))
        m, pos, t = int(rng.integers(0, 7)), int(rng.integers(2, 7)), int(rng.integers(8, 19))
        out.append(dict(M=M, N=N, naca=m * 1000 + (pos * 100 if m else 0) + t, mach=float(rng.uniform(0.1, 3.0)),
                        aoa=float(rng.uniform(-4.0, 8.0)), scheme=int(rng.integers(0, 3))))
    return out


def build_spec_solver(ausm, sp, cfg):
    s = ausm.Solver(sp["M"], sp["N"])
    s.set_body_naca4(sp["naca"], 0.5, 0.0)
    s.set_outer_circle(cfg["far_chords"])
    s.set_radial_stretch(cfg["first_spacing"])
    s.generate_grid(cfg["grid_iters"], "multicolor")
    s.set_params(gamma=1.4, in_rho=1.0, in_pressure=1.0 / 1.4, mach=sp["mach"], aoa_deg=sp["aoa"], K_p=0.0,
                 K_u=0.75, cfl=cfg["cfl"], maxdt=math.inf, muscl=1, scheme=sp["scheme"], ramp=0.0)
    s.prepare_state("freestream")
    return s


def run_batched(ausm, cfg, warmup, plain=True):
    """Config: BATCH.  The same 64 solves (a) in one batch (one launch per RK stage and
    scheme group over all their tiles, graph-replayed chunks of cfg['chunk'] steps) and
    (b) by the plain path, one solve after another, each ausm_step(chunk) call launching
    its own three stage kernels per step.  dt is recomputed every chunk steps in both.
    Both start from the freestream state; solves/s = 64 / elapsed.  The surface Cp of
    both runs is compared at the end.  plain=False skips (b) (profiling runs)."""
    import numpy as np
    specs = batch_specs(cfg)
    sols = [build_spec_solver(ausm, sp, cfg) for sp in specs]
    cells = sum(sp["M"] * sp["N"] for sp in specs)
    steps, chunk = cfg["steps"], cfg["chunk"]
    b = ausm.Batch()
    for s in sols:
        b.add(s)
    for _ in range(warmup):
        b.step(chunk, wait=False)
    for s in sols:
        s.prepare_state("freestream")
    b.synchronize()
    t0 = time.perf_counter()
    ms = b.time_steps(chunk, steps // chunk)
    wall_b = time.perf_counter() - t0
    cp_b = [s.forces(with_cp=True)["Cp"] for s in sols]
    diverged = int(sum(1 for s in sols if not math.isfinite(s.max_wave_speed())))
    for s in list(b.members):
        b.remove(s)
    b.close()
    wall_p, err = None, None
    if plain:
        for s in sols:  # plain path warm-up, then the same start
            s.step(1)
            s.prepare_state("freestream")
            s.synchronize()
        t0 = time.perf_counter()
        for s in sols:  # dt held over `chunk` steps, as in the batch
            for _ in range(steps // chunk):
                s.step(chunk, wait=False)
            s.synchronize()
        wall_p = time.perf_counter() - t0
        cp_p = [s.forces(with_cp=True)["Cp"] for s in sols]
        err = 0.0
        for a, c in zip(cp_b, cp_p):
            if np.all(np.isfinite(a)) and np.all(np.isfinite(c)):
                err = max(err, float(np.abs(a - c).max() / max(np.abs(c).max(), 1e-30)))
    # (c) the plain path as the comparison list of the benchmark configurations defines it:
    # one solve at a time on the unfused reference-shaped engine (the reference's five
    # dispatches per stage), timed on a bounded sample of the same run (the first
    # ref_steps of every solve's steps) and scaled to the full step count
    ref_plain = None
    if plain and cfg.get("ref_steps"):
        rs = cfg["ref_steps"]
        for s in sols:
            s.set_engine("reference")
            s.prepare_state("freestream")
            s.step(1)
            s.prepare_state("freestream")
            s.synchronize()
        t0 = time.perf_counter()
        for s in sols:
            for _ in range(rs // chunk):
                s.step(chunk, wait=False)
            s.synchronize()
        wall_r = (time.perf_counter() - t0) * steps / rs
        ref_plain = {"engine": "reference-shaped (unfused, 5 dispatches per stage)", "sample_steps": rs,
                     "wall_s_scaled": wall_r, "solves_per_s": len(sols) / wall_r}
    for s in sols:
        s.close()
    n = len(specs)
    return {"metric": "batched solves/s", "value": n / (ms * 1e-3), "unit": "solves/s",
            "workload": f"{cfg['name']}_{steps}steps", "solves": n, "cells_total": cells, "steps_per_solve": steps,
            "device_ms": ms, "wall_s": wall_b, "solves_per_s_wall": n / wall_b,
            "plain_one_launch_per_solve": {"wall_s": wall_p, "solves_per_s": n / wall_p} if plain else None,
            "speedup_vs_plain": wall_p / wall_b if plain else None, "cp_max_rel_diff_vs_plain": err,
            "plain_reference_shaped": ref_plain,
            "speedup_vs_plain_reference_shaped": ref_plain["wall_s_scaled"] / wall_b if ref_plain else None,
            "diverged": diverged, "mcell_updates_per_s": cells * steps / (ms * 1e-3) / 1e6,
            "gpu_launches": (3 * chunk * len({sp["scheme"] for sp in specs}) + 3) * (steps // chunk),
            "sizes": f"{min(sp['M'] * sp['N'] for sp in specs)}..{max(sp['M'] * sp['N'] for sp in specs)} cells"}


def workload_grid_host(wl, M=None, N=None):
    """The workload's O-grid built on the host cores with the library's generator restated
    in the oracle (test infrastructure): NACA body (chord 1 at the origin), circular far
    field, the geometric radial stretch (oracle/geometry_ref.stretched_guess) and
    wl['grid_iters'] multicolour TTM sweeps in double (the oracle's restatement of the
    library's FP64 generator), rounded to float32.  Used by the CPU legs only."""
    import numpy as np
    from oracle.geometry_ref import circular_outer, naca4_boundary, stretched_guess
    from oracle.oracle import Oracle
    M = M or wl["M"]
    N = N or wl["N"]
    body = naca4_boundary(M, wl["naca"], 0.5, 0.0)
    outer = circular_outer(M, wl["far_chords"])
    o = Oracle(M, N, "f64")
    o.set_vertices(stretched_guess(body, outer, N, wl["first_spacing"]))
    o.grid_multicolor(wl["grid_iters"], 0.0)
    v = o.vertices().astype(np.float32)
    o.close()
    return v


def cpu_reference_sample(wl, vertices=None, target_s=20.0, K=1):
    """Time the reference's step on the host cores (oracle/_ref, else the oracle port).
    The sample is the whole workload grid when K steps of it fit in target_s seconds at
    the probed host rate (vertices: the GPU run's grid; None: built on the host with the
    same generator), else a sub-grid of the same flow on a linear-interpolation grid."""
    import numpy as np
    from oracle.oracle import Oracle, RefWGSL, make_params, oracle_lib, ref_available
    from oracle.geometry_ref import naca4_boundary, circular_outer
    kind = "reference" if ref_available() else "port"
    p = make_params(mach=wl["mach"], aoa_deg=wl["aoa_deg"], scheme=wl["scheme"], cfl=wl["cfl"])

    def make(M, N, verts):
        if verts is None:
            o = Oracle(M, N, "f32")
            v = np.zeros((N + 1, M, 2), np.float32)
            v[0] = naca4_boundary(M, wl["naca"], 0.5, 0.0)
            v[N] = circular_outer(M, wl["far_chords"])
            o.set_vertices(v)
            o.grid_interpolate()
            verts = o.vertices()
            o.close()
        if kind == "reference":
            r = RefWGSL(M, N)
            r.set_uniforms(p)
            r.set_grid(verts)
            r.prepare_state(1)
            return r, r.frame
        o = Oracle(M, N, "f32")
        o.set_params(p)
        o.set_vertices(verts)
        o.metrics()
        o.init_state(1)
        return o, o.step

    # probe the host rate on a small grid, then size the sample
    obj, fn = make(256, 192, None)
    fn(1)
    t = time.perf_counter()
    fn(1)
    rate = 256 * 192 / (time.perf_counter() - t)
    del obj
    cells_budget = rate * target_s / max(K, 1)
    same = wl["M"] * wl["N"] <= cells_budget
    if same:
        M, N = wl["M"], wl["N"]
        verts = vertices if vertices is not None else workload_grid_host(wl)
    else:
        scale = max(min(math.sqrt(cells_budget / (wl["M"] * wl["N"])), 1.0), 1 / 32)
        M = max(32, int(wl["M"] * scale) // 4 * 4)
        N = max(24, int(wl["N"] * scale) // 3 * 3)
        verts = None
    obj, fn = make(M, N, verts)
    return kind, M, N, fn, obj, same


def threads_used():
    try:
        from oracle.oracle import oracle_lib
        return int(oracle_lib().orc_num_threads())
    except Exception:
        return os.cpu_count() or 1


def run_reference_arm(args):
    rank, local_rank, world = env_rank()
    if rank != 0:
        return 0
    wl = WORKLOAD
    # the whole run (warm-up and timed steps) within about two and a half minutes
    kind, M, N, fn, obj, same = cpu_reference_sample(wl, None, target_s=150.0, K=args.steps + args.warmup)
    for _ in range(args.warmup):
        fn(1)
    t = time.perf_counter()
    for _ in range(args.steps):
        fn(1)
    el = time.perf_counter() - t
    value = M * N * args.steps / el / 1e6
    sample = f"{args.steps} RK3 steps of a {M}x{N} O-grid of the same flow (NACA 00{wl['naca']:02d}, M {wl['mach']}, " \
             f"AoA {wl['aoa_deg']}, {wl['scheme']})"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl["name"], "sample_grid": f"{M}x{N}", "same_config": same,
                       "grid": "the workload's stretched O-grid, 200 multicolour sweeps, built on the host" if same
                       else "linear-interpolation sub-grid", "parallelism": "host cores"},
            "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": threads_used(), "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="fused", choices=["fused", "reference"])
    ap.add_argument("--e2e-calls", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--small", action="store_true", help="512x384 grid (profiling and quick checks)")
    ap.add_argument("--grid", default=None, help="MxN grid of the same flow instead of 4096x3072 (profiling cases)")
    ap.add_argument("--mode", default="step", choices=["step", "batch", "serve", "precision"],
                    help="step: the 4096x3072 step (headline line, with the batched measurement "
                         "attached); batch: the batched measurement alone; serve: the served stream; "
                         "precision: FP32 against FP64 on the 4096x3072 workload")
    ap.add_argument("--precision-steps", type=int, default=100000)
    ap.add_argument("--precision-noise", action="store_true",
                    help="also an FP64 run from a start with round-off-sized per-cell noise")
    ap.add_argument("--precision-reference", action="store_true",
                    help="also the reference-shaped FP32 engine against FP64")
    ap.add_argument("--precision-sensitivity", action="store_true",
                    help="also an FP64 run from the freestream in double (sensitivity of the flow)")
    ap.add_argument("--precision-ensemble", type=int, default=0,
                    help="K > 0: the FP32 engines from K starts one rounding apart against FP64 "
                         "(on --grid MxN of the same flow, --precision-steps steps)")
    ap.add_argument("--batch-steps", type=int, default=BATCH["steps"],
                    help="steps per solve of the batched measurement (shorter runs for profiling only)")
    ap.add_argument("--no-plain", action="store_true", help="batched measurement without the plain comparison")
    ap.add_argument("--serve-requests", type=int, default=SERVE["requests"])
    ap.add_argument("--serve-rate", type=float, default=SERVE["rate"])
    ap.add_argument("--serve-max-steps", type=int, default=SERVE["max_steps"])
    ap.add_argument("--serve-slots", type=int, default=SERVE["slots"])
    ap.add_argument("--no-serve", action="store_true", help="skip the served stream in --mode step")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched measurement in --mode step")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference_arm(args)

    rank, local_rank, world = env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))

    import numpy as np
    import ausm
    ausm.set_device(local_rank % max(1, ausm.device_count()))
    if args.mode == "batch":
        res = run_batched(ausm, dict(BATCH, steps=args.batch_steps), args.warmup, plain=not args.no_plain)
        if rank == 0:
            print(json.dumps(res))
        return 0
    if args.mode == "precision" and args.precision_ensemble > 0:
        wl = dict(WORKLOAD)
        if args.grid:
            gm, gn = (int(x) for x in args.grid.lower().split("x"))
            wl.update(M=gm, N=gn, name=f"naca0024_{gm}x{gn}_m6_aoa4_slau2")
        res = run_precision_ensemble(ausm, wl, args.precision_steps, args.precision_ensemble)
        if rank == 0:
            print(json.dumps(res))
        return 0
    if args.mode == "precision":
        res = run_precision(ausm, args.precision_steps, sensitivity=args.precision_sensitivity,
                            reference=args.precision_reference, noise=args.precision_noise)
        if rank == 0:
            print(json.dumps(res))
        return 0
    if args.mode == "serve":
        cfg = dict(SERVE, requests=args.serve_requests, rate=args.serve_rate, max_steps=args.serve_max_steps,
                   slots=args.serve_slots)
        res = run_serve_mode(ausm, cfg, rank, world, dist)
        if world > 1:
            res["parallelism"] = f"requests placed on {world} GPUs by budget and work, one server each"
        if rank == 0:
            print(json.dumps(res))
        return 0
    wl = dict(WORKLOAD)
    if args.small:
        wl.update(M=512, N=384, name="naca0024_512x384_m6_aoa4_slau2")
    if args.grid:
        gm, gn = (int(x) for x in args.grid.lower().split("x"))
        wl.update(M=gm, N=gn, name=f"naca0024_{gm}x{gn}_m6_aoa4_slau2")
    s = build_solver(ausm, wl, engine=args.engine)
    M, N = s.M, s.N
    cells = M * N

    # The clock sampler runs from before the warm-up to the end of the timed regions.  The
    # timed region (K steps, CUDA events on the solver's stream, synchronised, barrier
    # first) is repeated until about TIMED_S seconds have passed, so that the clock record
    # covers it; the median region counts.  Every rank repeats it the same number of times.
    # A timed region is one reference frame of K steps, step(K): dt from the state at its
    # start, held for the K steps, and one CFL wave-speed reduction at its end, as the
    # reference's frame loop (main.js:744-791).  Regions of K separate step(1) calls (dt
    # and the reduction every step) alternate with them and are reported beside.
    with Clocks(local_rank) as clk:
        for _ in range(args.warmup):
            s.step(1, wait=False)
        s.synchronize()
        probe = s.time_steps(args.steps, 1)
        reps = int(max_over_ranks(max(3, min(500, math.ceil(TIMED_S * 1e3 / max(probe, 1e-3)))), dist))
        times, walls, times_each = [], [], []
        for _ in range(reps):
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            times.append(s.time_steps(args.steps, 1))
            walls.append(time.perf_counter() - t0)
            if dist:
                dist.barrier()
            times_each.append(s.time_steps(1, args.steps))
    clocks = clk.summary()
    dt_check = s.step(0)  # raises if the run diverged
    ms_med = statistics.median(times)
    ms_each = max_over_ranks(statistics.median(times_each), dist)
    ms = max_over_ranks(ms_med, dist)
    wall = statistics.median(walls)
    value = world * cells * args.steps / (ms * 1e-3) / 1e6

    # end to end through the public API with pinned host buffers
    e2e = None
    if args.e2e_calls > 0:
        try:
            import torch
            host = torch.empty(((N + 3), M, 4), dtype=torch.float32, pin_memory=True).numpy()
        except Exception:
            host = np.empty(((N + 3), M, 4), dtype=np.float32)
        s.state(out=host)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_calls):
            s.set_state(host)
            s.step(args.e2e_steps)
            s.forces(with_cp=True)
            s.state(out=host)
        e2e_t = max_over_ranks(time.perf_counter() - t0, dist)
        state_bytes = (N + 3) * M * 16
        e2e = {"value": world * cells * args.e2e_steps * args.e2e_calls / e2e_t / 1e6, "unit": "Mcell-updates/s",
               "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes + 8 * M + 48 + 8,
               "step": f"ausm_set_state + ausm_step(n={args.e2e_steps}) + ausm_forces(Cp) + ausm_get_state "
                       f"from/to pinned host memory", "calls": args.e2e_calls}

    peak, peak_kind = peaks()
    achieved = cells * ALG_BYTES_PER_CELL_STEP * args.steps / (ms_med * 1e-3) / 1e9
    traffic = traffic_from_profile(cells)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind ==
                "measured" else "fallback 6650 GB/s",
                "bytes_per_cell_step": ALG_BYTES_PER_CELL_STEP,
                "kernel": "k_fused_tile_tma (3 launches per RK3 step; achieved over the whole step)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            verts = s.vertices()
            kind, cM, cN, fn, obj, _ = cpu_reference_sample(wl, verts, target_s=args.cpu_seconds, K=2)
            fn(1)
            t0 = time.perf_counter()
            fn(2)
            el = time.perf_counter() - t0
            cpu = {"value": cM * cN * 2 / el / 1e6, "unit": "Mcell-updates/s", "cores": threads_used(), "kind": kind,
                   "sample": f"2 RK3 steps of a {cM}x{cN} O-grid of the same flow on the host cores"}
            del obj
            # the same on one core (a smaller sub-grid of the same flow)
            from oracle.oracle import oracle_lib
            L, n0 = oracle_lib(), threads_used()
            L.orc_set_num_threads(1)
            try:
                kind1, M1, N1, fn1, obj1, _ = cpu_reference_sample(wl, None, target_s=max(2.0, args.cpu_seconds / 3), K=1)
                t0 = time.perf_counter()
                fn1(1)
                el1 = time.perf_counter() - t0
                cpu["value_1core"] = M1 * N1 / el1 / 1e6
                cpu["sample_1core"] = f"1 RK3 step of a {M1}x{N1} O-grid of the same flow on 1 core"
                del obj1
            finally:
                L.orc_set_num_threads(n0)
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Mcell-updates/s", "cores": None, "kind": None, "sample": f"failed: {e}"}

    batched = None
    if world == 1 and not args.no_batch and not args.small:
        s.close()
        s = None
        batched = run_batched(ausm, BATCH, args.warmup)
    served = None
    if world == 1 and not args.no_serve and not args.small:
        if s is not None:
            s.close()
            s = None
        served = run_serve_mode(ausm, dict(SERVE, requests=args.serve_requests, rate=args.serve_rate,
                                           max_steps=args.serve_max_steps, slots=args.serve_slots))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mcell-updates/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": wl["name"], "cells": cells, "grid": f"{M}x{N}", "engine": args.engine,
                           "parallelism": f"replicas{world}", "l2": ("inputs larger than L2" if cells * 16 > 126e6 else "inputs fit in L2") +
                           f" ({cells * 16 / 1e6:.0f} MB state, {cells * 32 / 1e6:.0f} MB face records)",
                           "wall_s": wall, "timed_regions": len(times),
                           "ms_per_step_min_max": [min(times) / args.steps, max(times) / args.steps],
                           "timed_region": f"one frame of {args.steps} steps (dt held, one CFL reduction)",
                           "ms_per_step_dt_every_step": ms_each / args.steps},
                # per step(1): fused, three stage kernels (dt is computed in stage 1); reference,
                # 5 dispatches per stage, the dt kernel and the wave-speed reduction
                "gpu_launches": 3 * args.steps if args.engine == "fused" else 15 * args.steps + 3, "clocks": clocks, "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e, "batched": batched, "served": served}
        print(json.dumps(line))
    if s is not None:
        s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
