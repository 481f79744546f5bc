"""Helpers to rebuild the oracle inputs of a golden case (tests/golden/ref_cases.npz)."""
import numpy as np

from oracle.oracle import Params

RUNS = ["run_ausmup_m03_kp_fs", "run_ausmup_m2_a3_4412", "run_ausmup_m8_a0_fs", "run_defaults_m38",
        "run_slau2_long", "run_slau2_m05_a2_fs", "run_slau2_m05_rest", "run_slau2_m08_a4_odd",
        "run_slau2_nomuscl_m15", "run_slau_m2_a0_fs", "run_slau_m6_odd"]
GRIDS = ["grid_33x17", "grid_48x20", "grid_64x32"]


def params_of(g, name) -> Params:
    a = g[f"{name}/params"]
    p = Params()
    p.gamma, p.in_rho, p.in_pressure = a[0], a[1], a[2]
    p.inflow[0], p.inflow[1] = a[3], a[4]
    for k in range(4):
        p.in_state[k] = a[5 + k]
    p.K_p, p.K_u, p.cfl, p.maxdt = a[9], a[10], a[11], a[12]
    p.muscl, p.scheme = int(a[13]), int(a[14])
    return p


def grid_of(g, name):
    gname = str(g[f"{name}/grid"][0])
    M, N = (int(x) for x in g[f"{gname}/meta"][:2])
    return gname, M, N, g[f"{gname}/gridPoints1"]


def kwargs_of(g, name) -> dict:
    """Solver parameters of a case as given to make_params (mach, aoa_deg, scheme, ...)."""
    import json
    kw = json.loads(str(g[f"{name}/kw"][0]))
    kw.setdefault("maxdt", float("inf"))
    return kw
