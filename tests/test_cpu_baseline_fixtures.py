"""The benchmark-configuration fixtures on the host (no GPU): each was made on the grid
that tests/baseline_cases.py builds now (checksums), holds the checkpoints its recipe
writes, and its values are finite and consistent with themselves."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from baseline_cases import CONFIG1, CONFIG2, CONFIG5_SUB, make_grid, make_grid_multicolor

GOLDEN = Path(__file__).resolve().parent / "golden"


def sha(v):
    return hashlib.sha256(v.tobytes()).hexdigest()


@pytest.mark.parametrize("name,cfg", [("baseline_c1.npz", CONFIG1), ("baseline_c2.npz", CONFIG2)])
def test_jacobi_grid_fixtures(name, cfg):
    g = np.load(GOLDEN / name)
    assert sha(make_grid(cfg)) == str(g["grid_sha256"][0])


def test_config5_subgrid_fixture():
    g = dict(np.load(GOLDEN / "baseline_c5sub.npz"))
    cfg = CONFIG5_SUB
    assert sha(make_grid_multicolor(cfg)) == str(g["grid_sha256"][0])
    M, N, sub = cfg["M"], cfg["N"], cfg["sub"]
    for c in cfg["checkpoints"]:
        k = str(c)
        assert g[k + "/rho_sub"].shape == (N // sub, M // sub) and g[k + "/p_sub"].shape == (N // sub, M // sub)
        assert g[k + "/cp"].shape == (M,)
        for key in ("rho_sub", "p_sub", "cp", "forces"):
            assert np.all(np.isfinite(g[f"{k}/{key}"]))
        assert np.all(g[k + "/rho_sub"] > 0) and np.all(g[k + "/p_sub"] > 0)
        # the wall Cp is the first sampled row's pressure on every 8th cell
        p_wall = g[k + "/p_sub"][0]
        cp_from_p = (p_wall - 1.0 / 1.4) / (0.5 * cfg["mach"] ** 2)
        assert np.array_equal(cp_from_p, g[k + "/cp"][::sub])
        # lift and drag: Cl / Cd of the oracle's force record agree with its ratio entry
        F = g[k + "/forces"]
        assert F[5] == pytest.approx(F[3] / F[4], rel=1e-12)
