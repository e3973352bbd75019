"""The dispersive job generator (workloads.dispersive) on a small grid, on the
CPU: sphere coverage and placement, the two media and their single-pole
coefficients (opgen.ade_drude / ade_lorentz, apply step on), the oblique TFSF
and NF2FF inputs, determinism per seed, and an oracle run in which the
voltage-side ADE state evolves while the all-zero current side stays exactly
+0 (the case the CUDA engine skips)."""
import math

import numpy as np

from efs_b200 import opgen, workloads
from oracle.oracle import OracleEngine

GRID = (48, 40, 32)


def small(seed=5):
    return workloads.dispersive(grid=GRID, pml=4, chunk=8, steps=200, tfsf_inset=8, nf2ff_inset=6, seed=seed, workers=1)


def test_coverage_media_and_coefficients():
    job = small()
    N = GRID[0] * GRID[1] * GRID[2]
    target = job["dispersive_target"]
    assert 0 < target <= 0.3 * N
    assert target <= job["dispersive_cells"] < target + 4 * 4 * 4 * 8   # spheres stop once the target is covered
    orders = job["ade"]["orders"]
    assert job["ade"]["apply"] is True
    assert [o["hasLorentz"] for o in orders] == [False, True]
    assert sum(o["numCells"] for o in orders) == job["dispersive_cells"]
    cells = [np.asarray(o["directions"][0]["pos_idx"]) for o in orders]
    assert not (set(cells[0].tolist()) & set(cells[1].tolist()))      # a cell belongs to one medium
    # spheres inside the TFSF box with a 2-cell margin
    lo, hi = job["sphere_box"]
    for c in cells:
        xyz = np.stack([c // (GRID[1] * GRID[2]), (c // GRID[2]) % GRID[1], c % GRID[2]], 1)
        assert xyz.min() >= lo and np.all(xyz <= np.asarray(hi))
    # coefficients: the generator's Drude (implicit) and Lorentz (explicit) poles on the vacuum row
    dT = job["dT"]
    table, mat = job["coefficients"]["table"], job["coefficients"]["mat"]
    vac = np.asarray(table[mat[cells[1][0]]], np.float64)                # Lorentz cells keep the vacuum row
    drow = np.asarray(table[mat[cells[0][0]]], np.float64)
    assert np.all(mat[cells[0]] == mat[cells[0][0]]) and np.all(mat[cells[1]] == mat[cells[1][0]])
    for n in range(3):
        dr = opgen.ade_drude(vac[n:n + 1], vac[3 + n:4 + n], dT, 1.4e16, 3e13)
        lr = opgen.ade_lorentz(vac[n:n + 1], vac[3 + n:4 + n], dT, 2.0, 2 * math.pi * 15e9, 2 * math.pi * 1e9)
        assert dr["scheme"] == "implicit" and lr["scheme"] == "explicit"
        assert drow[n] == np.float32(dr["vv"][0]) and drow[3 + n] == np.float32(dr["vi"][0])
        d0, d1 = orders[0]["directions"][n], orders[1]["directions"][n]
        assert np.all(d0["v_int_ADE"] == np.float32(dr["v_int"][0])) and np.all(d0["v_ext_ADE"] == np.float32(dr["v_ext"][0]))
        assert np.all(d1["v_int_ADE"] == np.float32(lr["v_int"][0])) and np.all(d1["v_ext_ADE"] == np.float32(lr["v_ext"][0]))
        assert np.all(d1["v_Lor_ADE"] == np.float32(lr["v_lor"][0]))
        assert "i_int_ADE" not in d0 and "i_int_ADE" not in d1           # the current side has no coefficients
    # the state-only form keeps the vacuum row on the Drude cells
    off = workloads.dispersive(grid=GRID, pml=4, chunk=8, steps=200, tfsf_inset=8, nf2ff_inset=6, workers=1, apply=False)
    assert off["ade"]["apply"] is False
    t2, m2 = off["coefficients"]["table"], off["coefficients"]["mat"]
    assert np.array_equal(t2[m2[cells[0][0]]], t2[m2[cells[1][0]]])


def test_tfsf_nf2ff_and_determinism():
    job = small()
    assert len(job["nf2ff_freqs"]) == 5
    assert np.allclose(job["nf2ff_freqs"], [7.5e9, 8.75e9, 10e9, 11.25e9, 12.5e9])
    vp = job["tfsf"]["voltagePoints"]
    n = len(vp["field_idx"]) if isinstance(vp, dict) else len(vp)
    assert n > 0
    # oblique incidence (30 degrees in the xz plane): E has x and z components, so both appear
    comps = np.asarray(vp["field_idx"] if isinstance(vp, dict) else [p["field_idx"] for p in vp]) // np.prod(GRID)
    assert {0, 2} <= set(comps.tolist())
    again = small()
    assert np.array_equal(job["coefficients"]["mat"], again["coefficients"]["mat"])
    assert job["dispersive_cells"] == again["dispersive_cells"]
    other = small(seed=6)
    assert other["dispersive_cells"] != job["dispersive_cells"] or not np.array_equal(
        other["ade"]["orders"][0]["directions"][0]["pos_idx"], job["ade"]["orders"][0]["directions"][0]["pos_idx"])


def test_oracle_state_volt_side_only():
    job = small()
    o = OracleEngine(mode="f32")
    workloads.configure(o, job)
    o.iterate(60)
    volt = np.concatenate([o.read("ade_volt", oi, d) for oi in range(2) for d in range(3)])
    curr = np.concatenate([o.read("ade_curr", oi, d) for oi in range(2) for d in range(3)])
    assert np.abs(volt).max() > 0
    assert np.all(np.asarray(curr, np.float32).view(np.uint32) == 0)   # +0 bit for bit
    assert np.isfinite(o.energy()) and o.energy() > 0
