"""The dispersive job generator (workloads.dispersive) on a small grid, on the
CPU: sphere coverage, the two media and their single-pole coefficients, the
oblique TFSF and NF2FF inputs, determinism per seed, and an oracle run in
which the voltage-side ADE state evolves while the all-zero current side
stays exactly +0 (the case the CUDA engine skips)."""
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
    assert 0.30 <= job["dispersive_cells"] / N < 0.40          # spheres stop once 30% is covered
    orders = job["ade"]["orders"]
    assert [o["hasLorentz"] for o in orders] == [False, True]
    assert sum(o["numCells"] for o in orders) == job["dispersive_cells"]
    cells = [set(np.asarray(o["directions"][0]["pos_idx"]).tolist()) for o in orders]
    assert not (cells[0] & cells[1])                          # a cell belongs to one medium
    dT, delta = job["dT"], 0.25e-3
    wp, gam = 1.4e16, 3e13
    d_int = (1 - gam * dT / 2) / (1 + gam * dT / 2)
    d_ext = opgen.EPS0 * wp * wp * dT * delta / (1 + gam * dT / 2)
    w0, dl, de = 2 * math.pi * 15e9, 2 * math.pi * 1e9, 2.0
    for o, (ki, ke) in zip(orders, ((d_int, d_ext), ((1 - dl * dT) / (1 + dl * dT),
                                                     opgen.EPS0 * de * w0 * w0 * dT * delta / (1 + dl * dT)))):
        assert len(o["directions"]) == 3
        for d in o["directions"]:
            assert np.all(d["v_int_ADE"] == np.float32(ki)) and np.all(d["v_ext_ADE"] == np.float32(ke))
            assert "i_int_ADE" not in d                       # the current side has no coefficients
    lor = orders[1]["directions"][0]["v_Lor_ADE"]
    assert np.all(lor == np.float32(w0 * w0 * dT * dT))


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
