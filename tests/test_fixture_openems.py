"""The oracle against the reference's native-openEMS fixtures (CPU).

tests/fixtures/engine_comparison of the reference holds the probe voltage of
a 16x8x18 PEC cavity from openEMS's basic/sse/sse-compressed engines (bit
identical).  The operator generator plus the oracle reproduce it within the
1e-4 relative L2 bar in every arithmetic mode; this pins the oracle, the
generator's EC-FDTD conventions and the probe timing to native openEMS.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from efs_b200 import opgen, workloads
from oracle.oracle import OracleEngine

GOLD = os.path.join(ROOT, "tests", "golden")


def test_constants_match_fixture():
    c = json.load(open(os.path.join(GOLD, "constants.json")))
    assert abs(c["C0"] - opgen.C0) == 0 and abs(c["MUE0"] - opgen.MUE0) < 1e-22
    assert abs(c["EPS0"] - opgen.EPS0) < 1e-24 and abs(c["Z0"] - opgen.Z0) < 1e-9


@pytest.mark.parametrize("mode", ["f32", "js", "f64"])
def test_cavity_probe_matches_native_openems(mode):
    job = workloads.openems_cavity()
    ref = np.load(os.path.join(GOLD, "openems_cavity_vp.npy"))
    t = np.load(os.path.join(GOLD, "openems_cavity_t.npy"))
    assert abs(t[1] / 2 - job["dT"]) < 1e-22
    e = OracleEngine(job["grid"], job["coefficients"], mode=mode)
    v = workloads.run_probe_job(e, job)
    assert v.shape == ref.shape
    err = np.linalg.norm(v - ref) / np.linalg.norm(ref)
    assert err < 1e-4, err


def test_find_path_staircase():
    """The excitation curve (10,5,12)->(11,6,13) steps y, z, x (the order that
    reproduces the fixture; the other orders miss it by >15 %)."""
    job = workloads.openems_cavity()
    Nx, Ny, Nz = job["grid"]
    dirs = list(job["excitation"]["dir"])
    assert dirs == [1, 2, 0]
    assert list(job["excitation"]["pos"]) == [10 * Ny * Nz + 5 * Nz + 12, 10 * Ny * Nz + 6 * Nz + 12, 10 * Ny * Nz + 6 * Nz + 13]
