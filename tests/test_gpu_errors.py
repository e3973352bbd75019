"""Error statements of the CUDA engine (FP32) against an FP64 run of the
oracle, for the dispersive and the large plain workloads at reduced sizes
(the FP64 oracle finishes them in seconds).

Dispersive: workloads.dispersive at 48 x 40 x 32 (UPML on all faces,
Drude/Lorentz spheres with the ADE apply step on, so the dispersion reaches
the fields; TFSF at 30 degrees, NF2FF with 5 frequencies), 1200 steps (the
pulse through the spheres).  Plain: workloads.large_plain(64) (boxes, Mur, UPML on z, TFSF, NF2FF
with 3 frequencies), 800 steps.  Compared: E and H (relative L2), the energy
at every 100-step checkpoint (relative to its peak), the ADE state (relative
L2) and Dmax at every NF2FF frequency, from the engine's own far-field
kernel against the FP64 oracle's far field of its FP64 accumulators.  Bars
(the same as the patch antenna's): fields and ADE state 1e-4, energy and
Dmax 1e-3.  Set EFS_ACCURACY_OUT to a file path to keep the measured errors
as JSON (one object per workload, appended).
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _statement(cls, job, steps, name):
    from efs_b200 import workloads
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)
    g = cls()
    assert g.initGPU()
    workloads.configure(g, job)
    o = oracle.OracleEngine(mode="f64")
    workloads.configure(o, job)
    eg, eo = [], []
    for _ in range(steps // 100):
        g.iterate(100)
        o.iterate(100)
        eg.append(g.computeEnergy(lagged=False))
        eo.append(o.energy())
    f = g.getFields()
    out = {"workload": name, "steps": steps, "volt_relL2": _rel(f["volt"], o.volt), "curr_relL2": _rel(f["curr"], o.curr)}
    eg, eo = np.array(eg), np.array(eo)
    out["energy_max_rel"] = float(np.abs(eg - eo).max() / eo.max())
    if job.get("ade"):
        for nm in ("ade_volt", "ade_volt_lor"):
            ref = np.concatenate([o.read(nm, oi, d) for oi in range(2) for d in range(3)])
            out[nm + "_relL2"] = _rel(g.debugRead(nm), ref)
    ff = lambda aE, aH, meta, th, ph, fr: oracle.far_field(aE, aH, meta, th, ph, fr, 1.0, (0.0, 0.0, 0.0))
    dm = []
    for fi in range(len(job["nf2ff_freqs"])):
        dg = workloads.far_field_summary(g, job, freq_index=fi)["Dmax"]
        do = workloads.far_field_summary(o, job, freq_index=fi, far_field_fn=ff)["Dmax"]
        dm.append(abs(dg - do) / do)
    out["Dmax_max_rel"] = float(max(dm))
    g.destroy()
    if os.environ.get("EFS_ACCURACY_OUT"):
        with open(os.environ["EFS_ACCURACY_OUT"], "a") as fh:
            fh.write(json.dumps(out) + "\n")
    return out


def test_dispersive_against_f64(cuda_engine_cls):
    from efs_b200 import workloads
    job = workloads.dispersive(grid=(48, 40, 32), pml=4, chunk=8, steps=1200, tfsf_inset=8, nf2ff_inset=6, workers=1)
    assert job["ade"]["apply"]
    out = _statement(cuda_engine_cls, job, 1200, "dispersive 48x40x32 (ADE applied)")
    assert out["volt_relL2"] <= 1e-4 and out["curr_relL2"] <= 1e-4, out
    assert out["ade_volt_relL2"] <= 1e-4 and out["ade_volt_lor_relL2"] <= 1e-4, out
    assert out["energy_max_rel"] <= 1e-3 and out["Dmax_max_rel"] <= 1e-3, out


def test_large_plain_against_f64(cuda_engine_cls):
    from efs_b200 import workloads
    job = workloads.large_plain(64, tfsf_inset=12, nf2ff_inset=6, steps=800, chunk=16)
    out = _statement(cuda_engine_cls, job, 800, "large_plain 64^3")
    assert out["volt_relL2"] <= 1e-4 and out["curr_relL2"] <= 1e-4, out
    assert out["energy_max_rel"] <= 1e-3 and out["Dmax_max_rel"] <= 1e-3, out
