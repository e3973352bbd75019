"""Patch antenna (86 x 87 x 71 graded mesh, UPML 8, 50 ohm port) on the CUDA
engine against an FP64 run of the oracle: the error statement of the plain
single solve.

Both advance in chunks of 100 timesteps until the orchestrator's energy end
criterion (-50 dB of the peak, checked every 100 steps) or 30 000 steps.
Bars: port V and I time series within 1e-4 relative L2, S11 within 0.05 dB
over 0-3 GHz (f0 + fc), energy within 1e-3 relative at every checkpoint.  Set
EFS_ACCURACY_OUT to a file path to keep the measured errors as JSON.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_patch_antenna_against_f64(cuda_engine_cls):
    from efs_b200 import postprocess as pp
    from efs_b200 import workloads
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)
    job = workloads.patch_antenna()
    g = cuda_engine_cls()
    assert g.initGPU()
    sl_g = workloads.configure(g, job)
    o = oracle.OracleEngine(mode="f64")
    sl_o = workloads.configure(o, job)
    eg, eo = [], []
    steps = 0
    while steps < job["maxTS"]:
        g.iterate(100)
        o.iterate(100)
        steps += 100
        eg.append(g.computeEnergy(lagged=False))
        eo.append(o.energy())
        if eg[-1] < max(eg) * job["endCrit"]:
            break
    vg = workloads.probe_series(g, job, sl_g)
    vo = workloads.probe_series(o, job, sl_o)
    g.destroy()
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    err_v, err_i = rel(vg[:, 0], vo[:, 0]), rel(vg[:, 1], vo[:, 1])
    dT = job["dT"]
    t_v = pp.probe_times(job["probes"][0], len(vg), 1, dT)
    t_i = pp.probe_times(job["probes"][1], len(vg), 1, dT)
    s_g = pp.compute_s11((t_v, vg[:, 0]), (t_i, vg[:, 1]), fmax=3e9, nf=201)
    s_o = pp.compute_s11((t_v, vo[:, 0]), (t_i, vo[:, 1]), fmax=3e9, nf=201)
    err_s11 = float(np.abs(s_g["s11_dB"][1:] - s_o["s11_dB"][1:]).max())
    eg, eo = np.array(eg), np.array(eo)
    err_e = float(np.abs(eg - eo).max() / eo.max())
    out = {"steps": steps, "port_V_relL2": err_v, "port_I_relL2": err_i, "S11_max_dB_diff": err_s11,
           "energy_max_rel": err_e, "best_S11_dB": s_g["bestS11"], "best_freq_GHz": s_g["bestFreqGHz"],
           "best_S11_dB_f64": s_o["bestS11"]}
    if os.environ.get("EFS_ACCURACY_OUT"):
        with open(os.environ["EFS_ACCURACY_OUT"], "w") as f:
            json.dump(out, f)
    assert err_v <= 1e-4 and err_i <= 1e-4, out
    assert err_s11 <= 0.05, out
    assert err_e <= 1e-3, out
