"""Bit-exact parity at the benchmark workloads' own sizes.

The CUDA engine against the oracle's f32 mode (every product and sum rounded
in the reference's operand order) on the full jobs, not reduced copies:

* the plain large solve, 512^3 (workloads.large_plain(512): 40 boxes, Mur on
  +-x/+-y, UPML 8 on +-z, TFSF, NF2FF with 3 frequencies): 3 timesteps,
  fields and UPML fluxes bit for bit, NF2FF accumulators to 1e-6;
* the dispersive solve (workloads.dispersive: UPML on all faces, Drude and
  Lorentz spheres with the ADE apply step, 30-degree TFSF, NF2FF with 5
  frequencies) at 800 x 800 x 400 when the host has the memory for the
  oracle (about 40 GB free), else at 400 x 400 x 200: 2 timesteps, fields and
  ADE state bit for bit;
* the patch antenna (86 x 87 x 71 graded mesh, UPML 8 on all faces, 50 ohm
  port) run to its -50 dB energy end criterion: the probe ring and the final
  fields bit for bit.
"""
import os

import numpy as np
import pytest

from test_gpu_parity import assert_bitexact

pytestmark = pytest.mark.gpu


def _threads():
    from oracle import oracle
    oracle.set_threads(os.cpu_count() or 1)


def _fields_equal(g, o, what):
    f = g.getFields()
    assert_bitexact(f["volt"], o.volt, what + " volt")
    assert_bitexact(f["curr"], o.curr, what + " curr")


def test_large_plain_512_bitexact(cuda_engine_cls):
    from efs_b200 import workloads
    from oracle.oracle import OracleEngine
    _threads()
    job = dict(workloads.large_plain(512), probes=[])
    g = cuda_engine_cls()
    assert g.initGPU()
    workloads.configure(g, job)
    o = OracleEngine(mode="f32")
    workloads.configure(o, job)
    g.iterate(3)
    o.iterate(3)
    _fields_equal(g, o, "512^3 after 3 steps")
    for r in range(len(job["pml"])):
        assert_bitexact(g.debugRead("pml_volt_flux", r), o.read("pml_volt_flux", r), "vflux %d" % r)
        assert_bitexact(g.debugRead("pml_curr_flux", r), o.read("pml_curr_flux", r), "cflux %d" % r)
    ag, ao = g.readNF2FFAccumulation(True), o.readNF2FFAccumulation(True)
    for k in ("accumE", "accumH"):
        a, b = np.asarray(ag[k], np.float64), np.asarray(ao[k], np.float64)
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), k
    g.destroy()


def _dispersive_grid():
    try:
        import psutil
        free = psutil.virtual_memory().available
    except ImportError:
        free = 0
    return (800, 800, 400) if free > 40e9 else (400, 400, 200)


def test_dispersive_fullsize_bitexact(cuda_engine_cls):
    from efs_b200 import workloads
    from oracle.oracle import OracleEngine
    _threads()
    grid = _dispersive_grid()
    job = workloads.dispersive(grid=grid)
    assert job["ade"]["apply"]
    g = cuda_engine_cls()
    assert g.initGPU()
    workloads.configure(g, job)
    o = OracleEngine(mode="f32")
    workloads.configure(o, job)
    g.iterate(2)
    o.iterate(2)
    _fields_equal(g, o, "dispersive %s after 2 steps" % (grid,))
    for name in ("ade_volt", "ade_volt_lor"):
        ref = np.concatenate([o.read(name, oi, d) for oi in range(2) for d in range(3)])
        assert_bitexact(g.debugRead(name), ref, name)
    g.destroy()


def test_patch_full_run_bitexact(cuda_engine_cls):
    from efs_b200 import workloads
    from oracle.oracle import OracleEngine
    _threads()
    job = workloads.patch_antenna()
    g = cuda_engine_cls()
    assert g.initGPU()
    o = OracleEngine(mode="f32")
    steps = [workloads.run(e, job)[0] for e in (g, o)]
    assert steps[0] == steps[1] and steps[0] < job["maxTS"]     # both stop at the -50 dB criterion, same step
    rg, ro = g.readProbeGatherBuffered(), o.readProbeGatherBuffered()
    assert rg["numSamples"] == ro["numSamples"] == steps[0]
    assert_bitexact(rg["data"], ro["data"], "patch probe ring")
    _fields_equal(g, o, "patch after %d steps" % steps[0])
    g.destroy()
