"""Served form (efs_b200.serve): every result is the same alone and in the mix.

Requests of different sizes and kinds (lumped-port filters with probes, TFSF
jobs with NF2FF) arrive while others are running; the server admits them as
member slots free up, runs them together in one batch and retires each at its
own step count.  Each request's probe series, NF2FF accumulators and energy
must equal, bit for bit, those of the same request run alone on one engine.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def solo(job, steps):
    from efs_b200 import workloads
    from efs_b200.engine import CudaEngine
    e = CudaEngine()
    assert e.initGPU()
    slices = workloads.configure(e, job)
    e.iterate(steps)
    out = {}
    if job.get("probes"):
        out["probes"] = workloads.probe_series(e, job, slices)
    if job.get("nf2ff"):
        acc = e.readNF2FFAccumulation(True)
        out["nf2ff"] = (acc["accumE"], acc["accumH"])
    out["energy"] = e.energyNoAlloc()          # the reduction the server's retirement uses
    e.destroy()
    return out


def test_served_results_equal_alone(cuda_engine_cls):
    from efs_b200 import workloads
    from efs_b200.serve import Server
    templates = {(k, s): workloads.served_template(k, s, steps=400) for k, s in
                 (("port", 40), ("port", 48), ("tfsf", 40), ("tfsf", 32))}
    plan = [(("port", 40), 150), (("tfsf", 40), 90), (("port", 48), 200),      # first wave
            (("tfsf", 32), 64), (("port", 40), 130), (("tfsf", 40), 77)]      # arrive while the first wave runs
    srv = Server(hbm_budget=8e9, max_members=4, chunk=64)
    try:
        for key, steps in plan[:3]:
            srv.submit(templates[key], steps)
        assert srv.round()                       # first wave admitted and running
        for key, steps in plan[3:]:
            srv.submit(templates[key], steps)
        rounds = 0
        while srv.round():
            rounds += 1
            assert len(srv.active) <= 4
        assert not srv.waiting and not srv.active
    finally:
        srv.close()
    done = sorted(srv.finished, key=lambda r: r.rid)
    assert len(done) == len(plan)
    # at least one request was admitted while another was mid-run
    assert any(r.admitted > min(q.admitted for q in done) and r.rid >= 3 for r in done)
    for r, (key, steps) in zip(done, plan):
        ref = solo(templates[key], steps)
        assert r.result["energy"] == ref["energy"], (r.rid, key)
        if "probes" in ref:
            assert np.array_equal(r.result["probes"], ref["probes"]), (r.rid, key)
        if "nf2ff" in ref:
            for a, b in zip(r.result["nf2ff"], ref["nf2ff"]):
                assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32)), (r.rid, key)


def test_served_admission_respects_budget(cuda_engine_cls):
    """With a budget of one request's estimate, a second solve never fits beside a
    resident one (admission counts the resident solves' actual bytes plus the
    newcomer's estimate), so requests run one after another."""
    from efs_b200 import workloads
    from efs_b200.serve import Server, estimate_bytes
    job = workloads.served_template("port", 40, steps=200)
    srv = Server(hbm_budget=estimate_bytes(job) * 1.01, max_members=8, chunk=32)
    try:
        for steps in (40, 50, 60):
            srv.submit(job, steps)
        while srv.round():
            assert len(srv.active) <= 1
    finally:
        srv.close()
    assert [r.rid for r in srv.finished] == [0, 1, 2]


def test_evicted_solve_resumes_bit_exact(cuda_engine_cls):
    """With one member slot, a long solve is evicted (its state read to the host
    and its engine freed) so a short request can run, then restored into a new
    engine; both results equal the same requests run alone, bit for bit."""
    from efs_b200 import workloads
    from efs_b200.serve import Server
    long_job = workloads.served_template("tfsf", 40, steps=600)
    short_job = workloads.served_template("port", 40, steps=200)
    srv = Server(hbm_budget=8e9, max_members=1, chunk=64, evict_ratio=2.0)
    try:
        lid = srv.submit(long_job, 500)
        assert srv.round()
        sid = srv.submit(short_job, 120)
        while srv.round():
            assert len(srv.active) <= 1
    finally:
        srv.close()
    by = {r.rid: r for r in srv.finished}
    assert srv.evicted == 1 and by[lid].evictions == 1
    assert by[sid].done < by[lid].done
    for rid, job, steps in ((lid, long_job, 500), (sid, short_job, 120)):
        ref = solo(job, steps)
        assert by[rid].result["energy"] == ref["energy"], rid
        if "probes" in ref:
            assert np.array_equal(by[rid].result["probes"], ref["probes"]), rid
        if "nf2ff" in ref:
            for a, b in zip(by[rid].result["nf2ff"], ref["nf2ff"]):
                assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32)), rid
