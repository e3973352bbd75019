"""Batched form (efs_batch_*) against the same engines stepped alone.

Every member of a batch runs the single engine's thread bodies in the single
engine's phase order, so its fields, probe ring, UPML fluxes, ADE state and
NF2FF accumulators must equal, bit for bit, those of an identical engine
advanced on its own.  Members differ in grid size and extensions; batch calls use
irregular step counts (one spans two captured graphs) and shapes.
"""
import numpy as np
import pytest

from conftest import idx
from test_gpu_parity import assert_bitexact, mur_faces, nf2ff_inputs, pml_region, rand_coeffs

pytestmark = pytest.mark.gpu


def coeffs(N, seed, indexed):
    c = rand_coeffs(N, seed)
    if not indexed:
        return c
    from efs_b200 import opgen
    vv, vi, ii, iv = [c[k].reshape(3, *N) for k in ("vv", "vi", "ii", "iv")]
    # a handful of distinct tuples, so the material table stays small
    q = lambda a: np.round(a * 8) / 8
    mat, mt = opgen.to_indexed(q(vv), q(vi), q(ii), q(iv))
    return dict(mat=mat, table=mt.table())


def member(cls, kind, indexed):
    """Engine of a fixed configuration (kind selects grid and extensions)."""
    g = cls()
    assert g.initGPU()
    r = np.random.default_rng(100 + kind)
    if kind == 0:                         # Mur + lumped-port style excitation + probe ring; Nz odd (padded rows)
        N = (20, 18, 23)
        g.init(N, coeffs(N, 1, indexed))
        g.configureMur(mur_faces(N, 2))
        sig = np.sin(np.arange(60) * 0.3).astype(np.float32)
        pos = [idx(0, 10, 9, 12, *N), idx(0, 10, 9, 12, *N)]          # cell index; dir picks the component
        g.configureExcitation(dict(signal=sig, delay=[0, 4], amp=[1.0, -0.5], dir=[2, 2], pos=pos, period=0))
        g.configureProbeGatherBuffered([idx(2, 10, 9, 12, *N), idx(0, 3, 4, 5, *N)], maxSamples=80, sampleInterval=2)
    elif kind == 1:                       # UPML (overlapping) + TFSF + NF2FF
        N = (16, 13, 20)
        g.init(N, coeffs(N, 3, indexed))
        g.configurePML([pml_region((0, 0, 0), (16, 13, 4), 4), pml_region((0, 0, 16), (16, 13, 4), 5),
                        pml_region((0, 0, 2), (3, 13, 16), 6)])
        t = 3 * N[0] * N[1] * N[2]
        vp = [dict(field_idx=int(r.integers(0, t)), delay_int=int(r.integers(0, 6)), delay_frac=float(r.random()),
                   amp=float(r.standard_normal())) for _ in range(50)]
        cp = [dict(field_idx=int(r.integers(0, t)), delay_int=int(r.integers(0, 6)), delay_frac=float(r.random()),
                   amp=float(r.standard_normal())) for _ in range(30)]
        g.configureTFSF(dict(signal=np.cos(np.arange(40) * 0.4).astype(np.float32), period=0, voltagePoints=vp,
                             currentPoints=cp))
        g.configureNF2FFAccumulation(nf2ff_inputs(N, nfreq=2, inset=5))
    elif kind == 3:                       # dispersive: UPML on all faces, Drude/Lorentz ADE, oblique TFSF, NF2FF
        from efs_b200 import opgen, workloads
        job = workloads.dispersive(grid=(24, 20, 24), pml=3, chunk=8, steps=200, tfsf_inset=6, nf2ff_inset=4, workers=1)
        N = tuple(job["grid"])
        if not indexed:
            vv, vi, ii, iv = opgen.dense_from_indexed(job["coefficients"]["mat"], job["coefficients"]["table"])
            job = dict(job, coefficients=dict(vv=vv, vi=vi, ii=ii, iv=iv))
        from efs_b200.workloads import configure
        configure(g, job)
    elif kind == 4:                       # dense TFSF z faces (added inside the core update) + scattered entries
        N = (10, 14, 70)
        g.init(N, coeffs(N, 9, indexed))
        pt = lambda n, x, y, z: dict(field_idx=idx(n, x, y, z, *N), delay_int=int(r.integers(0, 6)),
                                     delay_frac=float(r.random()), amp=float(r.standard_normal()))
        vp = [pt(n, x, y, z) for z in (30, 64) for x in range(N[0]) for y in range(N[1]) for n in (0, 1)]
        vp += [pt(int(r.integers(0, 3)), int(r.integers(0, N[0])), int(r.integers(0, N[1])), int(r.integers(0, N[2])))
               for _ in range(40)]
        cp = [pt(int(r.integers(0, 3)), int(r.integers(0, N[0])), int(r.integers(0, N[1])), int(r.integers(0, N[2])))
              for _ in range(30)]
        g.configureTFSF(dict(signal=np.sin(np.arange(30) * 0.4).astype(np.float32), period=0, voltagePoints=vp,
                             currentPoints=cp))
    else:                                 # small grid, excitation only; Nz = 7 (padded rows)
        N = (9, 11, 7)
        g.init(N, coeffs(N, 7, indexed))
        g.configureExcitation(dict(signal=np.ones(5, np.float32), delay=[1], amp=[0.7], dir=[1],
                                   pos=[4 * 77 + 5 * 7 + 3], period=3))
    t = 3 * N[0] * N[1] * N[2]
    g.uploadFields(r.standard_normal(t).astype(np.float32), r.standard_normal(t).astype(np.float32))
    return g


def compare(a, b, kind, what):
    fa, fb = a.getFields(), b.getFields()
    assert_bitexact(fa["volt"], fb["volt"], "%s member %d volt" % (what, kind))
    assert_bitexact(fa["curr"], fb["curr"], "%s member %d curr" % (what, kind))
    assert a.numTS == b.numTS
    if kind == 0:
        ra, rb = a.readProbeGatherBuffered(), b.readProbeGatherBuffered()
        assert (ra is None) == (rb is None)          # None until the first sample is due
        if ra is not None:
            assert ra["numSamples"] == rb["numSamples"]
            assert_bitexact(ra["data"], rb["data"], "ring")
    if kind == 3:
        for name in ("ade_volt", "ade_volt_lor", "ade_curr", "ade_curr_lor"):
            assert_bitexact(a.debugRead(name), b.debugRead(name), "%s member 3 %s" % (what, name))
        na, nb = a.readNF2FFAccumulation(True), b.readNF2FFAccumulation(True)
        assert_bitexact(na["accumE"], nb["accumE"], "nf2ff E")
        assert_bitexact(na["accumH"], nb["accumH"], "nf2ff H")
    if kind == 1:
        for r in range(3):
            assert_bitexact(a.debugRead("pml_volt_flux", r), b.debugRead("pml_volt_flux", r), "vflux")
            assert_bitexact(a.debugRead("pml_curr_flux", r), b.debugRead("pml_curr_flux", r), "cflux")
        na, nb = a.readNF2FFAccumulation(True), b.readNF2FFAccumulation(True)
        assert_bitexact(na["accumE"], nb["accumE"], "nf2ff E")
        assert_bitexact(na["accumH"], nb["accumH"], "nf2ff H")


@pytest.mark.parametrize("indexed", [True, False])
def test_batch_members_match_solo_engines(cuda_engine_cls, indexed):
    from efs_b200.engine import CudaBatch
    kinds = (0, 1, 2, 3, 4)
    batched = [member(cuda_engine_cls, k, indexed) for k in kinds]
    solo = [member(cuda_engine_cls, k, indexed) for k in kinds]
    assert sorted(batched[4].debugRead("tfsf_faces")[1:]) == [30, 64]   # faces applied in the batched core
    b = CudaBatch(batched)
    try:
        for n, shape in ((1, None), (17, (4, 1)), (70, (8, 2)), (5, (3, 2))):
            if shape:
                b.setShape(*shape)
            b.iterate(n)
            b.sync()
            for s in solo:
                s.iterate(n)
            for k, a, s in zip(kinds, batched, solo):
                compare(a, s, k, "after +%d" % n)
    finally:
        b.destroy()
        for e in batched + solo:
            e.destroy()


def test_batch_replans_after_solo_steps_and_autotunes(cuda_engine_cls):
    """A member stepped on its own between batch calls (its parity flips) and
    the autotuner's timed steps leave every member equal to its solo twin."""
    from efs_b200.engine import CudaBatch
    kinds = (0, 2)
    batched = [member(cuda_engine_cls, k, True) for k in kinds]
    solo = [member(cuda_engine_cls, k, True) for k in kinds]
    b = CudaBatch(batched)
    try:
        b.iterate(6)
        batched[1].iterate(3)                 # member 1 alone: odd count flips its parity
        b.iterate(9)
        tuned = b.autotune(steps=2)           # 17 * 2 timesteps
        assert tuned["xchunk"] in (8, 16, 32, 64) and tuned["ctas_per_sm"] in (1, 2)
        b.iterate(4)
        b.sync()
        totals = [6 + 9 + 34 + 4, 6 + 3 + 9 + 34 + 4]
        for k, a, s, n in zip(kinds, batched, solo, totals):
            s.iterate(n)
            compare(a, s, k, "replan/autotune")
    finally:
        b.destroy()
        for e in batched + solo:
            e.destroy()


def test_batch_rejects_unsupported_members(cuda_engine_cls):
    from efs_b200.engine import CudaBatch, EfsError
    g = member(cuda_engine_cls, 2, True)
    odd = cuda_engine_cls()
    assert odd.initGPU()
    N = (6, 6, 7)
    odd.init(N, coeffs(N, 9, True))
    odd.configureRLC(dict(elements=[dict(field_idx=idx(0, 2, 2, 2, *N), direction=2, type_flag=0, i2v=0.1, ilv=0.2)]))
    with pytest.raises(EfsError):              # lumped RLC members are not batched
        CudaBatch([g, odd])
    with pytest.raises(EfsError):
        CudaBatch([g, g])
    g.destroy()
    odd.destroy()


@pytest.mark.parametrize("indexed", [False, True])
def test_phase_timing_runs_the_same_steps(cuda_engine_cls, indexed):
    """efs_time_phases / efs_batch_time_phases advance exactly as iterate does
    (kernel by kernel instead of a graph) and report non-negative phase times."""
    from efs_b200.engine import PHASES, CudaBatch
    kinds = (0, 1, 3)
    solo = [member(cuda_engine_cls, k, indexed) for k in kinds]
    timed = [member(cuda_engine_cls, k, indexed) for k in kinds]
    for s, t in zip(solo, timed):
        s.iterate(21)
        ph = t.timePhases(21)
        assert set(ph) == set(PHASES) and all(v >= 0 for v in ph.values()) and ph["core"] > 0
    for k, s, t in zip(kinds, solo, timed):
        compare(s, t, k, "timePhases")
    b = CudaBatch(timed)
    try:
        ph = b.timePhases(13)
        assert set(ph) == set(PHASES) and all(v >= 0 for v in ph.values()) and ph["core"] > 0
        b.sync()
    finally:
        b.destroy()
    for s in solo:
        s.iterate(13)
    for k, s, t in zip(kinds, solo, timed):
        compare(s, t, k, "batch timePhases")
    for e in solo + timed:
        e.destroy()
