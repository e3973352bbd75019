"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

The CUDA kernels evaluate every update with separately rounded f32 multiplies
and adds in the reference's operand order, so against the oracle's f32 mode
the fields, UPML fluxes, Mur/ADE/RLC/steady-state state and the probe ring
must agree BIT FOR BIT.  The NF2FF accumulators agree to 1e-6 relative (the
per-step cosine/sine come from two f64 libraries), the energy to 1e-7 and the
far field to 1e-4 (f32 sums in a different order against an f64 oracle).
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT, free_space, idx
from oracle.oracle import OracleEngine, far_field

pytestmark = pytest.mark.gpu

# Plane depth of the fused kernel (efs_set_plane_depth): the default, and 3
# x-planes per CTA so that CTA seams fall inside the test grids (results must
# not depend on it).
CORES = {
    "fused": None,
    "fused_x3": 3,
}


@pytest.fixture(autouse=True, params=list(CORES))
def core_path(request, monkeypatch):
    depth = CORES[request.param]
    if depth is not None:
        from efs_b200.engine import CudaEngine
        init_gpu = CudaEngine.initGPU

        def initGPU(self, *a, **k):
            ok = init_gpu(self, *a, **k)
            if ok:
                self.setPlaneDepth(depth)
            return ok
        monkeypatch.setattr(CudaEngine, "initGPU", initGPU)
    return request.param


def rand_coeffs(N, seed, pec_frac=0.05):
    Nx, Ny, Nz = N
    t = 3 * Nx * Ny * Nz
    r = np.random.default_rng(seed)
    c = dict(vv=(0.95 + 0.05 * r.random(t)).astype(np.float32), vi=(0.1 + 0.2 * r.random(t)).astype(np.float32),
             ii=(0.97 + 0.03 * r.random(t)).astype(np.float32), iv=(0.1 + 0.2 * r.random(t)).astype(np.float32))
    m = r.random(t) < pec_frac
    c["vv"][m] = 0
    c["vi"][m] = 0
    return c


def both(cuda_cls, N, coeffs, indexed=False):
    g = cuda_cls()
    assert g.initGPU()
    if indexed:
        from efs_b200 import opgen
        vv, vi, ii, iv = [coeffs[k].reshape(3, *N) for k in ("vv", "vi", "ii", "iv")]
        mat, mt = opgen.to_indexed(vv, vi, ii, iv)
        g.init(N, dict(mat=mat, table=mt.table()))
    else:
        g.init(N, coeffs)
    o = OracleEngine(N, coeffs, mode="f32")
    return g, o


def seed_fields(g, o, N, seed):
    r = np.random.default_rng(seed)
    n = 3 * N[0] * N[1] * N[2]
    v = r.standard_normal(n).astype(np.float32)
    c = r.standard_normal(n).astype(np.float32)
    g.uploadFields(v, c)
    o.uploadFields(v, c)


def assert_bitexact(a, b, what):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    assert a.shape == b.shape, what
    bad = np.flatnonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad.size == 0, "%s: %d mismatches, first at %d: %r vs %r" % (what, bad.size, bad[0], a[bad[0]], b[bad[0]])


def compare_fields(g, o, what=""):
    f = g.getFields()
    assert_bitexact(f["volt"], o.volt, what + " volt")
    assert_bitexact(f["curr"], o.curr, what + " curr")


@pytest.mark.parametrize("indexed", [False, True])
@pytest.mark.parametrize("N", [(3, 3, 3), (8, 1, 1), (17, 9, 35), (33, 40, 70), (9, 6, 71), (21, 19, 132)])
def test_core_bitexact(cuda_engine_cls, N, indexed):
    c = rand_coeffs(N, 1) if not indexed else free_space(*N)
    g, o = both(cuda_engine_cls, N, c, indexed)
    seed_fields(g, o, N, 2)
    for steps in (1, 5, 70):
        g.iterate(steps)
        o.iterate(steps)
        compare_fields(g, o, "core %s +%d" % (N, steps))
    assert g.numTS == o.numTS == 76


def test_excitation_and_ring(cuda_engine_cls):
    N = (12, 10, 14)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 3))
    sig = np.sin(np.arange(37) * 0.4).astype(np.float32)
    pos = [5 * 140 + 4 * 14 + 6, 2 * 140 + 3 * 14 + 7, 5 * 140 + 4 * 14 + 6]   # repeated target
    exc = dict(signal=sig, delay=[0, 3, 1], amp=[1.0, -0.7, 0.25], dir=[2, 0, 2], pos=pos, period=0)
    for e in (g, o):
        e.configureExcitation(exc)
    probe = [idx(2, 5, 4, 6, *N), idx(0, 1, 1, 1, *N), idx(1, 11, 9, 13, *N)]
    g.configureProbeGatherBuffered(probe, maxSamples=20, sampleInterval=3)
    o.configureProbeGatherBuffered(probe, 20, 3)
    g.iterate(50)
    o.iterate(50)
    compare_fields(g, o, "excitation")
    rg, ro = g.readProbeGatherBuffered(), o.readProbeGatherBuffered()
    assert rg["numSamples"] == ro["numSamples"] == 16 and rg["stride"] == 6
    assert_bitexact(rg["data"], ro["data"], "ring")
    # periodic excitation, past-end semantics
    g2, o2 = both(cuda_engine_cls, N, rand_coeffs(N, 4))
    exc2 = dict(signal=sig[:9], delay=[2], amp=[0.5], dir=[1], pos=[3 * 140 + 3 * 14 + 3], period=5)
    for e in (g2, o2):
        e.configureExcitation(exc2)
    g2.iterate(23)
    o2.iterate(23)
    compare_fields(g2, o2, "periodic excitation")


def pml_region(start, num, seed):
    r = np.random.default_rng(seed)
    t = 3 * num[0] * num[1] * num[2]
    return dict(startPos=list(start), numLines=list(num),
                vv=(0.8 + 0.2 * r.random(t)).astype(np.float32), vvfo=(0.7 + 0.3 * r.random(t)).astype(np.float32),
                vvfn=(1.0 + 0.3 * r.random(t)).astype(np.float32), ii=(0.8 + 0.2 * r.random(t)).astype(np.float32),
                iifo=(0.7 + 0.3 * r.random(t)).astype(np.float32), iifn=(1.0 + 0.3 * r.random(t)).astype(np.float32))


@pytest.mark.parametrize("overlap", [False, True])
def test_pml_bitexact(cuda_engine_cls, overlap):
    N = (20, 18, 24)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 5))
    regs = [pml_region((0, 0, 0), (20, 18, 4), 6), pml_region((0, 0, 20), (20, 18, 4), 7),
            pml_region((0, 0, 4), (4, 18, 16), 8)]
    if overlap:
        regs.append(pml_region((2, 3, 2), (6, 5, 7), 9))   # overlaps three others
    for e in (g, o):
        e.configurePML(regs)
    seed_fields(g, o, N, 10)
    g.iterate(25)
    o.iterate(25)
    compare_fields(g, o, "pml")
    for r in range(len(regs)):
        assert_bitexact(g.debugRead("pml_volt_flux", r), o.read("pml_volt_flux", r), "vflux %d" % r)
        assert_bitexact(g.debugRead("pml_curr_flux", r), o.read("pml_curr_flux", r), "cflux %d" % r)


# 8-cell z-slab regions are updated inside the fused kernel from TMA-staged flux
# (a slab overlapping other regions keeps its shared cells in the UPML passes)
ZSLAB_CASES = {
    "z_only": ((20, 23, 50), [((0, 0, 0), (20, 23, 8)), ((0, 0, 42), (20, 23, 8))]),
    "six_faces": ((24, 22, 40), [((0, 0, 0), (8, 22, 40)), ((16, 0, 0), (8, 22, 40)), ((0, 0, 0), (24, 8, 40)),
                                 ((0, 14, 0), (24, 8, 40)), ((0, 0, 0), (24, 22, 8)), ((0, 0, 32), (24, 22, 8))]),
    "both_in_one_tile": ((12, 17, 20), [((0, 0, 0), (12, 17, 8)), ((0, 0, 12), (12, 17, 8))]),
    "partial_rows": ((14, 21, 37), [((2, 3, 0), (8, 11, 8)), ((0, 9, 29), (14, 12, 8)), ((5, 0, 10), (6, 21, 8))]),
}


@pytest.mark.parametrize("indexed", [False, True])
@pytest.mark.parametrize("case", list(ZSLAB_CASES))
def test_pml_zslab_bitexact(cuda_engine_cls, case, indexed):
    N, boxes = ZSLAB_CASES[case]
    c = rand_coeffs(N, 21) if not indexed else free_space(*N)
    g, o = both(cuda_engine_cls, N, c, indexed)
    regs = [pml_region(s, n, 60 + i) for i, (s, n) in enumerate(boxes)]
    for e in (g, o):
        e.configurePML(regs)
    seed_fields(g, o, N, 22)
    for steps in (1, 6, 23):
        g.iterate(steps)
        o.iterate(steps)
        compare_fields(g, o, "zslab %s +%d" % (case, steps))
    for r in range(len(regs)):
        assert_bitexact(g.debugRead("pml_volt_flux", r), o.read("pml_volt_flux", r), "vflux %d" % r)
        assert_bitexact(g.debugRead("pml_curr_flux", r), o.read("pml_curr_flux", r), "cflux %d" % r)


def test_pml_dense_coefficients_bitexact(cuda_engine_cls):
    """A UPML region with more distinct coefficient tuples than the compact
    form holds (65,535) keeps its dense arrays; next to a compact region."""
    N = (40, 41, 48)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 50))
    regs = [pml_region((0, 0, 0), (40, 41, 41), 51), pml_region((0, 0, 41), (40, 41, 7), 52)]
    for e in (g, o):
        e.configurePML(regs)
    seed_fields(g, o, N, 53)
    g.iterate(9)
    o.iterate(9)
    compare_fields(g, o, "pml dense")
    for r in range(len(regs)):
        assert_bitexact(g.debugRead("pml_volt_flux", r), o.read("pml_volt_flux", r), "vflux %d" % r)
        assert_bitexact(g.debugRead("pml_curr_flux", r), o.read("pml_curr_flux", r), "cflux %d" % r)


def mur_faces(N, coeff_seed):
    """Dual-component Mur on the x and y faces, with coinciding normals at the corners."""
    Nx, Ny, Nz = N
    r = np.random.default_rng(coeff_seed)
    nP, sP, nPP, sPP = [], [], [], []
    for ny, line, shift in ((0, 0, 1), (0, Nx - 1, Nx - 2), (1, 0, 1), (1, Ny - 1, Ny - 2)):
        P, PP = (ny + 1) % 3, (ny + 2) % 3
        nl = [Nx, Ny, Nz]
        for i1 in range(nl[PP]):
            for i0 in range(nl[P]):
                pos = [0, 0, 0]
                pos[ny], pos[P], pos[PP] = line, i0, i1
                sh = list(pos)
                sh[ny] = shift
                nP.append(idx(P, *pos, *N)); sP.append(idx(P, *sh, *N))
                nPP.append(idx(PP, *pos, *N)); sPP.append(idx(PP, *sh, *N))
    return dict(coeff_nyP=(r.random(len(nP)) * 0.5).astype(np.float32), coeff_nyPP=(r.random(len(nPP)) * 0.5).astype(np.float32),
                normal_idx_nyP=nP, shifted_idx_nyP=sP, normal_idx_nyPP=nPP, shifted_idx_nyPP=sPP)


def test_mur_with_pml_corners_bitexact(cuda_engine_cls):
    N = (14, 12, 20)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 11))
    regs = [pml_region((0, 0, 0), (14, 12, 3), 12), pml_region((0, 0, 17), (14, 12, 3), 13)]
    mur = mur_faces(N, 14)
    for e in (g, o):
        e.configurePML(regs)
        e.configureMur(mur)
    seed_fields(g, o, N, 15)
    g.iterate(30)
    o.iterate(30)
    compare_fields(g, o, "mur")
    assert_bitexact(g.debugRead("mur_saved"), o.read("mur_saved"), "mur_saved")


@pytest.mark.parametrize("N", [(16, 18, 24), (16, 17, 24)])
def test_mur_six_faces_with_sources_bitexact(cuda_engine_cls, N):
    """Mur on all six faces (edge and corner cells carry two entries), an
    excitation and TFSF points inside: on the TMA path the Mur post-update and
    apply run inside the core kernel; Ny = 17 (a y tile would start on the
    y-hi face) keeps them in their own kernels.  Both bit for bit."""
    from efs_b200 import opgen
    mesh = opgen.Mesh(*[opgen.uniform_lines(n, 1e-3) for n in N])
    mur = opgen.mur_dual(mesh, 1.5e-12, [(a, s) for a in range(3) for s in ("lo", "hi")])
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 43))
    sig = np.sin(np.arange(30) * 0.4).astype(np.float32)
    exc = dict(signal=sig, delay=[0, 2], amp=[1.0, 0.5], dir=[2, 1], pos=[idx(0, 8, 9, 12, *N), idx(0, 5, 6, 7, *N)],
               period=0)
    t = 3 * N[0] * N[1] * N[2]
    r = np.random.default_rng(44)
    inner = [idx(int(r.integers(0, 3)), int(r.integers(3, N[0] - 3)), int(r.integers(3, N[1] - 3)),
                 int(r.integers(3, N[2] - 3)), *N) for _ in range(20)]
    vp = [dict(field_idx=f, delay_int=int(r.integers(0, 4)), delay_frac=float(r.random()), amp=float(r.standard_normal()))
          for f in inner]
    cp = [dict(field_idx=int(r.integers(0, t)), delay_int=1, delay_frac=0.5, amp=0.3) for _ in range(10)]
    for e in (g, o):
        e.configureMur(mur)
        e.configureExcitation(exc)
        e.configureTFSF(dict(signal=sig, period=0, voltagePoints=vp, currentPoints=cp))
    seed_fields(g, o, N, 45)
    for n in (1, 30):
        g.iterate(n)
        o.iterate(n)
        compare_fields(g, o, "mur6 +%d" % n)
        assert_bitexact(g.debugRead("mur_saved"), o.read("mur_saved"), "mur_saved")


def test_tfsf_bitexact(cuda_engine_cls):
    N = (10, 11, 12)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 16))
    r = np.random.default_rng(17)
    vp = [dict(field_idx=int(r.integers(0, 3 * 1320)), delay_int=int(r.integers(0, 6)), delay_frac=float(r.random()),
               amp=float(r.standard_normal())) for _ in range(60)]
    vp.append(dict(vp[0]))          # duplicate target, applied in order
    cp = [dict(field_idx=int(r.integers(0, 3 * 1320)), delay_int=int(r.integers(0, 6)), delay_frac=float(r.random()),
               amp=float(r.standard_normal())) for _ in range(40)]
    cfg = dict(signal=np.cos(np.arange(25) * 0.5).astype(np.float32), period=0, voltagePoints=vp, currentPoints=cp)
    for e in (g, o):
        e.configureTFSF(cfg)
    g.iterate(35)
    o.iterate(35)
    compare_fields(g, o, "tfsf")


def test_tfsf_on_tile_seams_bitexact(cuda_engine_cls):
    """TFSF targets on the seams of the core kernel's 64 x 8 (z x y) tiles
    (halo rows, halo columns and their corners), on every x plane (x-chunk
    seams in the small-chunk variants) and inside UPML regions, with repeated
    targets: the H cells next to them are redone after the TFSF pass."""
    N = (13, 20, 136)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 40))
    regs = [pml_region((0, 0, 120), (13, 20, 16), 41), pml_region((0, 14, 0), (13, 6, 120), 42)]
    for e in (g, o):
        e.configurePML(regs)
    r = np.random.default_rng(43)
    ys, zs = [0, 7, 8, 15, 16, 19], [0, 1, 63, 64, 65, 127, 128, 135]

    def pt(seam):
        x = int(r.integers(0, N[0]))
        y = int(r.choice(ys)) if seam else int(r.integers(0, N[1]))
        z = int(r.choice(zs)) if seam else int(r.integers(0, N[2]))
        return dict(field_idx=idx(int(r.integers(0, 3)), x, y, z, *N), delay_int=int(r.integers(0, 8)),
                    delay_frac=float(r.random()), amp=float(r.standard_normal()))
    vp = [pt(True) for _ in range(400)] + [pt(False) for _ in range(100)]
    vp += [dict(vp[i]) for i in range(0, 400, 7)]          # repeated targets, applied in order
    cp = [pt(True) for _ in range(150)]
    cfg = dict(signal=np.sin(np.arange(50) * 0.3).astype(np.float32), period=0, voltagePoints=vp, currentPoints=cp)
    for e in (g, o):
        e.configureTFSF(cfg)
    seed_fields(g, o, N, 44)
    for n in (1, 6, 30):
        g.iterate(n)
        o.iterate(n)
        compare_fields(g, o, "tfsf seams +%d" % n)
    for k in range(len(regs)):
        assert_bitexact(g.debugRead("pml_curr_flux", k), o.read("pml_curr_flux", k), "cflux %d" % k)


@pytest.mark.parametrize("indexed", [False, True])
def test_tfsf_faces_in_core_bitexact(cuda_engine_cls, indexed):
    """Dense Ex/Ey TFSF targets on two z planes (63: last owned column of a
    64-wide tile, 64: its halo column and the next tile's first column) are
    added inside the fused update from a per-step face array; repeated targets
    on those planes, targets of other components and scattered targets stay in
    the point pass, some inside a UPML region."""
    N = (13, 20, 136)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 50) if not indexed else free_space(*N), indexed)
    regs = [pml_region((0, 12, 0), (13, 8, 136), 51)]
    for e in (g, o):
        e.configurePML(regs)
    r = np.random.default_rng(52)
    pt = lambda n, x, y, z: dict(field_idx=idx(n, x, y, z, *N), delay_int=int(r.integers(0, 8)),
                                 delay_frac=float(r.random()), amp=float(r.standard_normal()))
    vp = [pt(n, x, y, z) for z in (63, 64) for x in range(N[0]) for y in range(N[1]) for n in (0, 1)]
    vp += [pt(int(r.integers(0, 3)), int(r.integers(0, N[0])), int(r.integers(0, N[1])), int(r.integers(0, N[2])))
           for _ in range(120)]
    vp += [dict(vp[i]) for i in range(0, len(vp), 37)]     # repeated targets: back to the point pass, in order
    cp = [pt(int(r.integers(0, 3)), int(r.integers(0, N[0])), int(r.integers(0, N[1])), int(r.integers(0, N[2])))
          for _ in range(80)]
    cfg = dict(signal=np.sin(np.arange(40) * 0.35).astype(np.float32), period=0, voltagePoints=vp, currentPoints=cp)
    for e in (g, o):
        e.configureTFSF(cfg)
    assert sorted(g.debugRead("tfsf_faces")[1:]) == [63, 64]
    seed_fields(g, o, N, 53)
    for n in (1, 5, 44):                                  # past the signal's end too (identity adds)
        g.iterate(n)
        o.iterate(n)
        compare_fields(g, o, "tfsf faces +%d" % n)
    assert_bitexact(g.debugRead("pml_curr_flux", 0), o.read("pml_curr_flux", 0), "cflux")


@pytest.mark.parametrize("apply", [False, True])
def test_ade_in_and_out_of_pml_bitexact(cuda_engine_cls, apply):
    """Two orders on the same cells (with the apply step: entries grouped per
    field location, applied in configuration order), both sides, some cells
    inside a UPML slab."""
    N = (12, 10, 16)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 18))
    regs = [pml_region((0, 0, 0), (12, 10, 4), 19)]
    r = np.random.default_rng(20)
    cells = r.choice(12 * 10 * 16, 80, replace=False)   # some inside the UPML slab
    orders = []
    for lor in (False, True):
        dirs = []
        for d in range(3):
            k = len(cells)
            dirs.append(dict(dir=d, pos_idx=cells, v_int_ADE=r.random(k) * 0.9, v_ext_ADE=r.random(k) * 0.3,
                             v_Lor_ADE=r.random(k) * 0.1, i_int_ADE=r.random(k) * 0.9, i_ext_ADE=r.random(k) * 0.3,
                             i_Lor_ADE=r.random(k) * 0.1))
        orders.append(dict(numCells=len(cells), hasLorentz=lor, directions=dirs))
    for e in (g, o):
        e.configurePML(regs)
        e.configureLorentzADE({"orders": orders, "apply": apply})
    seed_fields(g, o, N, 21)
    g.iterate(12)
    o.iterate(12)
    compare_fields(g, o, "ade apply=%s" % apply)
    for name in ("ade_volt", "ade_volt_lor", "ade_curr", "ade_curr_lor"):
        ref = np.concatenate([o.read(name, oi, d) for oi in range(2) for d in range(3)])
        assert_bitexact(g.debugRead(name), ref, name)


def test_ade_apply_runs_bitexact(cuda_engine_cls):
    """Apply step with one entry per field location (entries stored as runs):
    rows of ADE cells crossing a UPML slab, a TFSF point and an excitation on
    ADE cells (their H neighbours are deferred twice over), Drude and Lorentz
    orders on disjoint cells, both sides."""
    N = (14, 11, 23)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 40))
    regs = [pml_region((0, 0, 0), (14, 11, 4), 41)]
    r = np.random.default_rng(42)
    rows = [idx(0, x, y, 0, *N) for x in range(2, 12, 3) for y in range(1, 10, 2)]
    cells = np.unique(np.concatenate([np.arange(c, c + 20) for c in rows]))   # z rows 0..19: runs
    half = len(cells) // 2
    orders = []
    for lor, cl in ((False, cells[:half]), (True, cells[half:])):
        k = len(cl)
        dirs = [dict(dir=d, pos_idx=cl, v_int_ADE=0.5 + 0.4 * r.random(k), v_ext_ADE=0.05 * r.random(k),
                     v_Lor_ADE=0.02 * r.random(k), i_int_ADE=0.5 + 0.4 * r.random(k), i_ext_ADE=0.05 * r.random(k),
                     i_Lor_ADE=0.02 * r.random(k)) for d in range(3)]
        orders.append(dict(numCells=k, hasLorentz=lor, directions=dirs))
    c0 = int(cells[3])
    sig = np.sin(np.arange(30) * 0.5).astype(np.float32)
    tf = dict(signal=sig, period=0, voltagePoints=[dict(field_idx=c0, delay_int=1, delay_frac=0.25, amp=0.7)],
              currentPoints=[dict(field_idx=int(N[0] * N[1] * N[2] + cells[7]), delay_int=0, delay_frac=0.5, amp=0.3)])
    exc = dict(signal=sig, delay=[2], amp=[0.8], dir=[2], pos=[int(cells[10])], period=0)
    for e in (g, o):
        e.configurePML(regs)
        e.configureLorentzADE({"orders": orders, "apply": True})
        e.configureTFSF(tf)
        e.configureExcitation(exc)
    seed_fields(g, o, N, 43)
    for n in (1, 9, 30):
        g.iterate(n)
        o.iterate(n)
        compare_fields(g, o, "ade apply runs +%d" % n)
    for name in ("ade_volt", "ade_volt_lor", "ade_curr", "ade_curr_lor"):
        ref = np.concatenate([o.read(name, oi, d) for oi in range(2) for d in range(3)])
        assert_bitexact(g.debugRead(name), ref, name)


def test_rlc_bitexact(cuda_engine_cls):
    N = (8, 8, 8)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 22))
    r = np.random.default_rng(23)
    els = []
    for k in range(12):
        els.append(dict(field_idx=int(r.integers(0, 512)), direction=int(r.integers(0, 3)), type_flag=int(k % 2),
                        i2v=float(r.random()), ilv=float(r.random() * 0.1), vvd=float(0.5 + 0.4 * r.random()),
                        vv2=float(r.random() * 0.1), vj1=float(r.random() * 0.1), vj2=float(r.random() * 0.1),
                        ib0=float(r.random() * 0.3), b1=float(r.random() * 0.1), b2=float(r.random() * 0.1)))
    els.append(dict(els[1]))        # two series elements on one edge: sequential
    for e in (g, o):
        e.configureRLC(dict(elements=els))
    seed_fields(g, o, N, 24)
    g.iterate(20)
    o.iterate(20)
    compare_fields(g, o, "rlc")
    for name in ("rlc_vdn", "rlc_jn", "rlc_vil"):
        assert_bitexact(g.debugRead(name), o.read(name), name)


def test_steady_state_bitexact(cuda_engine_cls):
    N = (9, 9, 9)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 25))
    probes = [idx(0, 4, 4, 4, *N), idx(2, 3, 5, 2, *N)]
    cfg = dict(probe_idx=probes, periodSamples=4, threshold=1e-3)
    for e in (g, o):
        e.configureSteadyState(cfg)
    seed_fields(g, o, N, 26)
    g.iterate(3)
    o.iterate(3)
    g.setSteadyStateRecording(True)
    o.setSteadyState(True)
    g.iterate(6)
    o.iterate(6)
    g.setSteadyStateRecording(False)
    o.setSteadyState(False)
    g.iterate(2)
    o.iterate(2)
    s = g.readSteadyState()
    assert s["currentSample"] == o.steadyStateSample == 6
    assert_bitexact(s["energy_period1"], o.read("ss_e1"), "ss_e1")
    assert_bitexact(s["energy_period2"], o.read("ss_e2"), "ss_e2")
    assert s["converged"] == o.checkConvergence()


@pytest.mark.parametrize("phase", [0.0, 0.7])
def test_pbc_bitexact(cuda_engine_cls, phase):
    N = (10, 12, 9)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 27, pec_frac=0))
    cfg = dict(axes=[dict(axis=0, phase=phase), dict(axis=2, phase=0.0)])
    for e in (g, o):
        e.configurePBC(cfg)
    seed_fields(g, o, N, 28)
    g.iterate(15)
    o.iterate(15)
    compare_fields(g, o, "pbc")
    if phase:
        assert_bitexact(g.debugRead("pbc_imag"), o.read("pbc_imag"), "pbc_imag")


def nf2ff_inputs(N, lines_delta=1e-3, nfreq=3, inset=2):
    """Points on the six faces of a box `inset` cells inside the grid."""
    Nx, Ny, Nz = N
    lo = [inset] * 3
    hi = [Nx - 1 - inset, Ny - 1 - inset, Nz - 1 - inset]
    pts = []
    for d in range(3):
        for face in (lo[d], hi[d]):
            rng = [range(lo[k], hi[k] + 1) if k != d else [face] for k in range(3)]
            for x in rng[0]:
                for y in rng[1]:
                    for z in rng[2]:
                        pts.append((x, y, z))
    pts = np.asarray(pts, np.uint32)
    el = []
    for n in range(3):
        e = np.full(N[n], lines_delta, np.float32)
        el.append(e)
    dual = []
    for n in range(3):
        d = np.full(N[n], lines_delta, np.float32)
        d[0] = d[-1] = 0.5 * lines_delta
        dual.append(d)
    return dict(surfaceIndices=pts.ravel(), numPoints=len(pts), omegas=[2e10 * (k + 1) for k in range(nfreq)],
                dT=1.5e-12, gridSize=list(N), primalEdgeLens=el, dualEdgeLens=dual, maxTS=400, windowType=0)


@pytest.mark.parametrize("window", [0, 1])
def test_nf2ff_accumulation(cuda_engine_cls, window):
    N = (14, 13, 15)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 29, pec_frac=0))
    cfg = nf2ff_inputs(N)
    cfg["windowType"] = window
    g.configureNF2FFAccumulation(cfg)
    o.configureNF2FFAccumulation(cfg)
    seed_fields(g, o, N, 30)
    g.iterate(40)
    o.iterate(40)
    compare_fields(g, o, "nf2ff fields")
    ag, ao = g.readNF2FFAccumulation(True), o.readNF2FFAccumulation(True)
    for k in ("accumE", "accumH"):
        a, b = np.asarray(ag[k], np.float64), np.asarray(ao[k], np.float64)
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), k


def test_nf2ff_buffered_batches(cuda_engine_cls):
    """Surface samples are buffered and folded into the accumulators every 16th
    step and at each batch's end: irregular iterate() sizes (one spans two
    captured graphs) and 5 frequencies (two register groups) must still match
    the oracle's per-step accumulation after every call."""
    N = (14, 13, 15)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 41, pec_frac=0))
    cfg = nf2ff_inputs(N, nfreq=5)
    g.configureNF2FFAccumulation(cfg)
    o.configureNF2FFAccumulation(cfg)
    seed_fields(g, o, N, 42)
    for n in (1, 17, 70, 16, 5):
        g.iterate(n)
        o.iterate(n)
        ag, ao = g.readNF2FFAccumulation(True), o.readNF2FFAccumulation(True)
        for k in ("accumE", "accumH"):
            a, b = np.asarray(ag[k], np.float64), np.asarray(ao[k], np.float64)
            assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), (n, k)


def test_far_field_against_f64(cuda_engine_cls):
    N = (14, 13, 15)
    g, _ = both(cuda_engine_cls, N, rand_coeffs(N, 31, pec_frac=0))
    cfg = nf2ff_inputs(N, nfreq=2)
    g.configureNF2FFAccumulation(cfg)
    seed_fields(g, _, N, 32)
    g.iterate(30)
    acc = g.readNF2FFAccumulation(True)
    pts = cfg["surfaceIndices"].reshape(-1, 3).astype(np.float64) * 1e-3
    r = np.random.default_rng(33)
    meta = np.zeros((cfg["numPoints"], 8), np.float32)
    meta[:, :3] = pts
    meta[:, 3] = r.integers(0, 3, cfg["numPoints"])
    meta[:, 4] = r.choice([-1.0, 1.0], cfg["numPoints"])
    meta[:, 5] = 1e-6
    theta = np.deg2rad(np.arange(0, 181, 15)).astype(np.float32)
    phi = np.deg2rad(np.arange(0, 361, 20)).astype(np.float32)
    for fi in range(2):
        out = g.computeNF2FFfarField(dict(pointMeta=meta, theta=theta, phi=phi, center=[7e-3, 6e-3, 7e-3],
                                          frequency=cfg["omegas"][fi] / (2 * np.pi), radius=1.0,
                                          numPoints=cfg["numPoints"], freqIndex=fi)).reshape(-1, 5)
        ref = far_field(acc["accumE"][fi], acc["accumH"][fi], meta, theta, phi, cfg["omegas"][fi] / (2 * np.pi),
                        1.0, (7e-3, 6e-3, 7e-3))
        scale = np.abs(ref[:, 1:]).max()
        assert np.abs(out[:, 1:] - ref[:, 1:]).max() <= 1e-4 * scale
        assert np.abs(out[:, 0] - ref[:, 0]).max() <= 2e-4 * ref[:, 0].max()


def test_energy_and_lag(cuda_engine_cls):
    N = (11, 12, 13)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 34))
    seed_fields(g, o, N, 35)
    assert g.computeEnergy() == 0.0          # first lagged call returns 0 (:2995-3020)
    e0 = o.energy()
    g.iterate(4)
    o.iterate(4)
    assert abs(g.computeEnergy() - e0) <= 1e-7 * e0   # f32 per-cell partials vs f64 (reference bar: 1e-4)
    e1 = o.energy()
    assert abs(g.flushEnergy() - e1) <= 1e-7 * e1
    assert abs(g.computeEnergy(lagged=False) - e1) <= 1e-7 * e1


def test_state_roundtrip(cuda_engine_cls):
    N = (10, 9, 12)
    g, o = both(cuda_engine_cls, N, rand_coeffs(N, 36))
    regs = [pml_region((0, 0, 0), (10, 9, 3), 37)]
    g.configurePML(regs)
    g.configureNF2FFAccumulation(nf2ff_inputs(N, nfreq=1))
    seed_fields(g, o, N, 38)
    g.iterate(7)
    blob = g.getState()
    f7 = g.getFields()
    g.iterate(5)
    f12 = g.getFields()
    g.setState(blob)
    assert g.numTS == 7
    assert_bitexact(g.getFields()["volt"], f7["volt"], "restored")
    g.iterate(5)
    assert_bitexact(g.getFields()["curr"], f12["curr"], "replayed")


def test_invalid_inputs_raise(cuda_engine_cls):
    from efs_b200.engine import EfsError
    g = cuda_engine_cls()
    assert g.initGPU()
    with pytest.raises(EfsError):
        g.iterate(1)                      # before init: EFS_ERR_STATE
    N = (4, 4, 4)
    g.init(N, free_space(*N))
    with pytest.raises(EfsError):
        g.configureExcitation(dict(signal=[1.0], delay=[0], amp=[1.0], dir=[3], pos=[0], period=0))
    with pytest.raises(EfsError):
        g.configureMur(dict(coeff=0.1, normal_idx=[3 * 64], shifted_idx=[0]))
    with pytest.raises(EfsError):
        g.configurePML([pml_region((2, 0, 0), (3, 4, 4), 1)])
    g.iterate(2)                          # engine still usable
    assert g.numTS == 2
    mat = np.zeros(4 * 4 * 4, np.uint32)
    mat[10] = 2
    with pytest.raises(EfsError):
        g.init(N, dict(mat=mat, table=np.ones((2, 12), np.float32)))     # index 2 of a 2-row table
    with pytest.raises(EfsError):
        g.iterate(1)                      # a failed init leaves the engine uninitialised
    mat[10] = 1
    g.init(N, dict(mat=mat, table=np.full((2, 12), 0.5, np.float32)))
    g.iterate(2)
    assert g.numTS == 2
    g.destroy()


def test_openems_cavity_fixture_on_gpu(cuda_engine_cls):
    """Native-openEMS engine_comparison cavity (tests/fixtures/engine_comparison,
    16x8x18 PEC box, 500 steps) reproduced by the CUDA engine: relative L2 of
    the probe voltage < 1e-4."""
    from efs_b200 import workloads
    job = workloads.openems_cavity()
    ref = np.load(os.path.join(ROOT, "tests", "golden", "openems_cavity_vp.npy"))
    g = cuda_engine_cls()
    assert g.initGPU()
    v = workloads.run_probe_job(g, job)
    err = np.linalg.norm(v - ref) / np.linalg.norm(ref)
    assert err < 1e-4, err


def test_openems_cavity_modes_fixture_on_gpu(cuda_engine_cls):
    """Native-openEMS cavity-resonator fixture (tests/fixtures/cavity, 26x11x32
    PEC box, 20000 steps, 6667 probe samples) reproduced by the CUDA engine:
    relative L2 of the probe voltage < 1e-4, and bit for bit the oracle's f32
    series."""
    from efs_b200 import workloads
    g_ = np.load(os.path.join(ROOT, "tests", "golden", "openems_cavity_modes.npz"))
    job = workloads.openems_cavity_modes()
    g = cuda_engine_cls()
    assert g.initGPU()
    v = workloads.run_probe_job(g, job)
    err = np.linalg.norm(v - g_["voltage"]) / np.linalg.norm(g_["voltage"])
    assert err < 1e-4, err
    vo = workloads.run_probe_job(OracleEngine(job["grid"], job["coefficients"], mode="f32"), job)
    assert_bitexact(v.astype(np.float32), vo.astype(np.float32), "cavity modes probe")
    g.destroy()


@pytest.mark.parametrize("apply", [True, False])
def test_dispersive_small_bitexact(cuda_engine_cls, apply):
    """The dispersive workload at a small size: UPML on all faces, Drude and
    Lorentz ADE on the voltage side (the current side has all-zero
    coefficients and its kernel is skipped), TFSF at 30 degrees, NF2FF with 5
    frequencies; with the apply step (the default) and in the reference's
    state-only form."""
    from efs_b200 import workloads
    job = workloads.dispersive(grid=(48, 40, 32), pml=4, chunk=8, steps=200, tfsf_inset=8, nf2ff_inset=6, workers=1,
                               apply=apply)
    g = cuda_engine_cls()
    assert g.initGPU()
    o = OracleEngine(mode="f32")
    workloads.configure(g, job)
    workloads.configure(o, job)
    for n in (1, 40):
        g.iterate(n)
        o.iterate(n)
        compare_fields(g, o, "dispersive +%d" % n)
    for name in ("ade_volt", "ade_volt_lor", "ade_curr", "ade_curr_lor"):
        ref = np.concatenate([o.read(name, oi, d) for oi in range(2) for d in range(3)])
        assert_bitexact(g.debugRead(name), ref, name)
    assert np.abs(np.asarray(g.debugRead("ade_volt"))).max() > 0
    ag, ao = g.readNF2FFAccumulation(True), o.readNF2FFAccumulation(True)
    for k in ("accumE", "accumH"):
        a, b = np.asarray(ag[k], np.float64), np.asarray(ao[k], np.float64)
        assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), k
    # A restored state may hold non-zero values on the zero-coefficient side:
    # the next step must run that side again, which sets them back to 0.
    blob = bytearray(np.asarray(g.getState(), np.uint8).tobytes())
    pos, nb = 32, []
    while pos < len(blob):
        n = int(np.frombuffer(blob, np.uint64, 1, pos)[0])
        nb.append((pos + 8, n))
        pos += 8 + n
    off, n = nb[-4]                     # ..., ADE curr state, ADE curr lor, NF2FF E, NF2FF H
    assert n == 4 * 3 * sum(od["numCells"] for od in job["ade"]["orders"])
    blob[off:off + n] = np.ones(n // 4, np.float32).tobytes()
    g.setState(np.frombuffer(bytes(blob), np.uint8))
    assert np.all(np.asarray(g.debugRead("ade_curr")) == 1)
    g.iterate(1)
    o.iterate(1)
    compare_fields(g, o, "dispersive after restore")
    assert np.all(np.asarray(g.debugRead("ade_curr")).view(np.uint32) == 0)
    g.destroy()
