"""Known-answer tests of the reference's CPU engine, ported to the oracle.

Each test restates a section of tests/test_webgpu.mjs (line numbers cited) and
runs in all three arithmetic modes of the oracle (f32 = the CUDA engine's
order, js = the reference CPUFDTDEngine's f64-intermediate / f32-storage
arithmetic, f64).  These pin the oracle before it is used to check the CUDA
engine.
"""
import math

import numpy as np
import pytest

from conftest import free_space, idx
from oracle.oracle import OracleEngine

MODES = ["f32", "js", "f64"]


def eng(N, mode, coeffs=None):
    Nx, Ny, Nz = N
    return OracleEngine(N, coeffs or free_space(Nx, Ny, Nz), mode=mode)


@pytest.mark.parametrize("mode", MODES)
def test_indexing(mode):  # :395-437
    e = eng((5, 4, 3), mode)
    assert e.idx(0, 0, 0, 0) == 0
    assert e.idx(1, 0, 0, 0) == 5 * 4 * 3
    assert e.idx(0, 1, 0, 0) == 12 and e.idx(0, 0, 1, 0) == 3 and e.idx(0, 0, 0, 1) == 1
    assert idx(2, 4, 3, 2, 5, 4, 3) == 3 * 60 - 1


@pytest.mark.parametrize("mode", MODES)
def test_voltage_boundary_self_reference(mode):  # :443-489
    N = (3, 3, 3)
    e = eng(N, mode)
    curr = np.zeros(3 * 27)
    for n in range(3):
        for x in range(3):
            for y in range(3):
                for z in range(3):
                    curr[idx(n, x, y, z, *N)] = (n + 1) * 0.1 * (x + y + z + 1)
    e.write("curr", curr)
    e.updateVoltages()
    v = e.volt
    assert abs(v[idx(0, 0, 0, 0, *N)]) < 1e-10
    c = np.float32(curr)
    curl = c[idx(2, 1, 1, 1, *N)] - c[idx(2, 1, 0, 1, *N)] - c[idx(1, 1, 1, 1, *N)] + c[idx(1, 1, 1, 0, *N)]
    assert abs(v[idx(0, 1, 1, 1, *N)] - 0.3 * curl) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_current_loop_bounds(mode):  # :495-561
    N = (4, 4, 4)
    e = eng(N, mode)
    volt = np.zeros(3 * 64)
    for n in range(3):
        for x in range(4):
            for y in range(4):
                for z in range(4):
                    volt[idx(n, x, y, z, *N)] = n * 0.1 + x * 0.01 + y * 0.001 + z * 0.0001
    e.write("volt", volt)
    e.updateCurrents()
    c = e.curr
    for x in range(4):
        for n in range(3):
            assert c[idx(n, x, 3, 0, *N)] == 0 and c[idx(n, x, 0, 3, *N)] == 0
    ez11, ez21 = 0.2 + 0.01 + 0.001 + 0.0001, 0.2 + 0.01 + 0.002 + 0.0001
    ey11, ey12 = 0.1 + 0.01 + 0.001 + 0.0001, 0.1 + 0.01 + 0.001 + 0.0002
    assert abs(c[idx(0, 1, 1, 1, *N)] - 0.3 * (ez11 - ez21 - ey11 + ey12)) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_full_timestep_values(mode):  # :567-631
    N = (8, 8, 8)
    e = eng(N, mode)
    e.set("volt", idx(0, 4, 4, 4, *N), 1.0)
    e.updateVoltages()
    e.updateCurrents()
    e.numTS = 1
    assert abs(e.volt[idx(0, 4, 4, 4, *N)] - 1.0) < 1e-6
    assert abs(e.curr[idx(1, 4, 4, 4, *N)] - 0.3) < 1e-6
    assert abs(e.curr[idx(2, 4, 4, 4, *N)] + 0.3) < 1e-6
    for _ in range(3):
        e.updateVoltages()
        e.updateCurrents()
    ex = e.volt[:512]
    assert np.count_nonzero(np.abs(ex) > 1e-10) > 1


@pytest.mark.parametrize("mode", MODES)
def test_excitation_injection(mode):  # :637-675 (C++ past-end semantics)
    N = (5, 5, 5)
    e = eng(N, mode)
    e.configureExcitation(dict(signal=[1.0, 0.5, 0.25, 0.125], delay=[0], amp=[2.0], dir=[0],
                               pos=[2 * 25 + 2 * 5 + 2], period=0))
    g = idx(0, 2, 2, 2, *N)
    e.applyExcitation()
    assert abs(e.volt[g] - 2.0) < 1e-6
    e.write("volt", np.zeros(375))
    e.numTS = 2
    e.applyExcitation()
    assert abs(e.volt[g] - 0.5) < 1e-6
    e.write("volt", np.zeros(375))
    e.numTS = 10
    e.applyExcitation()
    assert abs(e.volt[g] - 2.0) < 1e-6   # beyond the end: amp * signal[0]


@pytest.mark.parametrize("mode", MODES)
def test_excitation_delay(mode):  # :681-710
    N = (5, 5, 5)
    e = eng(N, mode)
    e.configureExcitation(dict(signal=[1.0, 2.0, 3.0, 4.0, 5.0], delay=[3], amp=[1.0], dir=[1],
                               pos=[25 + 5 + 1], period=0))
    g = idx(1, 1, 1, 1, *N)
    e.numTS = 3
    e.applyExcitation()
    assert abs(e.volt[g] - 1.0) < 1e-6
    e.write("volt", np.zeros(375))
    e.numTS = 1
    e.applyExcitation()
    assert abs(e.volt[g] - 1.0) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_multistep_with_excitation(mode):  # :716-756
    N = (10, 10, 10)
    e = eng(N, mode)
    sig = [math.exp(-(((i - 25) / 5) ** 2)) for i in range(50)]
    e.configureExcitation(dict(signal=sig, delay=[0], amp=[1.0], dir=[2], pos=[5 * 100 + 5 * 10 + 5], period=0))
    e.iterate(20)
    assert e.numTS == 20
    assert np.abs(e.volt).max() > 0.01 and np.abs(e.curr).max() > 0.01


@pytest.mark.parametrize("mode", MODES)
def test_pec_boundary(mode):  # :762-804
    N = (6, 6, 6)
    c = free_space(*N)
    for n in range(3):
        for y in range(6):
            for z in range(6):
                i = idx(n, 0, y, z, *N)
                c["vv"][i] = 0
                c["vi"][i] = 0
    e = eng(N, mode, c)
    e.set("volt", idx(0, 3, 3, 3, *N), 1.0)
    e.iterate(5)
    v = e.volt.reshape(3, 6, 6, 6)
    assert np.abs(v[:, 0]).max() < 1e-10


@pytest.mark.parametrize("mode", MODES)
def test_energy_bounded(mode):  # :810-858
    N = (10, 10, 10)
    e = eng(N, mode)
    e.set("volt", idx(0, 5, 5, 5, *N), 1.0)
    es = []
    for _ in range(3):
        e.step()
        es.append(float((e.volt ** 2).sum() + (e.curr ** 2).sum()))
    assert es[1] > 0 and es[2] > 0
    assert max(es[1] / es[0], es[2] / es[1]) < 2.0


@pytest.mark.parametrize("mode", MODES)
def test_determinism(mode):  # :1043-1073
    N = (7, 6, 5)
    rng = np.random.default_rng(0)
    out = []
    for _ in range(2):
        e = eng(N, mode)
        e.write("volt", np.random.default_rng(1).standard_normal(3 * 210))
        e.iterate(7)
        out.append((e.volt, e.curr))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    del rng


@pytest.mark.parametrize("mode", MODES)
def test_pml_pre_post_voltage(mode):  # :1165-1242
    N = (8, 1, 1)
    e = eng(N, mode)
    t = 3 * 3
    e.configurePML([dict(startPos=[0, 0, 0], numLines=[3, 1, 1], vv=np.full(t, 0.8), vvfo=np.full(t, 0.2),
                         vvfn=np.full(t, 1.5), ii=np.full(t, 0.9), iifo=np.full(t, 0.1), iifn=np.full(t, 1.3))])
    g = idx(0, 1, 0, 0, *N)
    p = idx(0, 1, 0, 0, 3, 1, 1)
    e.set("volt", g, 2.0)
    e.set("pml_volt_flux", p, 0.5)
    e.preVoltageUpdatePML()
    assert abs(e.volt[g] - 0.5) < 1e-6 and abs(e.read("pml_volt_flux")[p] - 1.5) < 1e-6
    e.updateVoltages()
    e.postVoltageUpdatePML()
    assert abs(e.read("pml_volt_flux")[p] - 0.5) < 1e-6 and abs(e.volt[g] - 2.25) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_pml_pre_post_current(mode):  # :1244-1300
    N = (8, 2, 2)
    e = eng(N, mode)
    t = 3 * 3 * 2 * 2
    e.configurePML([dict(startPos=[0, 0, 0], numLines=[3, 2, 2], vv=np.ones(t), vvfo=np.zeros(t), vvfn=np.ones(t),
                         ii=np.full(t, 0.7), iifo=np.full(t, 0.3), iifn=np.full(t, 1.2))])
    g = idx(0, 1, 0, 0, *N)
    p = idx(0, 1, 0, 0, 3, 2, 2)
    e.set("curr", g, 3.0)
    e.set("pml_curr_flux", p, 0.4)
    e.preCurrentUpdatePML()
    assert abs(e.curr[g] - 0.4) < 1e-6 and abs(e.read("pml_curr_flux")[p] - 1.98) < 1e-6
    e.set("curr", g, 0.6)
    e.postCurrentUpdatePML()
    assert abs(e.read("pml_curr_flux")[p] - 0.6) < 1e-6 and abs(e.curr[g] - 2.7) < 1e-6


def _ade(N, mode, orders):
    e = eng(N, mode)
    e.configureLorentz({"orders": orders})
    return e


@pytest.mark.parametrize("mode", MODES)
def test_ade_drude(mode):  # :1921-1958
    N = (4, 4, 4)
    e = _ade(N, mode, [dict(numCells=1, hasLorentz=False, directions=[dict(
        dir=0, pos_idx=[16 + 4 + 1], v_int_ADE=[0.8], v_ext_ADE=[0.3], v_Lor_ADE=[0.0])])])
    e.set("volt", idx(0, 1, 1, 1, *N), 2.0)
    e.updateVoltADE()
    assert abs(e.read("ade_volt")[0] - 0.6) < 1e-7
    e.updateVoltADE()
    assert abs(e.read("ade_volt")[0] - (0.8 * 0.6 + 0.6)) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_ade_lorentz(mode):  # :1960-2003
    N = (4, 4, 4)
    e = _ade(N, mode, [dict(numCells=1, hasLorentz=True, directions=[dict(
        dir=0, pos_idx=[16 + 4 + 1], v_int_ADE=[0.9], v_ext_ADE=[0.2], v_Lor_ADE=[0.1])])])
    e.set("volt", idx(0, 1, 1, 1, *N), 3.0)
    e.updateVoltADE()
    assert abs(e.read("ade_volt_lor")[0]) < 1e-7 and abs(e.read("ade_volt")[0] - 0.6) < 1e-7
    e.updateVoltADE()
    assert abs(e.read("ade_volt_lor")[0] - 0.06) < 1e-7
    assert abs(e.read("ade_volt")[0] - (0.9 * 0.6 + 0.2 * (3.0 - 0.06))) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_ade_multiple_orders_and_zero(mode):  # :2005-2080
    N = (4, 4, 4)
    lp = 16 + 4 + 1
    e = _ade(N, mode, [
        dict(numCells=1, hasLorentz=False, directions=[dict(dir=0, pos_idx=[lp], v_int_ADE=[0.5], v_ext_ADE=[0.4])]),
        dict(numCells=1, hasLorentz=False, directions=[dict(dir=0, pos_idx=[lp], v_int_ADE=[0.7], v_ext_ADE=[0.2])])])
    e.set("volt", idx(0, 1, 1, 1, *N), 1.0)
    e.updateVoltADE()
    assert abs(e.read("ade_volt", 0, 0)[0] - 0.4) < 1e-7 and abs(e.read("ade_volt", 1, 0)[0] - 0.2) < 1e-7
    z = _ade(N, mode, [dict(numCells=1, hasLorentz=False, directions=[dict(
        dir=0, pos_idx=[lp], v_int_ADE=[0.0], v_ext_ADE=[0.0], v_Lor_ADE=[0.0])])])
    z.set("volt", idx(0, 1, 1, 1, *N), 5.0)
    z.updateVoltADE()
    assert abs(z.read("ade_volt")[0]) < 1e-10


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("case", [
    # signal, period, numTS, point(field comp, xyz), delay_int, frac, amp, expected  (:2081-2197)
    ([1, 2, 3, 4, 5], 0, 0, (0, 1, 1, 1), 0, 0.0, 0.5, 0.5),
    ([0, 1, 2, 3, 4], 0, 3, (1, 2, 2, 2), 1, 0.25, 1.0, 2.25),
    ([1, 2, 3], 0, 10, (0, 1, 1, 1), 0, 0.0, 1.0, 0.0),
    ([10, 20, 30, 40, 50], 3, 5, (0, 1, 1, 1), 0, 0.0, 1.0, 30.0),
])
def test_tfsf_injection(mode, case):
    sig, period, ts, pt, dint, frac, amp, expect = case
    N = (4, 4, 4)
    e = eng(N, mode)
    fi = idx(*pt, *N)
    e.configureTFSF(dict(signal=sig, period=period, voltagePoints=[dict(field_idx=fi, delay_int=dint, delay_frac=frac, amp=amp)]))
    e.numTS = ts
    e.applyTFSFVoltage()
    assert abs(e.volt[fi] - expect) < 1e-6


def _rlc(**kw):
    base = dict(i2v=0, ilv=0, vvd=0, vv2=0, vj1=0, vj2=0, ib0=0, b1=0, b2=0)
    base.update(kw)
    return base


@pytest.mark.parametrize("mode", MODES)
def test_rlc_parallel_series_history_mixed(mode):  # :2199-2358
    N = (4, 4, 4)
    lp = 16 + 4 + 1
    g = idx(0, 1, 1, 1, *N)
    e = eng(N, mode)
    e.set("volt", g, 5.0)
    e.configureRLC(dict(elements=[_rlc(field_idx=lp, direction=0, type_flag=0, i2v=0.1, ilv=0.2)]))
    e.updateRLC()
    assert abs(e.read("rlc_vil")[0]) < 1e-10
    e.updateRLC()
    assert abs(e.read("rlc_vil")[0] - 0.1 * 0.2 * 5.0) < 1e-7

    s = eng(N, mode)
    s.set("volt", g, 2.0)
    s.configureRLC(dict(elements=[_rlc(field_idx=lp, direction=0, type_flag=1, vvd=0.5, vv2=0.1, ib0=0.3)]))
    s.updateRLC()
    assert abs(s.volt[g] - 1.0) < 1e-7 and abs(s.read("rlc_jn")[0] - 0.3) < 1e-7

    h = eng(N, mode)
    h.configureRLC(dict(elements=[_rlc(field_idx=0, direction=0, type_flag=0)]))
    for k, v in enumerate((1.0, 2.0, 3.0)):
        h.set("volt", 0, v)
        h.updateRLC()
    assert list(h.read("rlc_vdn")) == [3.0, 2.0, 1.0]

    m = eng(N, mode)
    m.set("volt", 0, 1.0)
    m.set("volt", 1, 2.0)
    m.configureRLC(dict(elements=[_rlc(field_idx=0, direction=0, type_flag=0, i2v=0.5, ilv=0.3),
                                  _rlc(field_idx=1, direction=0, type_flag=1, vvd=0.8, ib0=0.4)]))
    m.updateRLC()
    assert abs(m.read("rlc_vil")[0]) < 1e-10 and abs(m.volt[1] - 1.6) < 1e-7


@pytest.mark.parametrize("mode", MODES)
def test_mur_three_phase(mode):  # :2360-2394, :2420-2462
    N = (6, 4, 4)
    e = eng(N, mode)
    n_, s_ = idx(0, 0, 1, 1, *N), idx(0, 1, 1, 1, *N)
    e.set("volt", n_, 1.0)
    e.set("volt", s_, 2.0)
    e.configureMur(dict(coeff=0.3, normal_idx=[n_], shifted_idx=[s_]))
    e.murPreVoltage()
    assert abs(e.read("mur_saved")[0] - 1.7) < 1e-7
    e.set("volt", s_, 3.5)
    e.murPostVoltage()
    assert abs(e.read("mur_saved")[0] - (1.7 + 0.3 * 3.5)) < 1e-7
    e.murApply()
    assert abs(e.volt[n_] - (1.7 + 0.3 * 3.5)) < 1e-7


def test_mur_coefficient():  # :2396-2418
    c, dT, d = 3e8, 1e-12, 1e-4
    assert abs((c * dT - d) / (c * dT + d) - 0.5) < 1e-10


@pytest.mark.parametrize("mode", MODES)
def test_mur_dual_component(mode):  # :2464-2527
    N = (6, 6, 6)
    e = eng(N, mode)
    nP, sP = idx(1, 0, 2, 2, *N), idx(1, 1, 2, 2, *N)
    nPP, sPP = idx(2, 0, 2, 2, *N), idx(2, 1, 2, 2, *N)
    for i, v in ((nP, 1.0), (sP, 2.0), (nPP, 3.0), (sPP, 4.0)):
        e.set("volt", i, v)
    e.configureMur(dict(coeff_nyP=[0.3], coeff_nyPP=[0.5], normal_idx_nyP=[nP], shifted_idx_nyP=[sP],
                        normal_idx_nyPP=[nPP], shifted_idx_nyPP=[sPP]))
    e.murPreVoltage()
    s = e.read("mur_saved")
    assert abs(s[0] - 1.7) < 1e-7 and abs(s[1] - 2.5) < 1e-7
    e.set("volt", sP, 5.0)
    e.set("volt", sPP, 6.0)
    e.murPostVoltage()
    e.murApply()
    assert abs(e.volt[nP] - (1.7 + 1.5)) < 1e-6 and abs(e.volt[nPP] - (2.5 + 3.0)) < 1e-6


@pytest.mark.parametrize("mode", MODES)
def test_steady_state(mode):  # :2566-2673
    N = (4, 4, 4)
    p = idx(0, 1, 1, 1, *N)
    e = eng(N, mode)
    e.set("volt", p, 3.0)
    e.configureSteadyState(dict(probe_idx=[p], periodSamples=5, threshold=1e-6))
    e.setSteadyState(True, 0)
    e.accumulateEnergy()
    assert abs(e.read("ss_e1")[0] - 9.0) < 1e-7 and e.read("ss_e2")[0] == 0
    f = eng(N, mode)
    f.set("volt", p, 2.0)
    f.configureSteadyState(dict(probe_idx=[p], periodSamples=3, threshold=1e-6))
    f.setSteadyState(True, 3)
    f.accumulateEnergy()
    assert abs(f.read("ss_e2")[0] - 4.0) < 1e-7 and f.read("ss_e1")[0] == 0
    c = eng(N, mode)
    c.configureSteadyState(dict(probe_idx=[p], periodSamples=2, threshold=1e-3))
    c.write("ss_e1", [100.0])
    c.write("ss_e2", [100.00005])
    c.setSteadyState(True, 4)
    assert c.checkConvergence() is True
    c.write("ss_e2", [110.0])
    assert c.checkConvergence() is False
    r = eng(N, mode)
    r.set("volt", p, 100.0)
    r.configureSteadyState(dict(probe_idx=[p], periodSamples=5, threshold=1e-6))
    r.accumulateEnergy()
    assert r.read("ss_e1")[0] == 0 and r.read("ss_e2")[0] == 0


def test_modes_agree_closely():
    """f32 (CUDA order) and js (reference CPU) arithmetic differ by rounding only."""
    N = (9, 8, 7)
    rng = np.random.default_rng(3)
    c = free_space(*N)
    c["vi"] = (0.2 + 0.1 * rng.random(c["vi"].size)).astype(np.float32)
    out = {}
    for m in MODES:
        e = eng(N, m, c)
        e.configureExcitation(dict(signal=np.sin(np.arange(40) * 0.3), delay=[0, 2], amp=[1.0, -0.5], dir=[0, 2],
                                   pos=[4 * 56 + 4 * 7 + 3, 2 * 56 + 3 * 7 + 4], period=0))
        e.iterate(30)
        out[m] = e.volt
    scale = np.abs(out["f64"]).max()
    assert np.abs(out["f32"] - out["f64"]).max() < 1e-5 * scale
    assert np.abs(out["js"] - out["f64"]).max() < 1e-5 * scale


def test_far_field_infinitesimal_dipole():  # tests/test_api.mjs:1694-1786
    """The reference's NF2FF known answer: an x-directed surface current
    Js = 1 (Hy = -1 on a z-normal face, 3 x 3 points 1 mm apart) at 1 GHz.
    Its far field is an x dipole: P(theta = pi/2, phi = 0) / P(0, 0) < 0.05,
    and the directivity from angular integration of P_rad over a 91 x 73
    grid is 1.5 within 10 % (measured 1.490; the null ratio 2e-15).  Checks
    the oracle's far-field projections (the f64 reference the CUDA far field
    is compared with)."""
    from oracle.oracle import far_field
    xs = [-0.001, 0.0, 0.001]
    pts = [(x, y) for x in xs for y in xs]
    meta = np.zeros((len(pts), 8), np.float32)
    accE = np.zeros((len(pts), 6), np.float32)
    accH = np.zeros((len(pts), 6), np.float32)
    for i, (x, y) in enumerate(pts):
        meta[i] = (x, y, 0.0, 2, 1.0, 1e-6, 0, 0)        # position, normal z, sign +, area
        accH[i, 2] = -1.0                                 # Hy (re) = -Js0 -> Js_x = Js0
    nt, nph = 91, 73
    theta = np.arange(nt) * math.pi / (nt - 1)
    phi = np.arange(nph) * 2 * math.pi / (nph - 1)
    out = far_field(accE.ravel(), accH.ravel(), meta.ravel(), theta, phi, 1e9)
    P = out[:, 0].reshape(nt, nph)
    assert P.max() > 0
    assert P[nt // 2, 0] / P[0, 0] < 0.05
    prad = (P * np.sin(theta)[:, None]).sum() * (math.pi / (nt - 1)) * (2 * math.pi / (nph - 1))
    dmax = 4 * math.pi * P.max() / prad
    assert abs(dmax - 1.5) / 1.5 < 0.10, dmax


# order of the reference's timestep (tests/test_webgpu.mjs:2675-2776)
STEP_ORDER = ["accumulateEnergy", "preVoltageUpdatePML", "updateVoltADE", "murPreVoltage", "preVoltageRLC",
              "updateVoltages", "postVoltageUpdatePML", "applyTFSFVoltage", "murPostVoltage", "applyExcitation",
              "murApply", "applyRLC", "preCurrentUpdatePML", "updateCurrADE", "updateCurrents",
              "postCurrentUpdatePML", "applyTFSFCurrent"]


def _all_extensions(N, seed=11):
    """f32 oracle with every extension, their targets overlapping: UPML slab
    z = 0..1, Lorentz ADE on UPML and interior cells, Mur on the z = Nz-1 face,
    excitation, TFSF and RLC on Mur and UPML cells, a steady-state probe in
    the UPML slab; random fields."""
    r = np.random.default_rng(seed)
    Nx, Ny, Nz = N
    e = OracleEngine(N, free_space(*N), mode="f32")
    cell = lambda x, y, z: x * Ny * Nz + y * Nz + z
    t = 3 * Nx * Ny * 2
    u = lambda lo, hi: r.uniform(lo, hi, t)
    e.configurePML([dict(startPos=[0, 0, 0], numLines=[Nx, Ny, 2], vv=u(0.6, 1.0), vvfo=u(0.0, 0.3), vvfn=u(0.8, 1.2),
                         ii=u(0.6, 1.0), iifo=u(0.0, 0.3), iifn=u(0.8, 1.2))])
    lp = [cell(2, 2, 1), cell(3, 2, 3), cell(2, 3, Nz - 1)]
    e.configureLorentz({"orders": [dict(numCells=len(lp), hasLorentz=True, directions=[dict(
        dir=n, pos_idx=lp, v_int_ADE=[0.9, 0.8, 0.7], v_ext_ADE=[0.2, 0.1, 0.3], v_Lor_ADE=[0.1, 0.2, 0.05],
        i_int_ADE=[0.85, 0.9, 0.6], i_ext_ADE=[0.1, 0.2, 0.1], i_Lor_ADE=[0.05, 0.1, 0.2]) for n in range(3)])]})
    normal = [n * Nx * Ny * Nz + cell(x, y, Nz - 1) for n in (0, 1) for x in range(Nx) for y in range(Ny)]
    shifted = [n * Nx * Ny * Nz + cell(x, y, Nz - 2) for n in (0, 1) for x in range(Nx) for y in range(Ny)]
    e.configureMur(dict(coeff=0.3, normal_idx=normal, shifted_idx=shifted))
    e.configureExcitation(dict(signal=(0.5 + np.sin(np.arange(8) * 0.7)).astype(np.float32), delay=[0, 1], amp=[0.7, -0.4],
                               dir=[0, 2], pos=[cell(2, 3, Nz - 1), cell(3, 3, 1)], period=0))
    vp = [dict(field_idx=0 * Nx * Ny * Nz + cell(2, 3, Nz - 1), delay_int=0, delay_frac=0.25, amp=0.5),
          dict(field_idx=1 * Nx * Ny * Nz + cell(3, 2, Nz - 2), delay_int=0, delay_frac=0.5, amp=-0.3),
          dict(field_idx=2 * Nx * Ny * Nz + cell(2, 2, 1), delay_int=0, delay_frac=0.0, amp=0.8)]
    cp = [dict(field_idx=1 * Nx * Ny * Nz + cell(2, 2, 1), delay_int=0, delay_frac=0.75, amp=0.4),
          dict(field_idx=0 * Nx * Ny * Nz + cell(3, 3, Nz - 2), delay_int=0, delay_frac=0.0, amp=0.6)]
    e.configureTFSF(dict(signal=np.cos(np.arange(8) * 0.5).astype(np.float32), period=0, voltagePoints=vp,
                         currentPoints=cp))
    e.configureRLC(dict(elements=[
        _rlc(field_idx=cell(2, 3, Nz - 1), direction=0, type_flag=0, i2v=0.1, ilv=0.2),
        _rlc(field_idx=cell(3, 3, 1), direction=2, type_flag=1, i2v=0.2, ilv=0.1, vvd=0.5, vv2=0.1, vj1=0.2,
             vj2=0.1, ib0=0.3, b1=0.2, b2=0.1)]))
    e.configureSteadyState(dict(probe_idx=[2 * Nx * Ny * Nz + cell(2, 2, 1)], periodSamples=4, threshold=1e-6))
    e.setSteadyState(True, 0)
    tot = 3 * Nx * Ny * Nz
    e.uploadFields(r.standard_normal(tot).astype(np.float32), r.standard_normal(tot).astype(np.float32))
    return e


def test_step_follows_the_reference_phase_order():  # tests/test_webgpu.mjs:2675-2776
    """One step of the oracle equals the reference's 17 phases run one by one
    in its order (the C++ extension priorities), bit for bit, with every
    extension acting on shared cells; the same phases with the excitation and
    the Mur apply swapped do not, so the comparison sees the order."""
    N = (6, 6, 6)
    a, b, c = _all_extensions(N), _all_extensions(N), _all_extensions(N)
    a.step()
    for name in STEP_ORDER:
        b.phase(name)
    swapped = list(STEP_ORDER)
    i, j = swapped.index("applyExcitation"), swapped.index("murApply")
    swapped[i], swapped[j] = swapped[j], swapped[i]
    for name in swapped:
        c.phase(name)
    for f in ("volt", "curr"):
        assert np.array_equal(np.asarray(a.read(f), np.float32).view(np.uint32),
                              np.asarray(b.read(f), np.float32).view(np.uint32)), f
    for f in ("ss_e1", "pml_volt_flux", "pml_curr_flux", "ade_volt", "ade_curr"):
        assert np.array_equal(np.asarray(a.read(f)), np.asarray(b.read(f))), f
    assert a.numTS == 1
    assert not np.array_equal(np.asarray(a.read("volt")), np.asarray(c.read("volt")))
