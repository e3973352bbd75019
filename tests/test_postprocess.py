"""Port post-processing (efs_b200.postprocess) against the reference's own
port tests and golden data, on the CPU.

* tests/test_api.mjs:85-130: a DFT peak within 1% of a 3 GHz sine, and
  |Z| = 75 ohm within 5% from V = 75 sin, I = sin.
* tests/test_api.mjs:585-620 on the native-openEMS coax fixture (committed as
  tests/golden/coax_ports.npz by tests/golden/make_golden.py): |U/I| over
  0.1-0.5 GHz inside the analytic Z0 band, incident + reflected = total.
* computeS11 on loads with known reflection, and the probe text format.
"""
import math
import os

import numpy as np

from efs_b200 import postprocess as pp

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def loop_dft(time, values, freq):
    """analysis.mjs:43-62 as written (sequential loops)."""
    re, im = [], []
    for f in freq:
        om = 2 * math.pi * f
        sr = si = 0.0
        for n in range(len(time)):
            w = time[n] - time[n - 1] if n > 0 else (time[1] - time[0] if len(time) > 1 else 1.0)
            sr += values[n] * math.cos(om * time[n]) * w
            si -= values[n] * math.sin(om * time[n]) * w
        re.append(sr)
        im.append(si)
    return np.array(re), np.array(im)


def test_dft_matches_reference_loops():
    r = np.random.default_rng(0)
    t = np.cumsum(r.uniform(0.5e-12, 1.5e-12, 300))
    v = r.standard_normal(300)
    f = np.linspace(0, 5e9, 37)
    a = pp.dft_time2freq(t, v, f)
    b = loop_dft(t, v, f)
    for x, y in zip(a, b):
        assert np.allclose(x, y, rtol=1e-12, atol=1e-12 * np.abs(y).max())


def test_dft_peak_and_impedance():
    N, dt, fsig = 2000, 1e-11, 3e9
    t = np.arange(N) * dt
    f = np.linspace(1e9, 5e9, 500)
    re, im = pp.dft_time2freq(t, np.sin(2 * math.pi * fsig * t), f)
    assert abs(f[np.argmax(np.hypot(re, im))] - fsig) / fsig < 0.01
    tf = np.linspace(0.5e9, 1.5e9, 100)
    vr, vi = pp.dft_time2freq(t, 75 * np.sin(2 * math.pi * 1e9 * t), tf)
    ir, ii = pp.dft_time2freq(t, np.sin(2 * math.pi * 1e9 * t), tf)
    z = (vr + 1j * vi) / (ir + 1j * ii)
    ci = np.argmin(np.abs(tf - 1e9))
    assert abs(abs(z[ci]) - 75) / 75 < 0.05


def test_coax_fixture_impedance_band_and_port_split():
    g = np.load(os.path.join(GOLDEN, "coax_ports.npz"))
    assert np.any(g["ut"] != 0)
    freq = np.linspace(0.1e9, 0.5e9, 200)
    port = pp.calc_port([(g["ut_time"], g["ut"])], [(g["it_time"], g["it"])], freq, 50.0)
    z = np.abs(port["uf_tot"] / port["if_tot"])
    z0 = float(g["z0"])
    assert np.all(z <= z0 * (1 + float(g["tol_upper"]))) and np.all(z >= z0 * (1 - float(g["tol_lower"])))
    assert np.allclose(port["uf_inc"] + port["uf_ref"], port["uf_tot"], rtol=1e-12, atol=0)
    assert np.allclose(port["if_inc"] - port["if_ref"], port["if_tot"], rtol=1e-12, atol=0)
    # a line matched to ~50 ohm: almost no reflected power
    assert np.all(port["P_ref"] < 0.01 * port["P_inc"])


def test_s11_of_known_loads():
    dt = 1e-12
    t = np.arange(4000) * dt
    pulse = np.exp(-((t - 400e-12) / 60e-12) ** 2)
    for z_load, want_db in ((100.0, 20 * math.log10(1 / 3)), (25.0, 20 * math.log10(1 / 3)), (75.0, 20 * math.log10(0.2))):
        out = pp.compute_s11((t, z_load * pulse), (t, pulse), fmax=5e9, nf=51)
        assert np.allclose(out["s11_dB"][1:], want_db, atol=1e-9)
        assert np.allclose(out["zRe"][1:], z_load) and np.allclose(out["zIm"][1:], 0, atol=1e-6)
    matched = pp.compute_s11((t, 50.0 * pulse), (t, pulse), fmax=5e9, nf=51)
    assert matched["bestS11"] < -200                      # |Gamma| ~ 0: the 1e-15 floor, -300 dB
    assert pp.compute_s11((t[:5], pulse[:5]), (t[:5], pulse[:5])) is None


def test_probe_file_round_trip_and_number_format():
    assert pp.js_number(1e-7) == "1e-7" and pp.js_number(1.5e-6) == "0.0000015"
    assert pp.js_number(2.5e-5) == "0.000025" and pp.js_number(0.1) == "0.1"
    assert pp.js_number(123456.0) == "123456" and pp.js_number(1e21) == "1e+21"
    assert pp.js_number(1e20) == "100000000000000000000" and pp.js_number(-3.25e-12) == "-3.25e-12"
    assert pp.js_number(0.0) == "0" and pp.js_number(1.2345e-300) == "1.2345e-300"
    probe = {"type": 1}
    times = pp.probe_times(probe, 4, 3, 1e-12)
    assert np.allclose(times, [3.5e-12, 6.5e-12, 9.5e-12, 12.5e-12])
    vals = np.array([0.0, 1.25e-9, -3.0, 7e-8])
    text = pp.probe_file(probe, times, vals)
    assert text.startswith("% time-domain current integration by openEMS (WebGPU)\n% t/s\tcurrent\n")
    t2, v2 = pp.parse_probe(text)
    assert np.array_equal(t2, times) and np.array_equal(v2, vals)
