"""Extract the golden vectors used by the parity tests from the reference's
native-openEMS fixtures (reference tree: tests/fixtures/).

Usage: python tests/golden/make_golden.py <reference checkout>
The outputs are committed so the tests never read the reference tree.
  openems_cavity_vp.npy   engine_comparison/reference.json, engine "basic":
                          probe voltage vp, 251 samples every 2 steps from t=0
  openems_cavity_t.npy    the matching sample times (s)
  constants.json          physical constants of the fixtures
  openems_cavity_modes.npz  cavity/reference.json: the 26x11x32 PEC cavity's probe
                          voltage (6667 samples every 3 steps from t=0), its analytic
                          TE/TM mode frequencies and the reference's analysis
                          tolerances (tests/test_wasm.mjs:140-246)
  coax_ports.npz          coax/reference.json: port voltage and current series
                          (time_s, values), the analytic Z0 and the tolerance band
                          the reference's port test applies (tests/test_api.mjs:585-620)
  openems_dipole.npz      dipole/probe_*.csv: the four field probes of the hard-source
                          dipole with Mur on all faces (24 samples every 21 steps from
                          t=0): all three components per probe (E probes et1/et2 in
                          V/m, H probes ht1/ht2 in A/m), their sample times, the probe
                          nodes of the file headers and the fixture's amplitude floors
"""
import json
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py <path of the reference checkout>")
REF = sys.argv[1]
OUT = os.path.dirname(os.path.abspath(__file__))

fx = os.path.join(REF, "tests", "fixtures")
ref = json.load(open(os.path.join(fx, "engine_comparison", "reference.json")))["engine_probes"]
basic = ref["basic"]
# the three native engines agree bit for bit (comparison.json); keep that check
for other in ("sse", "sse-compressed"):
    assert ref[other]["voltage"] == basic["voltage"]
np.save(os.path.join(OUT, "openems_cavity_vp.npy"), np.asarray(basic["voltage"], np.float64))
np.save(os.path.join(OUT, "openems_cavity_t.npy"), np.asarray(basic["time_s"], np.float64))
with open(os.path.join(fx, "constants.json")) as f, open(os.path.join(OUT, "constants.json"), "w") as g:
    g.write(f.read())
coax = json.load(open(os.path.join(fx, "coax", "reference.json")))
np.savez(os.path.join(OUT, "coax_ports.npz"),
         ut_time=np.asarray(coax["probe_ut1"]["time_s"], np.float64), ut=np.asarray(coax["probe_ut1"]["voltage"], np.float64),
         it_time=np.asarray(coax["probe_it1"]["time_s"], np.float64), it=np.asarray(coax["probe_it1"]["voltage"], np.float64),
         z0=np.float64(coax["Z0_analytical_ohm"]), tol_upper=np.float64(coax["tolerances"]["upper_error"]),
         tol_lower=np.float64(coax["tolerances"]["lower_error"]))
cav = json.load(open(os.path.join(fx, "cavity", "reference.json")))
modes = dict(cav["te_modes"], **cav["tm_modes"])
names = sorted(modes)
np.savez(os.path.join(OUT, "openems_cavity_modes.npz"),
         time_s=np.asarray(cav["probe_data"]["time_s"], np.float64), voltage=np.asarray(cav["probe_data"]["voltage"], np.float64),
         mode_names=np.asarray(names), mode_freqs=np.asarray([modes[k] for k in names], np.float64),
         tolerances=np.asarray([cav["tolerances"][k] for k in ("te_freq_rel", "tm_freq_lower_rel", "te_min_amplitude",
                                                               "tm_min_amplitude")], np.float64),
         dims=np.asarray([cav["dimensions_m"][k] for k in ("a", "b", "d")], np.float64))


def probe_csv(path):
    """(node [i, j, k] of the header, rows of t and the three components)."""
    node, rows = None, []
    for line in open(path):
        if line.startswith("%"):
            if "start-coordinates" in line:
                node = [int(v) for v in line.split("[")[1].split("]")[0].split(",")]
            continue
        if line.strip():
            rows.append([float(v) for v in line.split()])
    return node, np.asarray(rows, np.float64)


dip = json.load(open(os.path.join(fx, "dipole", "reference.json")))
arrays = {}
for name in ("et1", "et2", "ht1", "ht2"):
    node, rows = probe_csv(os.path.join(fx, "dipole", "probe_%s.csv" % name))
    # the fixture's json keeps |field| per sample; the files hold the components
    assert np.allclose(np.sqrt((rows[:, 1:] ** 2).sum(1)), dip["probe_" + name]["voltage"], rtol=1e-9, atol=0)
    arrays[name + "_t"] = rows[:, 0]
    arrays[name] = rows[:, 1:]
    arrays[name + "_node"] = np.asarray(node, np.int64)
tol = dip["tolerances"]
np.savez(os.path.join(OUT, "openems_dipole.npz"), min_e_amp=np.float64(tol["min_e_amp"]),
         min_h_amp=np.float64(tol["min_h_amp"]), **arrays)
print("wrote", OUT)
