"""The opt-in ADE apply step against the analytic single-pole response.

With the apply step on, the ADE state (a branch current scaled to volts) is
subtracted from E after the update, so a Drude or Lorentz medium disperses
the wave.  A plane wave crosses a 20 mm slab in a periodic 4 x 4 x 2400 grid
(workloads.slab_1d, 0.5 mm cells, Mur on the z faces); the FP64 oracle's
reflection R(f) and transmission T(f) over 3-12 GHz (spectra of the probe
series against a vacuum run) are compared with the Fabry-Perot response of a
slab of eps(f) (opgen.slab_rt):

* Lorentz, delta_eps = 2, omega_0 = 2 pi 15 GHz, delta = 2 pi 1 GHz (the
  dispersive workload's Lorentz medium; explicit scheme): |R|, |T| within
  0.02, complex T within 0.04 (measured 0.010, 0.006, 0.020: numerical
  dispersion over 40-100 cells per wavelength);
* Drude plasma, omega_p = 2 pi 10 GHz, gamma = 2 pi 0.5 GHz (explicit
  scheme; evanescent below 10 GHz): |R|, |T| and complex T within 0.01
  (measured 0.002);
* the workload's stiff Drude metal, omega_p = 1.4e16 rad/s, gamma = 3e13 1/s
  (omega_p dT ~ 1.3e4: implicit scheme): |R| within 0.01 of the analytic
  good-conductor value (~1), |T| below 1e-6, and no growth over a long run.

The CUDA engine equals the oracle's f32 mode bit for bit with the apply step
on (tests/test_gpu_parity.py), so these bars carry over to it.
"""
import math

import numpy as np
import pytest

from efs_b200 import opgen, workloads
from oracle.oracle import OracleEngine

LORENTZ = ("lorentz", 2.0, 2 * math.pi * 15e9, 2 * math.pi * 1e9)
PLASMA = ("drude", 2 * math.pi * 10e9, 2 * math.pi * 0.5e9)
METAL = ("drude", 1.4e16, 3e13)


@pytest.fixture(scope="module")
def vacuum():
    job = workloads.slab_1d(None)
    return workloads.run_slab_1d(OracleEngine(mode="f64"), job)


def response(medium, vacuum):
    job = workloads.slab_1d(medium)
    e = workloads.run_slab_1d(OracleEngine(mode="f64"), job)
    dT, D = job["dT"], job["delta"]
    nfft = 1 << 16
    f = np.fft.rfftfreq(nfft, dT)
    band = (f > 3e9) & (f < 12e9)
    spec = lambda x: np.fft.rfft(x, nfft)[band]
    d = (job["slab"][1] - job["slab"][0]) * D
    # numerical vacuum wavenumber along an axis (Yee dispersion relation)
    w = 2 * math.pi * f[band]
    kt = (2 / D) * np.arcsin(D / (opgen.C0 * dT) * np.sin(w * dT / 2))
    R = spec(e[:, 0] - vacuum[:, 0]) / spec(vacuum[:, 0])
    T = spec(e[:, 1]) / spec(vacuum[:, 1]) * np.exp(-1j * kt * d)
    eps = opgen.lorentz_eps(f[band], *medium[1:]) if medium[0] == "lorentz" else opgen.drude_eps(f[band], *medium[1:])
    Ra, Ta = opgen.slab_rt(f[band], eps, d)
    return job, e, R, T, Ra, Ta


@pytest.mark.parametrize("medium,tol_mag,tol_cplx", [(LORENTZ, 0.02, 0.04), (PLASMA, 0.01, 0.01)])
def test_slab_against_analytic(vacuum, medium, tol_mag, tol_cplx):
    job, _, R, T, Ra, Ta = response(medium, vacuum)
    assert job["ade_scheme"] == "explicit"
    assert np.abs(np.abs(R) - np.abs(Ra)).max() < tol_mag
    assert np.abs(np.abs(T) - np.abs(Ta)).max() < tol_mag
    assert np.abs(T - Ta).max() < tol_cplx


def test_stiff_drude_metal(vacuum):
    job, e, R, T, Ra, _ = response(METAL, vacuum)
    assert job["ade_scheme"] == "implicit"
    assert np.abs(np.abs(R) - np.abs(Ra)).max() < 0.01
    assert np.abs(T).max() < 1e-6
    # stability: no growing or ringing field in the periodic cells after the
    # pulse (x, y < 3; the last line of each periodic axis lies outside the
    # period and is never read by it)
    job = workloads.slab_1d(METAL, steps=20000)
    o = OracleEngine(mode="f64")
    workloads.configure(o, job)
    o.iterate(job["maxTS"])
    v = np.asarray(o.getFields()["volt"]).reshape(3, 4, 4, -1)[:, :3, :3, :]
    assert np.all(np.isfinite(v)) and np.abs(v).max() < 1e-4


def test_apply_off_keeps_state_only(vacuum):
    """With the apply step off (the reference's behaviour) a Lorentz slab
    changes nothing in the fields: its probes equal the vacuum run's."""
    job = workloads.slab_1d(LORENTZ)
    job["ade"] = dict(job["ade"], apply=False)
    # the explicit scheme leaves the core coefficients as in vacuum
    e = workloads.run_slab_1d(OracleEngine(mode="f64"), job)
    assert np.array_equal(e, vacuum)
