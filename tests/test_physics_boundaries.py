"""Physics of the TFSF injection and the UPML absorber (operator generator
inputs, efs_b200/opgen.py) on the FP64 oracle.  The engine equals the
oracle's f32 mode bit for bit, so these properties hold for it too.

* TFSF leakage: a vacuum 48^3 grid (0.5 mm) with 8-cell UPML on all faces
  and a TFSF box 14 cells in; a Gaussian plane wave (10 +- 5 GHz) at normal
  incidence along +z and at 30 degrees in the xz plane.  The largest |E| in
  the scattered-field region (outside the box by more than 2 cells, inside
  the UPML) stays below 1e-3 of the largest |E| inside the box over 900 steps
  (measured 3.5e-4 and 2.1e-4: the plane wave's delays use the continuous
  phase velocity, the grid's differs by its numerical dispersion).
* UPML reflection: a point source (Ez, Gaussian 15 +- 10 GHz) at the centre of
  a 40^3 grid with 8-cell UPML (interface 12 cells from the source) against
  the same source in a 144^3 grid whose walls are too far to echo inside the
  270-step window: at probes 4 and 7 cells away (on axis and diagonal) the
  series differ by less than 3e-3 of their peak (measured 6e-5 .. 1.1e-3).
"""
import math

import numpy as np

from efs_b200 import opgen, workloads
from oracle.oracle import OracleEngine


def _grid(n, delta=0.5e-3, upml=0):
    grid = (n, n, n)
    mesh = opgen.Mesh(*[opgen.uniform_lines(k, delta) for k in grid])
    dT = opgen.cfl_dt(mesh)
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT)
    regs = []
    if upml:
        regs = opgen.upml_apply(mesh, dT, workloads._upml_boxes(grid, upml),
                                [opgen.pml_sigma(mesh, a, upml, upml) for a in range(3)], vv, vi, ii, iv)
    c = dict(vv=opgen.flat(vv), vi=opgen.flat(vi), ii=opgen.flat(ii), iv=opgen.flat(iv))
    return grid, mesh, dT, c, regs


def _leakage(k_hat, e_hat, n=48, W=8, inset=14, steps=900):
    grid, mesh, dT, c, regs = _grid(n, upml=W)
    sig = opgen.gauss_signal(10e9, 5e9, dT, steps).astype(np.float32)
    vi, iv = c["vi"].reshape(3, -1), c["iv"].reshape(3, -1)
    coef_at = lambda kind, comp, f: (vi if kind == "E" else iv)[comp][f].astype(np.float64)
    vp, cp = opgen.tfsf_plane_wave(mesh, dT, [inset] * 3, [n - 1 - inset] * 3, k_hat, e_hat, coef_at, len(sig))
    o = OracleEngine(grid, c, mode="f64")
    o.configurePML(regs)
    o.configureTFSF(dict(signal=sig, period=0, voltagePoints=vp, currentPoints=cp))
    work = np.zeros(grid, bool)
    work[W + 2:n - W - 2, W + 2:n - W - 2, W + 2:n - W - 2] = True
    near = np.zeros(grid, bool)
    near[inset - 2:n - inset + 2, inset - 2:n - inset + 2, inset - 2:n - inset + 2] = True
    total = np.zeros(grid, bool)
    total[inset + 2:n - inset - 2, inset + 2:n - inset - 2, inset + 2:n - inset - 2] = True
    inside = outside = 0.0
    for _ in range(steps // 10):
        o.iterate(10)
        v = np.abs(np.asarray(o.volt).reshape(3, *grid)).max(axis=0)
        inside = max(inside, float(v[total].max()))
        outside = max(outside, float(v[work & ~near].max()))
    return inside, outside


def test_tfsf_leakage_normal_and_oblique():
    th = math.radians(30.0)
    for k_hat, e_hat in (((0, 0, 1), (1, 0, 0)), ((math.sin(th), 0, math.cos(th)), (math.cos(th), 0, -math.sin(th)))):
        inside, outside = _leakage(k_hat, e_hat)
        assert inside > 0.8 * 0.5e-3                 # the incident wave reaches full amplitude (E0 * 0.5 mm)
        assert outside < 1e-3 * inside, (k_hat, outside / inside)


def _point_source(n, W, steps=270, offsets=(4, 7)):
    grid, mesh, dT, c, regs = _grid(n, upml=W)
    ctr = n // 2
    sig = opgen.gauss_signal(15e9, 10e9, dT, steps).astype(np.float32)
    o = OracleEngine(grid, c, mode="f64")
    if regs:
        o.configurePML(regs)
    o.configureExcitation(dict(signal=sig, delay=[0], amp=[1.0], dir=[2], pos=[(ctr * n + ctr) * n + ctr], period=0))
    N = n ** 3
    probes = [2 * N + ((ctr + d) * n + ctr) * n + ctr for d in offsets]
    probes += [2 * N + ((ctr + d) * n + ctr + d) * n + ctr for d in offsets]
    o.configureProbeGatherBuffered(probes, maxSamples=steps, sampleInterval=1)
    o.iterate(steps)
    r = o.readProbeGatherBuffered()
    return np.asarray(r["data"]).reshape(steps, -1)[:, 0::2]


def test_upml_reflection():
    a = _point_source(40, 8)
    b = _point_source(144, 0)
    err = np.abs(a - b).max(axis=0) / np.abs(b).max(axis=0)
    assert np.all(err < 3e-3), err
