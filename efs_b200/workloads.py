"""Jobs: the engine inputs of one solve, and the caller loop that drives them.

A job is a dict holding exactly what the reference's orchestrator extracts
from openEMS before it drives the engine (scripts/lib/sim-engine.mjs:533-638):
grid, coefficients, excitation, UPML regions, Mur config, TFSF config,
probes, NF2FF surface, dT, step budget and end criterion.  `configure`
replays the orchestrator's configure* sequence on any engine with the
WebGPUEngine method names (the CUDA engine, or the CPU oracle in tests), and
`run` replays its stepping loop (iterate in batches of 100, lagged energy
check, probe readback, :648-696).
"""
import math
import os

import numpy as np

from . import opgen


def openems_cavity():
    """The native-openEMS engine_comparison cavity (reference
    tests/generate_fixtures.py:439-500): 16x8x18 lines over 5x2x6 cm, PEC
    walls, Gaussian f0 = 5.5 GHz / fc = 4.5 GHz on the staircase from node
    (10,5,12) to (11,6,13), voltage probe on the z edge at (5,3,4) every 2
    steps, 500 steps.  dT is the fixture's (half its 1.23293515115e-11 s
    sample spacing)."""
    def lin(a, b, n):
        st = (b - a) / (n - 1)
        return [float("%.10e" % (a + i * st)) for i in range(n)]   # as written to the XML
    mesh = opgen.Mesh(lin(0, 5e-2, 16), lin(0, 2e-2, 8), lin(0, 6e-2, 18))
    dT = 1.23293515115e-11 / 2
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT)
    sig = opgen.gauss_signal(5.5e9, 4.5e9, dT, 500)
    Nx, Ny, Nz = mesh.shape
    p1 = [mesh.lines[k][i] for k, i in enumerate((10, 5, 12))]
    p2 = [mesh.lines[k][i] for k, i in enumerate((11, 6, 13))]
    amp, dirs, pos = [], [], []
    for n, (x, y, z) in opgen.find_path(mesh, p1, p2):
        amp.append(mesh.dl(n)[(x, y, z)[n]])
        dirs.append(n)
        pos.append(x * Ny * Nz + y * Nz + z)
    probe = opgen.voltage_probe(mesh, [5, 3, 4], [5, 3, 5], 1.0, 2)
    return dict(name="openems_cavity", grid=list(mesh.shape), dT=dT, maxTS=500, endCrit=0.0, mesh=mesh,
                coefficients=dict(vv=opgen.flat(vv), vi=opgen.flat(vi), ii=opgen.flat(ii), iv=opgen.flat(iv)),
                excitation=dict(signal=sig.astype(np.float32), delay=[0] * len(amp), amp=np.float32(amp), dir=dirs,
                                pos=pos, period=0),
                probes=[probe], include_t0=True)


def openems_dipole():
    """The native-openEMS dipole fixture (reference
    tests/generate_fixtures.py:313-423): a z-directed hard E source over one
    dipole length L = lambda/50 at f_max = 1 GHz, on a uniform mesh of
    step L/2 over +-20 L per axis (81 lines, drawing unit 1 um), Mur ABC on
    all six faces, a Gaussian pulse (f0 = 0, fc = f_max), 500 steps at the
    Courant step, and four field probes at the nodes nearest to (-+2.25 L, 0,
    0), sampled every 21 steps from t = 0.

    The hard source follows openEMS's hard E excitation: the source edges
    get vv = vi = 0 (the update leaves them at zero) and the excitation
    writes amplitude (edge length, E = 1 V/m along +z) x signal.  Mur faces are
    listed face by face in openEMS's order (xmin, xmax, ymin, ymax, zmin,
    zmax), each face's two tangential components after one another, so a
    corner edge keeps the value of the last face as in openEMS.  Probes:
    `field_probes` maps a probe name to (field, component, node, length):
    the raw field at the node divided by its edge length (E: primal, H:
    dual), which is what the fixture's probe files hold at these nodes."""
    du, f_max = 1e-6, 1e9
    lam = opgen.C0 / f_max / du
    L = lam / 50
    half, ext = L / 2, L * 20
    vals = []                                   # the generator's accumulated line values (um)
    v = -ext
    while v <= ext + 0.001:
        vals.append(v)
        v += half
    lines = [float("%.10e" % x) * du for x in vals]     # as written to the XML, in metres
    mesh = opgen.Mesh(lines, lines, lines)
    dT = opgen.cfl_dt(mesh)
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, bc=(-1,) * 6)
    Nx, Ny, Nz = mesh.shape
    amp, dirs, pos = [], [], []
    for n, (x, y, z) in opgen.find_path(mesh, [0.0, 0.0, -L / 2 * du], [0.0, 0.0, L / 2 * du]):
        vv[n][x, y, z] = 0.0
        vi[n][x, y, z] = 0.0
        amp.append(mesh.dl(n)[(x, y, z)[n]])
        dirs.append(n)
        pos.append(x * Ny * Nz + y * Nz + z)
    steps = 500
    sig = opgen.gauss_signal(0.0, f_max, dT, steps)
    faces = [(0, "lo"), (0, "hi"), (1, "lo"), (1, "hi"), (2, "lo"), (2, "hi")]
    coeff, normal, shifted = [], [], []
    for f in faces:
        m = opgen.mur_dual(mesh, dT, [f])
        for s in ("nyP", "nyPP"):
            coeff.append(m["coeff_" + s])
            normal.append(m["normal_idx_" + s])
            shifted.append(m["shifted_idx_" + s])

    def snap(val):                              # the generator's snap: first of the nearest lines
        return min(range(len(vals)), key=lambda i: abs(vals[i] - val))
    s = 4.5 * L / 2
    node = lambda px: (snap(px), snap(0.0), snap(0.0))
    dl2, dd1 = mesh.dl(2), mesh.dd(1)
    probes = {}
    for name, px in (("et1", -s), ("et2", s)):
        p = node(px)
        probes[name] = ("volt", 2, p, float(dl2[p[2]]))
    for name, px in (("ht1", -s), ("ht2", s)):
        p = node(px)
        probes[name] = ("curr", 1, p, float(dd1[p[1]]))
    return dict(name="openems_dipole", grid=list(mesh.shape), dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
                coefficients=dict(vv=opgen.flat(vv), vi=opgen.flat(vi), ii=opgen.flat(ii), iv=opgen.flat(iv)),
                excitation=dict(signal=sig.astype(np.float32), delay=[0] * len(amp), amp=np.float32(amp), dir=dirs,
                                pos=pos, period=0),
                mur=dict(coeff=np.concatenate(coeff), normal_idx=np.concatenate(normal),
                         shifted_idx=np.concatenate(shifted)),
                field_probes=probes, sample_interval=21)


def run_field_probes(engine, job):
    """Configure `engine` with the job and sample its `field_probes` at
    t = 0 and every `sample_interval` steps up to maxTS; returns
    {name: float64 series}.  Reads whole fields (getFields), so it suits
    small grids."""
    configure(engine, job)
    Nx, Ny, Nz = job["grid"]
    N = Nx * Ny * Nz
    out = {k: [] for k in job["field_probes"]}
    step, k = job["sample_interval"], 0
    while True:
        f = engine.getFields()
        for name, (field, n, (x, y, z), length) in job["field_probes"].items():
            out[name].append(float(np.asarray(f[field]).reshape(-1)[n * N + x * Ny * Nz + y * Nz + z]) / length)
        if k + step > job["maxTS"]:
            break
        engine.iterate(step)
        k += step
    return {k: np.asarray(v) for k, v in out.items()}


def openems_cavity_modes(steps=20000):
    """The native-openEMS cavity-resonator fixture (reference
    tests/generate_fixtures.py:63-178): 26x11x32 lines over 5x2x6 cm, PEC
    walls, Gaussian f0 = 5.5 GHz / fc = 4.5 GHz on the staircase from node
    (17,7,21) to (18,8,22), voltage probe on the z edge at (6,5,6) every 3
    steps, `steps` steps at the mesh's Courant step (what openEMS picked:
    the fixture's 1.14266409e-11 s sample spacing is 3 dT)."""
    def lin(a, b, n):
        st = (b - a) / (n - 1)
        return [float("%.10e" % (a + i * st)) for i in range(n)]   # as written to the XML
    mesh = opgen.Mesh(lin(0, 5e-2, 26), lin(0, 2e-2, 11), lin(0, 6e-2, 32))
    dT = opgen.cfl_dt(mesh)
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT)
    sig = opgen.gauss_signal(5.5e9, 4.5e9, dT, steps)
    Nx, Ny, Nz = mesh.shape
    ex = (Nx * 2 // 3, Ny * 2 // 3, Nz * 2 // 3)
    p1 = [mesh.lines[k][i] for k, i in enumerate(ex)]
    p2 = [mesh.lines[k][i + 1] for k, i in enumerate(ex)]
    amp, dirs, pos = [], [], []
    for n, (x, y, z) in opgen.find_path(mesh, p1, p2):
        amp.append(mesh.dl(n)[(x, y, z)[n]])
        dirs.append(n)
        pos.append(x * Ny * Nz + y * Nz + z)
    pr = (Nx // 4, Ny // 2, Nz // 5)
    probe = opgen.voltage_probe(mesh, list(pr), [pr[0], pr[1], pr[2] + 1], 1.0, 3)
    return dict(name="openems_cavity_modes", grid=list(mesh.shape), dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
                coefficients=dict(vv=opgen.flat(vv), vi=opgen.flat(vi), ii=opgen.flat(ii), iv=opgen.flat(iv)),
                excitation=dict(signal=sig.astype(np.float32), delay=[0] * len(amp), amp=np.float32(amp), dir=dirs,
                                pos=pos, period=0),
                probes=[probe], include_t0=True)


class _ChunkCells:
    """Per-cell eps_r of the cells with x index in [xs, xe), looked up by global x slice."""

    def __init__(self, ids, xs, values):
        self.ids, self.xs = ids, xs
        self.values = np.asarray(values, np.float64)

    def __getitem__(self, sl):
        return self.values[self.ids[sl.start - self.xs:sl.stop - self.xs]]


def _large_plain_chunk(args):
    """Operator rows of x-planes [x0, x1) for large_plain (runs in a worker)."""
    n, delta, dT, x0, x1, diel, eps_vals, pec_boxes, pml = args
    lines = opgen.uniform_lines(n, delta)
    mesh = opgen.Mesh(lines, lines, lines)
    xs, xe = max(x0 - 1, 0), min(x1, n - 1)
    ids = np.zeros((xe - xs, n - 1, n - 1), np.uint8)
    for k, (lo, hi) in enumerate(diel):
        a, b = max(lo[0], xs), min(hi[0], xe)
        if a < b:
            ids[a - xs:b - xs, lo[1]:hi[1], lo[2]:hi[2]] = k + 1

    def pec(nn, c0, c1):
        m = np.zeros((c1 - c0, n, n), bool)
        for lo, hi in pec_boxes:
            m |= opgen.edge_mask_in_box(mesh, nn, lo, hi, xslice=slice(c0, c1))
        return m
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, eps_r=_ChunkCells(ids, xs, eps_vals), pec_edges=pec,
                                          bc=(2, 2, 2, 2, 3, 3), x0=x0, x1=x1)
    if pml:
        boxes = [((0, 0, 0), (n, n, pml)), ((0, 0, n - pml), (n, n, pml))]
        opgen.upml_apply(mesh, dT, boxes, [None, None, opgen.pml_sigma(mesh, 2, pml, pml)], vv, vi, ii, iv,
                         x0=x0, build=False)
    m, mt = opgen.to_indexed(vv, vi, ii, iv)
    return x0, x1, m, mt.table()


def _parallel_map(fn, items, workers):
    if workers <= 1 or len(items) <= 1:
        return [fn(a) for a in items]
    import multiprocessing as mp
    ctx = mp.get_context("spawn")          # never fork a process that may hold a CUDA context
    with ctx.Pool(workers) as pool:
        return pool.map(fn, items, chunksize=1)


def large_plain(n=512, delta=0.5e-3, seed=2, nboxes=40, pml=8, nfreq=3, tfsf_inset=20, nf2ff_inset=10,
                steps=20000, f0=10e9, fc=5e9, chunk=32, tfsf=True, nf2ff=True):
    """Plain large solve (the benchmark's headline workload at n = 512):
    uniform n^3 lines with spacing delta; `nboxes` seeded axis-aligned boxes
    (numpy default_rng(seed)), the first half PEC, the rest dielectric with
    eps_r ~ U[2, 10]; Mur ABC on the x and y faces, `pml`-cell UPML on the z
    faces; a TFSF Gaussian plane wave (f0, fc) at normal incidence along +z,
    E along x, on the box `tfsf_inset` cells inside the boundary; NF2FF box
    `nf2ff_inset` cells inside with `nfreq` frequencies spread over the pulse
    band.  Coefficients come out as a material index + table."""
    lines = opgen.uniform_lines(n, delta)
    mesh = opgen.Mesh(lines, lines, lines)
    dT = opgen.cfl_dt(mesh)
    rng = np.random.default_rng(seed)
    nc = n - 1
    eps_vals = [1.0]
    pec_boxes, diel = [], []
    margin = tfsf_inset + 4
    lo_cap = max(margin, 1)
    if nboxes and n <= lo_cap + 1:
        raise ValueError("large_plain: n = %d leaves no room for boxes inside the TFSF inset %d (need n > %d)"
                         % (n, tfsf_inset, lo_cap + 1))
    for i in range(nboxes):
        size = rng.integers(max(2, n // 32), max(3, n // 8), 3)
        lo = np.array([rng.integers(lo_cap, max(lo_cap + 1, nc - margin - s)) for s in size])
        hi = np.minimum(lo + size, nc - margin)
        if i < nboxes // 2:
            pec_boxes.append(([lines[lo[a]] for a in range(3)], [lines[hi[a]] for a in range(3)]))
        else:
            eps_vals.append(float(rng.uniform(2.0, 10.0)))
            diel.append((lo.tolist(), hi.tolist()))
    boxes = [((0, 0, 0), (n, n, pml)), ((0, 0, n - pml), (n, n, pml))] if pml else []
    sig_fns = [None, None, opgen.pml_sigma(mesh, 2, pml, pml)] if pml else [None] * 3
    items = [(n, delta, dT, x0, min(n, x0 + chunk), diel, eps_vals, pec_boxes, pml) for x0 in range(0, n, chunk)]
    workers = min(len(items), max(1, (os.cpu_count() or 1)), 32) if n >= 128 else 1
    mt = opgen.MaterialTable()
    mat = np.empty(n * n * n, np.uint32)
    for x0, x1, m, tab in _parallel_map(_large_plain_chunk, items, workers):
        remap = mt.add(tab)
        mat[x0 * n * n:x1 * n * n] = remap[m]
    table = mt.table()
    job = dict(name="large_plain_%d" % n, grid=[n, n, n], dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
               coefficients=dict(mat=mat, table=table))
    if boxes:
        job["pml"] = opgen.upml_apply(mesh, dT, boxes, sig_fns, build=True)
    zr = (pml, n - 1 - pml) if pml else None   # Mur faces stop at the UPML slabs
    job["mur"] = opgen.mur_dual(mesh, dT, [(0, "lo"), (0, "hi"), (1, "lo"), (1, "hi")], ranges=[None, None, zr])
    sig = opgen.gauss_signal(f0, fc, dT, steps).astype(np.float32)
    if tfsf:
        def coef_at(kind, comp, flat):
            return table[mat[flat], (3 if kind == "E" else 9) + comp].astype(np.float64)
        lo = [tfsf_inset] * 3
        hi = [n - 1 - tfsf_inset] * 3
        vp, cp = opgen.tfsf_plane_wave(mesh, dT, lo, hi, (0, 0, 1), (1, 0, 0), coef_at, len(sig))
        job["tfsf"] = dict(signal=sig, period=0, voltagePoints=vp, currentPoints=cp)
    if nf2ff:
        lo = [nf2ff_inset] * 3
        hi = [n - 1 - nf2ff_inset] * 3
        pts, meta, primal, dual = opgen.nf2ff_box(mesh, lo, hi)
        freqs = [f0 + fc * (k - (nfreq - 1) / 2) / max(1, nfreq - 1) for k in range(nfreq)]
        job["nf2ff"] = dict(surfaceIndices=pts.ravel(), numPoints=len(pts), omegas=[2 * math.pi * f for f in freqs],
                            dT=dT, gridSize=[n, n, n], primalEdgeLens=primal, dualEdgeLens=dual, maxTS=steps,
                            windowType=0)
        job["nf2ff_meta"] = meta
        job["nf2ff_freqs"] = freqs
    return job


def _graded_axis(core, count, dmax=2e-3, ratio=1.4, below=None):
    """`core` lines (sorted, metres) extended at both ends by cells growing by
    `ratio` up to dmax until the axis holds exactly `count` lines; `below`
    fixes how many of the added lines go before the core (default: half)."""
    core = list(core)
    add = count - len(core)
    lo_n = add // 2 if below is None else below
    hi_n = add - lo_n
    lo, hi = [], []
    d = core[1] - core[0]
    x = core[0]
    for _ in range(lo_n):
        d = min(d * ratio, dmax)
        x -= d
        lo.append(x)
    d = core[-1] - core[-2]
    x = core[-1]
    for _ in range(hi_n):
        d = min(d * ratio, dmax)
        x += d
        hi.append(x)
    return np.asarray(lo[::-1] + core + hi)


def patch_antenna(steps=30000, end_db=-50.0, pml=8):
    """Plain single solve on a graded mesh: a patch antenna, 86 x 87 x 71 lines.
    Cells 0.508-2 mm, graded by at most 1.4: uniform 1 mm lines over the
    60 x 60 mm substrate footprint (patch edges, feed and centre on lines),
    three 0.508 mm cells through the 1.524 mm substrate (eps_r 3.38,
    0.0015 S/m), growing to 2 mm outside.  PEC ground sheet at z = 0 under the
    substrate, 32 x 40 mm PEC patch sheet on top, a 50 ohm lumped port from
    ground to patch at (-6, 0) mm driven by a Gaussian f0 = 2 GHz, fc = 1 GHz,
    `pml`-cell UPML on all faces, voltage and current probes at the port every
    step, `steps` timesteps or the energy end criterion `end_db`."""
    mm = 1e-3
    fine = [i * mm for i in range(-30, 31)]                 # 61 lines, 1 mm
    X = _graded_axis(fine, 86)
    Y = _graded_axis(fine, 87)
    zsub = [0.0, 0.508 * mm, 1.016 * mm, 1.524 * mm]
    Z = _graded_axis(zsub, 71, below=16)
    mesh = opgen.Mesh(X, Y, Z)
    Nx, Ny, Nz = mesh.shape
    dT = opgen.cfl_dt(mesh)
    # substrate cells
    ix0, ix1 = mesh.snap(0, -30 * mm), mesh.snap(0, 30 * mm)
    iy0, iy1 = mesh.snap(1, -30 * mm), mesh.snap(1, 30 * mm)
    iz0, iz1 = mesh.snap(2, 0.0), mesh.snap(2, 1.524 * mm)
    eps = np.ones((Nx - 1, Ny - 1, Nz - 1))
    kap = np.zeros((Nx - 1, Ny - 1, Nz - 1))
    eps[ix0:ix1, iy0:iy1, iz0:iz1] = 3.38
    kap[ix0:ix1, iy0:iy1, iz0:iz1] = 0.0015
    pec = []
    for n in range(3):
        m = np.zeros(mesh.shape, bool)
        if n < 2:
            m |= opgen.edge_mask_in_box(mesh, n, (-30 * mm, -30 * mm, 0.0), (30 * mm, 30 * mm, 0.0))            # ground
            m |= opgen.edge_mask_in_box(mesh, n, (-16 * mm, -20 * mm, 1.524 * mm), (16 * mm, 20 * mm, 1.524 * mm))  # patch
        pec.append(m)
    fx, fy = mesh.snap(0, -6 * mm), mesh.snap(1, 0.0)
    nport = iz1 - iz0
    lumped = [np.zeros(mesh.shape) for _ in range(3)]
    lumped[2][fx, fy, iz0:iz1] = nport / 50.0
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, eps_r=eps, kappa=kap, pec_edges=pec, lumped_g=lumped,
                                          bc=(0, 0, 0, 0, 0, 0))
    W = pml
    boxes = [((0, 0, 0), (W, Ny, Nz)), ((Nx - W, 0, 0), (W, Ny, Nz)),
             ((W, 0, 0), (Nx - 2 * W, W, Nz)), ((W, Ny - W, 0), (Nx - 2 * W, W, Nz)),
             ((W, W, 0), (Nx - 2 * W, Ny - 2 * W, W)), ((W, W, Nz - W), (Nx - 2 * W, Ny - 2 * W, W))]
    sig_fns = [opgen.pml_sigma(mesh, a, W, W) for a in range(3)]
    regions = opgen.upml_apply(mesh, dT, boxes, sig_fns, vv, vi, ii, iv, build=True)
    mat, mt = opgen.to_indexed(vv, vi, ii, iv)
    sig = opgen.gauss_signal(2e9, 1e9, dT, steps).astype(np.float32)
    pos = [fx * Ny * Nz + fy * Nz + z for z in range(iz0, iz1)]
    zm = (iz0 + iz1) // 2
    probes = [opgen.voltage_probe(mesh, (fx, fy, iz0), (fx, fy, iz1), interval=1),
              opgen.current_probe(mesh, (fx - 1, fy - 1, zm), (fx, fy, zm), 2, interval=1)]
    return dict(name="patch_antenna", grid=[Nx, Ny, Nz], dT=dT, maxTS=steps, endCrit=10.0 ** (end_db / 10.0),
                mesh=mesh, coefficients=dict(mat=mat, table=mt.table()), pml=regions, probes=probes,
                excitation=dict(signal=sig, delay=[0] * nport, amp=[1.0 / nport] * nport, dir=[2] * nport, pos=pos,
                                period=0))


def _upml_boxes(grid, W):
    """Six non-overlapping UPML slabs, `W` lines thick, on all faces of `grid`."""
    Nx, Ny, Nz = grid
    return [((0, 0, 0), (W, Ny, Nz)), ((Nx - W, 0, 0), (W, Ny, Nz)),
            ((W, 0, 0), (Nx - 2 * W, W, Nz)), ((W, Ny - W, 0), (Nx - 2 * W, W, Nz)),
            ((W, W, 0), (Nx - 2 * W, Ny - 2 * W, W)), ((W, W, Nz - W), (Nx - 2 * W, Ny - 2 * W, W))]


def _dispersive_chunk(args):
    """Operator rows of x-planes [x0, x1) for dispersive (runs in a worker):
    vacuum with UPML on all faces."""
    grid, delta, dT, x0, x1, pml = args
    mesh = opgen.Mesh(*[opgen.uniform_lines(n, delta) for n in grid])
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, bc=(0, 0, 0, 0, 0, 0), x0=x0, x1=x1)
    opgen.upml_apply(mesh, dT, _upml_boxes(grid, pml), [opgen.pml_sigma(mesh, a, pml, pml) for a in range(3)],
                     vv, vi, ii, iv, x0=x0, build=False)
    m, mt = opgen.to_indexed(vv, vi, ii, iv)
    return x0, x1, m, mt.table()


def dispersive(grid=(800, 800, 400), delta=0.25e-3, seed=5, pml=8, cover=0.3, nfreq=5, steps=40000, tfsf_inset=20,
               nf2ff_inset=10, angle_deg=30.0, chunk=16, workers=None, apply=True):
    """Plain dispersive solve: a uniform grid (800 x 800 x 400 lines, 0.25 mm),
    `pml`-cell UPML on all faces, seeded spheres (numpy default_rng(seed),
    radius 5-40 cells, smaller on small grids) inside the TFSF box covering
    `cover` of all cells (on small grids at most half of that box), each
    single-pole Drude (omega_p = 1.4e16 rad/s, gamma = 3e13 1/s) or Lorentz
    (delta_eps = 2, omega_0 = 2 pi 15 GHz, delta = 2 pi 1 GHz), a TFSF
    Gaussian plane wave (10 GHz +- 5 GHz) at `angle_deg` from +z in the xz
    plane, NF2FF with `nfreq` frequencies.

    The media are the ADE extension's inputs from opgen.ade_drude /
    opgen.ade_lorentz with the apply step on (`apply`): the Lorentz pole
    with the explicit scheme, the stiff Drude pole (omega_p dT ~ 6.7e3) with
    the implicit one, whose Drude cells get their own core coefficients (a
    material-table row).  With apply=False the job is the reference's
    state-only form: the same ADE inputs, vacuum core coefficients, and the
    dispersion never reaches the fields (webgpu-fdtd.mjs:405-454,
    :1129-1172).  Only the voltage side has coefficients; the current side
    is all zero."""
    Nx, Ny, Nz = grid
    N = Nx * Ny * Nz
    mesh = opgen.Mesh(*[opgen.uniform_lines(n, delta) for n in grid])
    dT = opgen.cfl_dt(mesh)
    items = [(tuple(grid), delta, dT, x0, min(Nx, x0 + chunk), pml) for x0 in range(0, Nx, chunk)]
    if workers is None:
        workers = min(len(items), max(1, os.cpu_count() or 1), 32)
    mt = opgen.MaterialTable()
    mat = np.empty(N, np.uint32)
    for x0, x1, m, tab in _parallel_map(_dispersive_chunk, items, workers):
        mat[x0 * Ny * Nz:x1 * Ny * Nz] = mt.add(tab)[m]
    regions = opgen.upml_apply(mesh, dT, _upml_boxes(grid, pml), [opgen.pml_sigma(mesh, a, pml, pml) for a in range(3)],
                               build=True)
    # spheres: label 1 = Drude, 2 = Lorentz; a later sphere never relabels a
    # cell.  Spheres lie inside the TFSF box with a 2-cell margin (the total
    # field region), away from the UPML and the injection surface.
    rng = np.random.default_rng(seed)
    label = np.zeros(grid, np.uint8)
    covered = 0
    lo_c = tfsf_inset + 2
    room = min(n - 1 - tfsf_inset - 2 - lo_c for n in grid)
    rmax = max(1, min(40, room // 2 - 1))
    box = int(np.prod([n - 1 - tfsf_inset - 2 - lo_c + 1 for n in grid]))
    target = min(cover * N, 0.5 * box)        # small grids: at most half of the box the spheres may fill
    while covered < target:
        r = int(rng.integers(min(5, rmax), rmax + 1))
        c = [int(rng.integers(lo_c + r, n - 1 - tfsf_inset - 2 - r + 1)) for n in grid]
        kind = 1 if rng.random() < 0.5 else 2
        sl = tuple(slice(c[a] - r, c[a] + r + 1) for a in range(3))
        ax = np.arange(-r, r + 1) ** 2
        ball = (ax[:, None, None] + ax[None, :, None] + ax[None, None, :]) <= r * r
        sub = label[sl]
        new = ball & (sub == 0)
        sub[new] = kind
        covered += int(new.sum())
    flat = label.reshape(-1)
    cells = [np.flatnonzero(flat == kind).astype(np.uint32) for kind in (1, 2)]
    del label, flat
    # ADE inputs from the sphere cells' core coefficients (one material row:
    # uniform vacuum inside the TFSF box)
    table = mt.table()
    probe = cells[0][0] if len(cells[0]) else cells[1][0]
    row = table[mat[probe]].astype(np.float64)
    drude = [opgen.ade_drude(row[n:n + 1], row[3 + n:4 + n], dT, 1.4e16, 3e13) for n in range(3)]
    lorentz = [opgen.ade_lorentz(row[n:n + 1], row[3 + n:4 + n], dT, 2.0, 2 * math.pi * 15e9, 2 * math.pi * 1e9)
               for n in range(3)]
    if apply and drude[0]["scheme"] == "implicit" and len(cells[0]):
        drow = row.copy()
        for n in range(3):
            drow[n], drow[3 + n] = drude[n]["vv"][0], drude[n]["vi"][0]
        did = np.uint32(mt.add(drow[None, :].astype(np.float32))[0])
        mat[cells[0]] = did
        table = mt.table()
    orders = []
    for kind, co, has_lor in ((1, drude, False), (2, lorentz, True)):
        n = len(cells[kind - 1])
        dirs = []
        for d in range(3):
            e = dict(dir=d, pos_idx=cells[kind - 1], v_int_ADE=np.full(n, co[d]["v_int"][0], np.float32),
                     v_ext_ADE=np.full(n, co[d]["v_ext"][0], np.float32))
            if has_lor:
                e["v_Lor_ADE"] = np.full(n, co[d]["v_lor"][0], np.float32)
            dirs.append(e)
        orders.append(dict(numCells=n, hasLorentz=has_lor, directions=dirs))
    f0, fc = 10e9, 5e9
    sig = opgen.gauss_signal(f0, fc, dT, steps).astype(np.float32)
    th = math.radians(angle_deg)

    def coef_at(kind_, comp, f):
        return table[mat[f], (3 if kind_ == "E" else 9) + comp].astype(np.float64)
    lo = [tfsf_inset] * 3
    hi = [n - 1 - tfsf_inset for n in grid]
    vp, cp = opgen.tfsf_plane_wave(mesh, dT, lo, hi, (math.sin(th), 0.0, math.cos(th)),
                                   (math.cos(th), 0.0, -math.sin(th)), coef_at, len(sig))
    pts, meta, primal, dual = opgen.nf2ff_box(mesh, [nf2ff_inset] * 3, [n - 1 - nf2ff_inset for n in grid])
    freqs = [f0 + fc * (k - (nfreq - 1) / 2) / max(1, nfreq - 1) for k in range(nfreq)]
    return dict(name="dispersive", grid=list(grid), dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
                coefficients=dict(mat=mat, table=table), pml=regions, ade=dict(orders=orders, apply=bool(apply)),
                tfsf=dict(signal=sig, period=0, voltagePoints=vp, currentPoints=cp),
                nf2ff=dict(surfaceIndices=pts.ravel(), numPoints=len(pts), omegas=[2 * math.pi * f for f in freqs],
                           dT=dT, gridSize=list(grid), primalEdgeLens=primal, dualEdgeLens=dual, maxTS=steps,
                           windowType=0),
                nf2ff_meta=meta, nf2ff_freqs=freqs, dispersive_cells=covered, dispersive_target=target,
                sphere_box=(lo_c, [n - 1 - tfsf_inset - 2 for n in grid]))


def _stub_filter_one(args):
    """Coefficients of one microstrip stub filter (runs in a worker)."""
    grid, delta, dT, sub, w, stub, xa, xb, yc = args
    Nx, Ny, Nz = grid
    lines = [opgen.uniform_lines(N, delta) for N in grid]
    mesh = opgen.Mesh(*lines)
    eps = np.ones((Nx - 1, Ny - 1, Nz - 1))
    eps[:, :, :sub] = 3.66                        # substrate on the ground plane
    X, Y, Z = lines
    y0t = yc - w // 2
    xs = Nx // 2 - w // 2
    zt = Z[sub]
    pec = []
    for n in range(3):
        m = np.zeros(grid, bool)
        if n < 2:                                 # trace and stub: sheets in the plane z = sub
            m |= opgen.edge_mask_in_box(mesh, n, (X[xa], Y[y0t], zt), (X[xb], Y[y0t + w], zt))
            m |= opgen.edge_mask_in_box(mesh, n, (X[xs], Y[y0t + w], zt), (X[xs + w], Y[y0t + w + stub], zt))
        pec.append(m)
    lumped = [np.zeros(grid) for _ in range(3)]
    for xp in (xa, xb):                           # 50 ohm ports: `sub` series z edges between ground and trace
        lumped[2][xp, yc, :sub] = sub / 50.0
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, eps_r=eps, pec_edges=pec, lumped_g=lumped, bc=(0, 0, 0, 0, 0, 0))
    mat, mt = opgen.to_indexed(vv, vi, ii, iv)
    return mat, mt.table()


def stub_filters(count=64, seed=3, delta=0.2e-3, steps=15000, workers=None):
    """The batched sweep workload: `count` microstrip stub filters with
    per-axis line counts ~ U[60, 180] (numpy default_rng(seed)), uniform `delta` mesh
    (so every instance shares dT and the excitation signal).  PEC ground on
    the z = 0 face, a 0.8 mm substrate eps_r = 3.66, a 1.8 mm PEC trace along
    x with a stub along +y of seeded length U[8, 20] mm (cut to the room the
    grid leaves), two single-column 50 ohm lumped ports at the trace ends, a
    Gaussian pulse f0 = fc = 3.5 GHz (0-7 GHz) driving port 1, voltage and
    current probes at both ports, Mur ABC on the other five faces."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(60, 181, (count, 3))
    stub_mm = rng.uniform(8e-3, 20e-3, count)
    sub = int(round(0.8e-3 / delta))
    w = int(round(1.8e-3 / delta))
    dT = opgen.cfl_dt(opgen.Mesh(*[opgen.uniform_lines(4, delta)] * 3))
    sig = opgen.gauss_signal(3.5e9, 3.5e9, dT, steps).astype(np.float32)
    interval = opgen.nyquist_interval(7e9, dT)
    items, jobs = [], []
    for i in range(count):
        Nx, Ny, Nz = (int(v) for v in sizes[i])
        xa, xb, yc = 6, Nx - 7, Ny // 2
        stub = max(1, min(int(round(stub_mm[i] / delta)), Ny - (yc - w // 2 + w) - 4))
        items.append(((Nx, Ny, Nz), delta, dT, sub, w, stub, xa, xb, yc))
        mesh = opgen.Mesh(*[opgen.uniform_lines(N, delta) for N in (Nx, Ny, Nz)])
        pos = [xa * Ny * Nz + yc * Nz + z for z in range(sub)]
        probes = []
        for xp in (xa, xb):
            probes.append(opgen.voltage_probe(mesh, (xp, yc, 0), (xp, yc, sub), interval=interval))
            probes.append(opgen.current_probe(mesh, (xp - 1, yc - 1, sub // 2), (xp, yc, sub // 2), 2, interval=interval))
        jobs.append(dict(name="stub_filter_%d" % i, grid=[Nx, Ny, Nz], dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
                         excitation=dict(signal=sig, delay=[0] * sub, amp=[1.0 / sub] * sub, dir=[2] * sub, pos=pos,
                                         period=0),
                         mur=opgen.mur_dual(mesh, dT, [(0, "lo"), (0, "hi"), (1, "lo"), (1, "hi"), (2, "hi")]),
                         probes=probes, stub_cells=stub))
    if workers is None:
        workers = min(count, max(1, os.cpu_count() or 1), 32)
    for job, (mat, table) in zip(jobs, _parallel_map(_stub_filter_one, items, workers)):
        job["coefficients"] = dict(mat=mat, table=table)
    return jobs


def _served_tfsf_one(args):
    """Coefficients of one served TFSF job: vacuum cube with a dielectric box (runs in a worker)."""
    side, nz, delta, dT = args
    grid = (side, side, nz)
    mesh = opgen.Mesh(*[opgen.uniform_lines(N, delta) for N in grid])
    eps = np.ones((side - 1, side - 1, nz - 1))
    a, b = side // 2 - side // 8, side // 2 + side // 8
    c, d = nz // 2 - nz // 8, nz // 2 + nz // 8
    eps[a:b, a:b, c:d] = 4.0
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, eps_r=eps, bc=(0, 0, 0, 0, 0, 0))
    mat, mt = opgen.to_indexed(vv, vi, ii, iv)
    return mat, mt.table()


def served_template(kind, side, delta=0.5e-3, steps=25000):
    """Inputs of one request of the served stream, for a cubic grid of
    `side` lines: kind "port" is a stub
    filter (two 50 ohm lumped ports, Mur on five faces, Gaussian 0-7 GHz at
    port 1, probes at both ports); kind "tfsf" is a vacuum cube holding a
    dielectric box (eps_r = 4), a TFSF Gaussian plane wave (normal incidence,
    10 GHz +- 5 GHz) on the box 6 cells in, NF2FF on the box 3 cells in at 2
    frequencies, Mur on all six faces.  The signal covers `steps` timesteps;
    a request runs its own step count on these inputs."""
    nz = side
    if kind == "port":
        sub, w = 4, 9
        d = 0.2e-3                                   # port jobs keep the stub filters' 0.2 mm cells
        dT = opgen.cfl_dt(opgen.Mesh(*[opgen.uniform_lines(4, d)] * 3))
        xa, xb, yc = 6, side - 7, side // 2
        stub = max(1, min(side // 3, side - (yc - w // 2 + w) - 4))
        grid = (side, side, nz)
        mat, table = _stub_filter_one((grid, d, dT, sub, w, stub, xa, xb, yc))
        mesh = opgen.Mesh(*[opgen.uniform_lines(N, d) for N in grid])
        sig = opgen.gauss_signal(3.5e9, 3.5e9, dT, steps).astype(np.float32)
        interval = opgen.nyquist_interval(7e9, dT)
        probes = []
        for xp in (xa, xb):
            probes.append(opgen.voltage_probe(mesh, (xp, yc, 0), (xp, yc, sub), interval=interval))
            probes.append(opgen.current_probe(mesh, (xp - 1, yc - 1, sub // 2), (xp, yc, sub // 2), 2, interval=interval))
        pos = [xa * side * nz + yc * nz + z for z in range(sub)]
        return dict(name="served_port_%d" % side, grid=list(grid), dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
                    coefficients=dict(mat=mat, table=table), probes=probes,
                    excitation=dict(signal=sig, delay=[0] * sub, amp=[1.0 / sub] * sub, dir=[2] * sub, pos=pos, period=0),
                    mur=opgen.mur_dual(mesh, dT, [(0, "lo"), (0, "hi"), (1, "lo"), (1, "hi"), (2, "hi")]))
    grid = (side, side, nz)
    mesh = opgen.Mesh(*[opgen.uniform_lines(N, delta) for N in grid])
    dT = opgen.cfl_dt(mesh)
    mat, table = _served_tfsf_one((side, nz, delta, dT))
    f0, fc = 10e9, 5e9
    sig = opgen.gauss_signal(f0, fc, dT, steps).astype(np.float32)

    def coef_at(kind_, comp, flat):
        return table[mat[flat], (3 if kind_ == "E" else 9) + comp].astype(np.float64)
    lo, hi = [6] * 3, [side - 7, side - 7, nz - 7]
    vp, cp = opgen.tfsf_plane_wave(mesh, dT, lo, hi, (0, 0, 1), (1, 0, 0), coef_at, len(sig))
    pts, meta, primal, dual = opgen.nf2ff_box(mesh, [3] * 3, [side - 4, side - 4, nz - 4])
    freqs = [f0 - fc / 2, f0 + fc / 2]
    faces = [(a, s_) for a in range(3) for s_ in ("lo", "hi")]
    return dict(name="served_tfsf_%d" % side, grid=list(grid), dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh,
                coefficients=dict(mat=mat, table=table), probes=[],
                mur=opgen.mur_dual(mesh, dT, faces),
                tfsf=dict(signal=sig, period=0, voltagePoints=vp, currentPoints=cp),
                nf2ff=dict(surfaceIndices=pts.ravel(), numPoints=len(pts), omegas=[2 * math.pi * f for f in freqs], dT=dT,
                           gridSize=list(grid), primalEdgeLens=primal, dualEdgeLens=dual, maxTS=steps, windowType=0),
                nf2ff_meta=meta, nf2ff_freqs=freqs)


def job_bytes_per_step(job):
    """Algorithmic HBM bytes of one timestep of `job` (fields read+written once,
    one u32 material index per cell, UPML/Mur/TFSF/NF2FF/probe traffic):
    core 48 B + 4 B per cell; UPML 48 B flux r/w (E and H) + 72 B coefficients
    per region cell (3 components); Mur 3 passes ~ 28 B per point; TFSF/excitation
    16 B per point; NF2FF 24 B field reads + 96 B accumulator r/w per
    point-frequency."""
    Nx, Ny, Nz = job["grid"]
    N = Nx * Ny * Nz
    coeff = 4 if "mat" in job["coefficients"] else 48
    b = N * (48 + coeff)
    for r in job.get("pml") or []:
        c = r["numLines"][0] * r["numLines"][1] * r["numLines"][2]
        b += c * (48 + 72)
    if job.get("mur"):
        b += 28 * (len(job["mur"]["coeff_nyP"]) + len(job["mur"]["coeff_nyPP"]))
    if job.get("tfsf"):
        t = job["tfsf"]
        nv = len(t["voltagePoints"]["field_idx"]) if isinstance(t["voltagePoints"], dict) else len(t["voltagePoints"])
        nc = len(t["currentPoints"]["field_idx"]) if isinstance(t["currentPoints"], dict) else len(t["currentPoints"])
        b += 16 * (nv + nc)
    if job.get("excitation"):
        b += 16 * len(job["excitation"]["amp"])
    if job.get("nf2ff"):
        nf = job["nf2ff"]
        b += nf["numPoints"] * (24 + 96 * len(nf.get("omegas") or [1]))
    return b


def configure(engine, job):
    """The orchestrator's configure sequence (sim-engine.mjs:541-638)."""
    engine.init(job["grid"], job["coefficients"])
    if job.get("excitation"):
        engine.configureExcitation(job["excitation"])
    if job.get("pml"):
        engine.configurePML(job["pml"])
    if job.get("mur"):
        engine.configureMur(job["mur"])
    if job.get("tfsf"):
        engine.configureTFSF(job["tfsf"])
    if job.get("ade"):
        engine.configureLorentzADE(job["ade"])
    if job.get("pbc"):
        engine.configurePBC(job["pbc"])
    if job.get("nf2ff"):
        engine.configureNF2FFAccumulation(job["nf2ff"])
    probes = job.get("probes") or []
    slices = None
    if probes:
        idx, slices = opgen.build_gather_indices(probes, job["grid"])
        interval = probes[0]["processInterval"]
        max_samples = int(math.ceil(job["maxTS"] / interval)) + 1
        engine.configureProbeGatherBuffered(idx, maxSamples=max_samples, sampleInterval=interval)
    return slices


def run(engine, job, batch=100, on_energy=None):
    """The orchestrator's stepping loop (sim-engine.mjs:640-681): iterate in
    batches, check the lagged energy every 100 steps against endCrit."""
    slices = configure(engine, job)
    total, max_e = 0, 0.0
    end = job.get("endCrit", 0.0) or 0.0
    while total < job["maxTS"]:
        n = min(batch, job["maxTS"] - total)
        engine.iterate(n)
        total += n
        if total % 100 < n:
            e = engine.computeEnergy()
            if on_energy:
                on_energy(total, e)
            max_e = max(max_e, e)
            if end > 0 and max_e > 0 and e / max_e <= end:
                break
    return total, slices


def probe_series(engine, job, slices):
    """Read the probe ring and integrate (sim-engine.mjs:683-696): (num_samples, num_probes)."""
    r = engine.readProbeGatherBuffered()
    if r is None:
        return np.zeros((0, len(job["probes"])))
    g = np.asarray(r["data"]).reshape(r["numSamples"], r["stride"])
    return opgen.probe_integrals(g, job["probes"], slices)


def far_field_summary(engine, job, freq_index=0, dtheta=3.0, dphi=5.0, far_field_fn=None):
    """The orchestrator's NF2FF post-processing (sim-engine.mjs:725-806):
    far field on a theta x phi grid (3 and 5 degrees as the Node runner),
    radiated power through the surface, Dmax = 4 pi P_max r^2 / P_rad.
    far_field_fn(accE, accH, meta, theta, phi, freq) replaces the engine's
    far-field kernel (tests pass the f64 oracle)."""
    theta = np.deg2rad(np.arange(0.0, 180.0 + 1e-9, dtheta)).astype(np.float32)
    phi = np.deg2rad(np.arange(0.0, 360.0 + 1e-9, dphi)).astype(np.float32)
    acc = engine.readNF2FFAccumulation(True)
    meta = job["nf2ff_meta"]
    freq = job["nf2ff_freqs"][freq_index]
    if far_field_fn is None:
        out = engine.computeNF2FFfarField(dict(pointMeta=meta, theta=theta, phi=phi, center=[0, 0, 0], frequency=freq,
                                               radius=1.0, numPoints=job["nf2ff"]["numPoints"],
                                               freqIndex=freq_index)).reshape(-1, 5).astype(np.float64)
    else:
        out = far_field_fn(acc["accumE"][freq_index], acc["accumH"][freq_index], meta, theta, phi, freq)
    p_max = float(out[:, 0].max())
    prad = opgen.rad_power(acc["accumE"][freq_index], acc["accumH"][freq_index], meta)
    dmax = p_max * 4 * math.pi / prad if prad > 0 else 0.0
    return {"freqHz": freq, "P_max": p_max, "P_rad": prad, "Dmax": dmax,
            "DmaxdBi": 10 * math.log10(max(dmax, 1e-15)), "pattern": out}


def run_probe_job(engine, job):
    """Run a probe-only job; returns the first probe's series (with t = 0 if the
    job's reference data starts there)."""
    _, slices = run(engine, job, batch=job.get("batch", 100))
    v = probe_series(engine, job, slices)[:, 0]
    if job.get("include_t0"):
        v = np.concatenate([[0.0], v])
    return v


def slab_1d(medium=None, delta=0.5e-3, nz=2400, z_src=50, z_r=400, slab=(800, 840), z_t=1200, steps=4700,
            f0=8e9, fc=6e9):
    """Plane wave through a dispersive slab, for checking the ADE apply step
    against the analytic single-pole response.  A 4 x 4 x `nz` grid with
    periodic x and y (configurePBC: fields stay uniform across the period)
    and Mur on the z faces; an x-polarised soft source (Gaussian f0 +- fc) on
    the plane z_src; the slab fills the E edges at nodes slab[0] .. slab[1]-1
    (dual cells, thickness (slab[1]-slab[0]) * delta).  medium: None
    (vacuum), ("drude", omega_p, gamma) or ("lorentz", d_eps, omega_0,
    delta).  probe_idx: Ex field indices at z_r (before the slab) and z_t
    (after it), sampled every step."""
    grid = (4, 4, nz)
    Nx, Ny, Nz = grid
    mesh = opgen.Mesh(*[opgen.uniform_lines(n, delta) for n in grid])
    dT = opgen.cfl_dt(mesh)
    vv, vi, ii, iv = opgen.operator_dense(mesh, dT, bc=(-1, -1, -1, -1, 0, 0))
    job = dict(name="slab_1d", grid=list(grid), dT=dT, maxTS=steps, endCrit=0.0, mesh=mesh)
    if medium is not None:
        z1, z2 = slab
        cells = np.array([x * Ny * Nz + y * Nz + z for x in range(Nx) for y in range(Ny) for z in range(z1, z2)],
                         np.uint32)
        xs, ys, zs = cells // (Ny * Nz), (cells // Nz) % Ny, cells % Nz
        dirs, lor = [], medium[0] == "lorentz"
        for n in range(3):
            if lor:
                c = opgen.ade_lorentz(vv[n][xs, ys, zs], vi[n][xs, ys, zs], dT, *medium[1:])
            else:
                c = opgen.ade_drude(vv[n][xs, ys, zs], vi[n][xs, ys, zs], dT, *medium[1:])
            vv[n][xs, ys, zs] = c["vv"]
            vi[n][xs, ys, zs] = c["vi"]
            d = dict(dir=n, pos_idx=cells, v_int_ADE=c["v_int"].astype(np.float32),
                     v_ext_ADE=c["v_ext"].astype(np.float32))
            if lor:
                d["v_Lor_ADE"] = c["v_lor"].astype(np.float32)
            dirs.append(d)
        job["ade"] = dict(orders=[dict(numCells=len(cells), hasLorentz=lor, directions=dirs)], apply=True)
        job["ade_scheme"] = c["scheme"]
    job["coefficients"] = dict(vv=opgen.flat(vv), vi=opgen.flat(vi), ii=opgen.flat(ii), iv=opgen.flat(iv))
    sig = opgen.gauss_signal(f0, fc, dT, steps).astype(np.float32)
    # the source covers the periodic cells (x, y < 3; the last line of each
    # periodic axis is outside the period and stays quiet)
    pos = [x * Ny * Nz + y * Nz + z_src for x in range(Nx - 1) for y in range(Ny - 1)]
    job["excitation"] = dict(signal=sig, delay=[0] * len(pos), amp=[1.0] * len(pos), dir=[0] * len(pos), pos=pos,
                             period=0)
    job["mur"] = opgen.mur_dual(mesh, dT, [(2, "lo"), (2, "hi")])
    job["pbc"] = dict(axes=[dict(axis=0, phase=0.0), dict(axis=1, phase=0.0)])
    job["probe_idx"] = [1 * Ny * Nz + 1 * Nz + z_r, 1 * Ny * Nz + 1 * Nz + z_t]
    job["slab"] = slab
    job["z_r"], job["z_t"], job["delta"] = z_r, z_t, delta
    return job


def run_slab_1d(engine, job):
    """Configure `job` (slab_1d) on `engine`, run it, return the Ex series at
    the two probes (steps x 2)."""
    configure(engine, job)
    engine.configureProbeGatherBuffered(job["probe_idx"], maxSamples=job["maxTS"], sampleInterval=1)
    engine.iterate(job["maxTS"])
    r = engine.readProbeGatherBuffered()
    g = np.asarray(r["data"], np.float64).reshape(r["numSamples"], r["stride"])
    return g[:, 0::2]

