"""Operator generator: EC-FDTD update coefficients and extension inputs.

The reference obtains the engine's inputs from openEMS through its embind
getters (src/embind_api.cpp:207-681, :905-961): per-edge coefficients
vv/vi/ii/iv, the excitation list and waveform, UPML region arrays, Mur
regions and probe descriptors.  openEMS is not part of the reference tree, so
this module re-derives those inputs from the published method for
rectilinear meshes:

* equivalent-circuit FDTD: an E edge is a capacitor C = eps*A_dual/l_primal
  with conductance G = kappa*A_dual/l_primal, an H edge an inductor
  L = mu*A_primal/l_dual; vv = (1 - dT G/2C)/(1 + dT G/2C),
  vi = (dT/C)/(1 + dT G/2C), ii = 1, iv = dT/L;  eps and kappa are the
  area-weighted averages of the four cells around an edge;
* PEC: E edges whose centre lies in a metal box, and the tangential E of
  every outer face (the operator always starts from PEC walls), are zeroed;
* Gaussian pulse sampled at n*dT over 2*9/(2*pi*fc)/dT samples (the
  sampling that reproduces the native-openEMS fixtures);
* a curve excitation follows the staircase of mesh edges closest to the
  segment (openEMS FindPath), each edge excited with amplitude = its length;
* UPML after Gedney's two-step D/E form (Taflove & Hagness), polynomial
  grading; Mur first order with coefficient (c*dT - d)/(c*dT + d)
  (the reference checks this formula, tests/test_webgpu.mjs:2396-2418);
* TFSF corrections for an analytic plane wave, expressed in the reference's
  injection format {field_idx, delay_int, delay_frac, amp}
  (src/webgpu-fdtd.mjs:694-733).

All arithmetic is float64; arrays handed to the engine are float32.
"""
import math

import numpy as np

C0 = 299792458.0
MUE0 = 4e-7 * math.pi
EPS0 = 1.0 / (MUE0 * C0 * C0)
Z0 = math.sqrt(MUE0 / EPS0)


class Mesh:
    """Rectilinear mesh: three sorted arrays of line coordinates in metres."""

    def __init__(self, x, y, z):
        self.lines = [np.asarray(v, dtype=np.float64) for v in (x, y, z)]
        self.shape = tuple(len(v) for v in self.lines)

    @property
    def N(self):
        return self.shape[0] * self.shape[1] * self.shape[2]

    def dl(self, n):
        """Primal edge lengths along n (index i: line i -> i+1; last = 0)."""
        L = self.lines[n]
        d = np.zeros(len(L))
        d[:-1] = np.diff(L)
        return d

    def dd(self, n):
        """Dual edge lengths along n (half cells at the ends)."""
        d = self.dl(n)
        out = np.zeros(len(d))
        if len(d) == 1:
            return out
        out[0] = 0.5 * d[0]
        out[1:-1] = 0.5 * (d[:-2] + d[1:-1])
        out[-1] = 0.5 * d[-2]
        return out

    def snap(self, n, coord):
        """Index of the line nearest to coord (sim-engine.mjs snapToMeshIndex :338-349)."""
        return int(np.argmin(np.abs(self.lines[n] - coord)))


def uniform_lines(n, delta, origin=0.0):
    return origin + delta * np.arange(n, dtype=np.float64)


def graded_lines(span, dmin, dmax, ratio, fine_regions=()):
    """Lines over [0, span] with cell size dmin inside `fine_regions` and grown
    by at most `ratio` per cell up to dmax elsewhere."""
    # target size field evaluated greedily from left to right
    lines = [0.0]
    d = dmin
    def target(x):
        t = dmax
        for lo, hi in fine_regions:
            if lo - 1e-12 <= x <= hi + 1e-12:
                return dmin
            dist = min(abs(x - lo), abs(x - hi))
            # allowed size grows geometrically with distance from a fine region
            k = dmin
            acc = 0.0
            while acc + k < dist and k < dmax:
                acc += k
                k = min(k * ratio, dmax)
            t = min(t, k)
        return t
    while lines[-1] < span - 1e-12:
        x = lines[-1]
        d = min(target(x), d * ratio, span - x)
        d = max(d, min(dmin, span - x))
        lines.append(x + d)
    return np.asarray(lines)


def cfl_dt(mesh, factor=1.0):
    """Courant limit of the non-uniform Yee grid: min over cells of
    1/(c*sqrt(1/dx^2+1/dy^2+1/dz^2)) (each term is largest at the smallest step)."""
    s = sum(1.0 / np.min(np.diff(L)) ** 2 for L in mesh.lines if len(L) > 1)
    return factor / (C0 * math.sqrt(s))


def gauss_signal(f0, fc, dT, nTS=None):
    """Gaussian pulse sampled at t = n dT:
    signal[n] = cos(2 pi f0 (t - t0)) exp(-(2 pi fc t / 3 - 3)^2), t0 = 9/(2 pi fc),
    length = floor(2 t0 / dT) (cut to nTS).  This sampling reproduces the
    native-openEMS cavity fixture (tests/fixtures/engine_comparison) to a
    relative L2 of 7e-5; the alternative with sample 0 forced to zero and
    t = (n-1) dT misses it by 30 %."""
    t0 = 9.0 / (2 * math.pi * fc)
    L = int(2.0 * t0 / dT)
    if nTS is not None:
        L = min(L, int(nTS))
    t = np.arange(L, dtype=np.float64) * dT
    return np.cos(2 * math.pi * f0 * (t - t0)) * np.exp(-((2 * math.pi * fc * t / 3 - 3) ** 2))


def nyquist_interval(f_max, dT):
    """Probe process interval: a third of the Nyquist step count."""
    nyq = int(1.0 / (2.0 * f_max * dT))
    return max(1, nyq // 3)


def _line_dist(P, a, b):
    d = b - a
    LL = float(d @ d)
    foot = float((P - a) @ d) / LL
    fp = a + foot * d
    return foot, float(np.sqrt(((P - fp) ** 2).sum()))


def find_path(mesh, p1, p2):
    """Staircase of mesh edges from p1 to p2: at each node take the
    neighbouring node closest to the segment among those that advance along
    it.  Returns [(dir, (x, y, z) of the edge start)]."""
    a, b = np.asarray(p1, float), np.asarray(p2, float)
    s = [mesh.snap(n, a[n]) for n in range(3)]
    t = [mesh.snap(n, b[n]) for n in range(3)]
    node = lambda p: np.array([mesh.lines[n][p[n]] for n in range(3)])
    cur = list(s)
    cur_foot, _ = _line_dist(node(s), a, b)
    stop_foot, _ = _line_dist(node(t), a, b)
    path = []
    min_foot = cur_foot
    while min_foot < stop_foot:
        best = None
        for n in range(3):
            for step in (-1, 1):
                q = list(cur)
                q[n] += step
                if q[n] < 0 or q[n] >= mesh.shape[n]:
                    continue
                foot, dist = _line_dist(node(q), a, b)
                if foot > cur_foot and (best is None or dist < best[0]):
                    best = (dist, foot, n, step)
        if best is None:
            break
        _, min_foot, n, step = best
        start = list(cur) if step > 0 else [cur[i] - (1 if i == n else 0) for i in range(3)]
        path.append((n, tuple(start)))
        cur[n] += step
        cur_foot = min_foot
    return path


def _shift(a, axis, k):
    """out[i] = a[i + k] along axis (zero outside)."""
    out = np.zeros_like(a)
    n = a.shape[axis]
    if k >= 0:
        src = [slice(None)] * a.ndim
        dst = [slice(None)] * a.ndim
        src[axis] = slice(k, n)
        dst[axis] = slice(0, n - k)
    else:
        src = [slice(None)] * a.ndim
        dst = [slice(None)] * a.ndim
        src[axis] = slice(0, n + k)
        dst[axis] = slice(-k, n)
    out[tuple(dst)] = a[tuple(src)]
    return out


def edge_mask_in_box(mesh, n, lo, hi, tol=1e-12, xslice=None):
    """Bool (Nx,Ny,Nz) mask of E_n edges whose centre lies in [lo, hi]."""
    masks = []
    for ax in range(3):
        L = mesh.lines[ax]
        if ax == n:
            c = np.empty(len(L))
            c[:-1] = 0.5 * (L[:-1] + L[1:])
            c[-1] = np.inf
        else:
            c = L
        m = (c >= min(lo[ax], hi[ax]) - tol) & (c <= max(lo[ax], hi[ax]) + tol)
        if ax == 0 and xslice is not None:
            m = m[xslice]
        masks.append(m)
    return masks[0][:, None, None] & masks[1][None, :, None] & masks[2][None, None, :]


def cell_mask_in_box(mesh, lo, hi):
    """Bool (Nx-1,Ny-1,Nz-1) mask of cells whose centre lies in [lo, hi]."""
    ms = []
    for ax in range(3):
        L = mesh.lines[ax]
        c = 0.5 * (L[:-1] + L[1:])
        ms.append((c >= min(lo[ax], hi[ax])) & (c <= max(lo[ax], hi[ax])))
    return ms[0][:, None, None] & ms[1][None, :, None] & ms[2][None, None, :]


def operator_dense(mesh, dT, eps_r=None, kappa=None, pec_edges=None, lumped_g=None, bc=(0, 0, 0, 0, 0, 0),
                   x0=0, x1=None):
    """vv, vi, ii, iv as (3, nx, Ny, Nz) float64 over x-planes [x0, x1).

    eps_r, kappa: per-cell (Nx-1, Ny-1, Nz-1) arrays (None = vacuum, lossless)
    pec_edges:    list of 3 bool arrays (Nx, Ny, Nz) of metal E edges, or None
    lumped_g:     list of 3 float arrays (Nx, Ny, Nz) of extra edge conductance
    bc:           xmin xmax ymin ymax zmin zmax; -1 marks a periodic face (no PEC)
    """
    Nx, Ny, Nz = mesh.shape
    x1 = Nx if x1 is None else x1
    nx = x1 - x0
    dl = [mesh.dl(n) for n in range(3)]
    dd = [mesh.dd(n) for n in range(3)]
    shp = (nx, Ny, Nz)
    vv = np.zeros((3,) + shp)
    vi = np.zeros((3,) + shp)
    ii = np.zeros((3,) + shp)
    iv = np.zeros((3,) + shp)
    # cell arrays padded by one cell on every side (zero outside the grid)
    cx0, cx1 = max(x0 - 1, 0), min(x1, Nx - 1)

    def padded(a, default):
        out = np.zeros((nx + 1, Ny + 1, Nz + 1))
        if a is None:
            src = np.full((cx1 - cx0, Ny - 1, Nz - 1), default)
        else:
            src = a[cx0:cx1]
        # padded[i+1] holds cell (x0 + i)
        off = cx0 - (x0 - 1)
        out[off:off + src.shape[0], 1:Ny, 1:Nz] = src
        return out
    eps_p = padded(eps_r, 1.0)
    kap_p = padded(kappa, 0.0)
    X = np.arange(x0, x1)
    for n in range(3):
        nP, nPP = (n + 1) % 3, (n + 2) % 3
        # quarter dual areas of the 4 cells around the edge; cell (pos + a) along nP/nPP
        idx = [np.arange(x0, x1), np.arange(Ny), np.arange(Nz)]
        half = [0.5 * dl[k] for k in range(3)]
        C = np.zeros(shp)
        G = np.zeros(shp)
        for a_ in (-1, 0):
            for b_ in (-1, 0):
                off = [0, 0, 0]
                off[nP] = a_
                off[nPP] = b_
                # quarter area: half primal length of the cell in nP and nPP
                qa_nP = np.where((idx[nP] + a_ >= 0), half[nP][np.clip(idx[nP] + a_, 0, None)], 0.0)
                qa_nPP = np.where((idx[nPP] + b_ >= 0), half[nPP][np.clip(idx[nPP] + b_, 0, None)], 0.0)
                shape_nP = [1, 1, 1]
                shape_nP[nP] = -1
                shape_nPP = [1, 1, 1]
                shape_nPP[nPP] = -1
                qa = qa_nP.reshape(shape_nP) * qa_nPP.reshape(shape_nPP)
                # cell (x+off0, y+off1, z+off2) sits at padded index +1
                sl = tuple(slice(1 + off[k], 1 + off[k] + shp[k]) for k in range(3))
                C = C + eps_p[sl] * qa
                G = G + kap_p[sl] * qa
        L_n = dl[n][idx[n]]
        shape_n = [1, 1, 1]
        shape_n[n] = -1
        L_n = L_n.reshape(shape_n)
        with np.errstate(divide="ignore", invalid="ignore"):
            Cc = np.where(L_n > 0, EPS0 * C / L_n, 0.0)
            Gc = np.where(L_n > 0, G / L_n, 0.0)
            if lumped_g is not None:
                Gc = Gc + lumped_g[n][x0:x1]
            a = dT * Gc / (2 * Cc)
            vvn = np.where(Cc > 0, (1 - a) / (1 + a), 0.0)
            vin = np.where(Cc > 0, (dT / Cc) / (1 + a), 0.0)
        # metal edges
        if pec_edges is not None:
            m = pec_edges(n, x0, x1) if callable(pec_edges) else pec_edges[n][x0:x1]
            vvn[m] = 0.0
            vin[m] = 0.0
        vv[n] = vvn
        vi[n] = vin
        # H edge: length = dual along n, area = primal nP x nPP
        Ld = dd[n][idx[n]].reshape(shape_n)
        A = dl[nP][idx[nP]].reshape(shape_nP) * dl[nPP][idx[nPP]].reshape(shape_nPP)
        A = np.broadcast_to(A, shp)
        with np.errstate(divide="ignore", invalid="ignore"):
            ivn = np.where(A > 0, dT * Ld / (MUE0 * A), 0.0)
        iv[n] = np.broadcast_to(ivn, shp)
        ii[n] = np.where(A > 0, 1.0, 0.0)
    # PEC walls: tangential E on every outer face that is not periodic
    for n in range(3):
        nP, nPP = (n + 1) % 3, (n + 2) % 3
        for side, pos in ((0, 0), (1, mesh.shape[n] - 1)):
            if bc[2 * n + side] == -1:
                continue
            for c in (nP, nPP):
                sl = [slice(None)] * 3
                if n == 0:
                    if not (x0 <= pos < x1):
                        continue
                    sl[0] = pos - x0
                else:
                    sl[n] = pos
                vv[c][tuple(sl)] = 0.0
                vi[c][tuple(sl)] = 0.0
        # E_n beyond the last line lies outside the domain
        sl = [slice(None)] * 3
        if n == 0:
            if x0 <= Nx - 1 < x1:
                sl[0] = Nx - 1 - x0
                vv[0][tuple(sl)] = 0.0
                vi[0][tuple(sl)] = 0.0
        else:
            sl[n] = mesh.shape[n] - 1
            vv[n][tuple(sl)] = 0.0
            vi[n][tuple(sl)] = 0.0
    return vv, vi, ii, iv


# ---------------------------------------------------------------------------
# Dispersive media: one Drude or Lorentz pole per E edge, as the inputs of
# the engine's ADE extension (configureLorentzADE, src/webgpu-engine.mjs:1358)
# with its apply step on.
# ---------------------------------------------------------------------------
# The reference has no generator for these inputs (no embind getter exists),
# so they are derived here from the equivalent circuit: a dispersive E edge
# carries, beside its capacitor C and conductance G, a branch current J
# through an inductor L and resistor R (Drude: L = 1/(omega_p^2 C0),
# R = gamma L) or through L, R and a capacitor C_L in series (Lorentz:
# L = 1/(d_eps omega_0^2 C0), R = delta L, C_L = d_eps C0), C0 = eps0 A/l the
# edge's vacuum capacitance.  The engine's state s is the branch current
# scaled to volts (the term the apply step subtracts from V after the core
# update V <- vv V + vi curl I); its update s <- v_int s + v_ext (V - lor),
# lor <- lor + v_Lor s (src/webgpu-fdtd.mjs:405-454) runs before the core
# update on the current V.
#
# "explicit": J at half steps, the branch equation centred on V^n (second
# order; the coupling is explicit, stable while (omega_p dT)^2 / eps_r stays
# well below 4): v_int = (1 - R dT/2L)/(1 + R dT/2L),
# v_ext = vi dT / (L (1 + R dT/2L)), Lorentz v_Lor = dT / (C_L vi); the core
# coefficients are unchanged.
# "implicit": for stiff poles (a good conductor at microwave steps,
# omega_p dT >> 1) the branch current is advanced with V^{n+1} (backward
# Euler in the branch, L-stable), which folds into the core coefficients:
# with a = 1/(1 + R dT/L), b = dT/(L + R dT):  vv' = vv/(1 + b vi),
# vi' = vi/(1 + b vi), v_int = a, v_ext = a b vi/(1 + b vi).  (With the
# trapezoidal loss of the core update, 1/vi = C/dT + G/2 and vv/vi =
# C/dT - G/2.)


def _edge_c0(vv, vi, dT, eps_r):
    """Vacuum capacitance C0 = C/eps_r of E edges from their core coefficients
    (vv = (1-g)/(1+g), vi = (dT/C)/(1+g), g = dT G / 2C), and the mask of
    edges that have an update (vi > 0; metal edges and edges outside the
    domain get no dispersive coupling: C0 is set to 1 there and their
    coefficients are zeroed by the callers)."""
    vv = np.asarray(vv, np.float64)
    vi = np.asarray(vi, np.float64)
    live = vi > 0
    g = (1.0 - vv) / (1.0 + vv)
    c0 = np.ones(vv.shape)
    c0[live] = dT / (vi[live] * (1.0 + g[live])) / eps_r
    return c0, live


def ade_drude(vv, vi, dT, omega_p, gamma, eps_r=1.0, scheme="auto"):
    """ADE inputs of a single-pole Drude medium on E edges with core
    coefficients vv, vi (arrays, float64): dict(vv, vi, v_int, v_ext, scheme).
    scheme "auto" picks "explicit" while (omega_p dT)^2 / eps_r < 1, else
    "implicit" (see above)."""
    vv = np.asarray(vv, np.float64)
    vi = np.asarray(vi, np.float64)
    c0, live = _edge_c0(vv, vi, dT, eps_r)
    L = 1.0 / (omega_p * omega_p * c0)
    if scheme == "auto":
        scheme = "explicit" if (omega_p * dT) ** 2 / eps_r < 1.0 else "implicit"
    if scheme == "explicit":
        h = 1.0 + gamma * dT / 2.0
        return dict(vv=vv, vi=vi, v_int=np.where(live, (1.0 - gamma * dT / 2.0) / h, 0.0),
                    v_ext=np.where(live, vi * dT / (L * h), 0.0), scheme=scheme)
    a = 1.0 / (1.0 + gamma * dT)
    b = dT / (L * (1.0 + gamma * dT))
    q = 1.0 + b * vi
    return dict(vv=np.where(live, vv / q, vv), vi=np.where(live, vi / q, vi), v_int=np.where(live, a, 0.0),
                v_ext=np.where(live, a * b * vi / q, 0.0), scheme="implicit")


def ade_lorentz(vv, vi, dT, d_eps, omega_0, delta, eps_r=1.0):
    """ADE inputs of a single-pole Lorentz medium (explicit scheme, see
    above): dict(vv, vi, v_int, v_ext, v_lor, scheme)."""
    vv = np.asarray(vv, np.float64)
    vi = np.asarray(vi, np.float64)
    c0, live = _edge_c0(vv, vi, dT, eps_r)
    L = 1.0 / (d_eps * omega_0 * omega_0 * c0)
    CL = d_eps * c0
    h = 1.0 + delta * dT / 2.0
    v_lor = np.zeros(vv.shape)
    v_lor[live] = dT / (CL[live] * vi[live])
    return dict(vv=vv, vi=vi, v_int=np.where(live, (1.0 - delta * dT / 2.0) / h, 0.0),
                v_ext=np.where(live, vi * dT / (L * h), 0.0), v_lor=v_lor, scheme="explicit")


def drude_eps(f, omega_p, gamma, eps_inf=1.0):
    """Relative permittivity of a Drude pole at frequency f (e^{j omega t})."""
    w = 2 * math.pi * np.asarray(f, np.float64)
    return eps_inf - omega_p ** 2 / (w * (w - 1j * gamma))


def lorentz_eps(f, d_eps, omega_0, delta, eps_inf=1.0):
    """Relative permittivity of a Lorentz pole at frequency f (e^{j omega t})."""
    w = 2 * math.pi * np.asarray(f, np.float64)
    return eps_inf + d_eps * omega_0 ** 2 / (omega_0 ** 2 - w * w + 1j * w * delta)


def slab_rt(f, eps, d):
    """Normal-incidence reflection and transmission of a slab of relative
    permittivity eps(f) and thickness d in vacuum (e^{j omega t}; T
    referred to the slab's two faces)."""
    k0 = 2 * math.pi * np.asarray(f, np.float64) / C0
    n = np.sqrt(np.asarray(eps, np.complex128))
    n = np.where(n.imag > 0, -n, n)                 # decaying branch for e^{j omega t}
    r = (1 - n) / (1 + n)
    p = np.exp(-1j * k0 * n * d)
    R = r * (1 - p * p) / (1 - r * r * p * p)
    T = (1 - r * r) * p / (1 - r * r * p * p)
    return R, T


def flat(a):
    """(3, Nx, Ny, Nz) -> NIJK float32 vector."""
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1)


_HASH_K = np.array([0x9E3779B97F4A7C15, 0xC2B2AE3D27D4EB4F, 0x165667B19E3779F9, 0xD6E8FEB86659FD93,
                    0xFF51AFD7ED558CCD, 0xC4CEB9FE1A85EC53, 0x94D049BB133111EB, 0xBF58476D1CE4E5B9,
                    0x2545F4914F6CDD1D, 0x5851F42D4C957F2D, 0x14057B7EF767814F, 0xA24BAED4963EE407], dtype=np.uint64)


class MaterialTable:
    """Incremental dedup of 12-float coefficient rows into (mat, table)."""

    def __init__(self):
        self.keys = {}
        self.rows = []

    def add(self, rows):
        """rows: (n, 12) float32 -> (n,) uint32 ids."""
        bits = np.ascontiguousarray(rows, dtype=np.float32).view(np.uint32).astype(np.uint64)
        h = (bits * _HASH_K[None, :]).sum(axis=1, dtype=np.uint64)
        h ^= h >> np.uint64(29)
        uh, first, inv = np.unique(h, return_index=True, return_inverse=True)
        ids = np.empty(len(uh), np.uint32)
        for j, (k, f) in enumerate(zip(uh.tolist(), first.tolist())):
            v = self.keys.get(k)
            if v is None:
                v = len(self.rows)
                self.keys[k] = v
                self.rows.append(np.array(rows[f], dtype=np.float32))
            ids[j] = v
        out = ids[inv]
        # hash collisions would map different rows to one id: verify exactly
        tab = self.table()
        if not np.array_equal(tab[out].view(np.uint32), np.ascontiguousarray(rows, np.float32).view(np.uint32)):
            raise RuntimeError("coefficient row hash collision")
        return out

    def table(self):
        return np.array(self.rows, dtype=np.float32).reshape(-1, 12)


def to_indexed(vv, vi, ii, iv, mt=None):
    """Dense (3, nx, Ny, Nz) arrays -> (mat uint32 of nx*Ny*Nz, MaterialTable)."""
    mt = mt or MaterialTable()
    rows = np.stack([vv[0], vv[1], vv[2], vi[0], vi[1], vi[2], ii[0], ii[1], ii[2], iv[0], iv[1], iv[2]], axis=-1)
    rows = rows.astype(np.float32).reshape(-1, 12)
    return mt.add(rows), mt


def dense_from_indexed(mat, table):
    """Inverse of to_indexed: NIJK vv, vi, ii, iv float32 vectors."""
    t = np.asarray(table, np.float32).reshape(-1, 12)[np.asarray(mat)]
    return [np.ascontiguousarray(t[:, 3 * a:3 * a + 3].T).reshape(-1) for a in range(4)]


# ---------------------------------------------------------------------------
# UPML (Gedney two-step form) and Mur
# ---------------------------------------------------------------------------
def field_pos(mesh, n, field, axis):
    """Coordinates along `axis` of component n of E ('E') or H ('H') at each line index."""
    L = mesh.lines[axis]
    half = np.empty(len(L))
    half[:-1] = 0.5 * (L[:-1] + L[1:])
    half[-1] = L[-1] + 0.5 * (L[-1] - L[-2]) if len(L) > 1 else L[-1]
    staggered = (axis == n) if field == "E" else (axis != n)
    return half if staggered else L


def pml_sigma(mesh, axis, width_lo, width_hi, order=3, R0=1e-6):
    """Conductivity profile function sigma(coord) for UPML slabs of `width`
    cells at the low/high end of `axis` (polynomial grading, sigma_max from
    the target reflection R0: -(m+1) ln R0 / (2 Z0 W))."""
    L = mesh.lines[axis]
    lo_if = L[width_lo] if width_lo else None
    hi_if = L[len(L) - 1 - width_hi] if width_hi else None

    def sig(c):
        s = np.zeros_like(c)
        if width_lo:
            W = L[width_lo] - L[0]
            smax = -(order + 1) * math.log(R0) / (2 * Z0 * W)
            d = np.clip((lo_if - c) / W, 0, None)
            s = s + smax * d ** order
        if width_hi:
            W = L[-1] - L[len(L) - 1 - width_hi]
            smax = -(order + 1) * math.log(R0) / (2 * Z0 * W)
            d = np.clip((c - hi_if) / W, 0, None)
            s = s + smax * d ** order
        return s
    return sig


def upml_apply(mesh, dT, regions_boxes, sig_fns, vv=None, vi=None, ii=None, iv=None, x0=0, build=True):
    """Build UPML region arrays and rewrite the core coefficients inside them.

    regions_boxes: list of (start[3], num[3]) line-index boxes (disjoint)
    sig_fns:       sigma(coord) per axis (None = no grading along that axis)
    vv..iv:        (3, nx, Ny, Nz) dense core coefficients over x-planes
                   [x0, x0+nx), modified in place for cells in the regions.
    For E component n (nP, nPP the next two axes), with a_k = sigma_k dT / (2 eps0):
      D-step (core):  vv' = (1 - a_nP)/(1 + a_nP), vi' = vi/(1 + a_nP)
      E-step (UPML):  vv = (1 - a_nPP)/(1 + a_nPP), vvfo = (1 - a_n)/(1 + a_nPP),
                      vvfn = (1 + a_n)/(1 + a_nPP)
    and the same for H with the conductivities at the H positions.
    """
    regions = []
    nx = vv.shape[1] if vv is not None else 0
    for start, num in regions_boxes:
        sl = [slice(start[k], start[k] + num[k]) for k in range(3)]
        arrs = {k: np.zeros((3,) + tuple(num)) for k in ("vv", "vvfo", "vvfn", "ii", "iifo", "iifn")}
        for field, core_a, core_b, names in (("E", vv, vi, ("vv", "vvfo", "vvfn")),
                                             ("H", ii, iv, ("ii", "iifo", "iifn"))):
            for n in range(3):
                a = []
                for ax in range(3):
                    if sig_fns[ax] is None:
                        a.append(np.zeros(num[ax]))
                    else:
                        c = field_pos(mesh, n, field, ax)[sl[ax]]
                        a.append(sig_fns[ax](c) * dT / (2 * EPS0))
                shp = [(num[0], 1, 1), (1, num[1], 1), (1, 1, num[2])]
                A = [a[k].reshape(shp[k]) for k in range(3)]
                nP, nPP = (n + 1) % 3, (n + 2) % 3
                one = np.ones(tuple(num))
                if build:
                    arrs[names[0]][n] = (1 - A[nPP]) / (1 + A[nPP]) * one
                    arrs[names[1]][n] = (1 - A[n]) / (1 + A[nPP]) * one
                    arrs[names[2]][n] = (1 + A[n]) / (1 + A[nPP]) * one
                # core D-step coefficients inside the region (x-planes held by this chunk)
                gx0, gx1 = max(start[0], x0), min(start[0] + num[0], x0 + nx)
                if core_a is not None and gx0 < gx1:
                    lx = slice(gx0 - start[0], gx1 - start[0])
                    cs = (n, slice(gx0 - x0, gx1 - x0), sl[1], sl[2])
                    anp = (A[nP] * one)[lx]
                    live = core_b[cs] != 0          # metal / outside edges stay zero
                    core_a[cs] = np.where(live, (1 - anp) / (1 + anp), core_a[cs])
                    core_b[cs] = np.where(live, core_b[cs] / (1 + anp), core_b[cs])
        if build:
            regions.append(dict(startPos=list(start), numLines=list(num),
                                **{k: np.ascontiguousarray(v, np.float32).reshape(-1) for k, v in arrs.items()}))
    return regions


def mur_dual(mesh, dT, faces, ranges=None):
    """Dual-component Mur config for the given faces: (axis, 'lo'|'hi').
    Coefficient (c dT - d)/(c dT + d) with d the spacing to the next line.
    ranges[a] = (first, last) line index limits the tangential extent along
    axis a (used to keep Mur faces out of UPML slabs on the other axes)."""
    Nx, Ny, Nz = mesh.shape
    nl = mesh.shape
    out = {k: [] for k in ("coeff_nyP", "coeff_nyPP", "normal_idx_nyP", "shifted_idx_nyP",
                            "normal_idx_nyPP", "shifted_idx_nyPP")}
    cs = Nx * Ny * Nz
    for ny, side in faces:
        L = mesh.lines[ny]
        line, shift = (0, 1) if side == "lo" else (nl[ny] - 1, nl[ny] - 2)
        d = abs(L[shift] - L[line])
        coeff = (C0 * dT - d) / (C0 * dT + d)
        P, PP = (ny + 1) % 3, (ny + 2) % 3
        rg = [(0, nl[a] - 1) if ranges is None or ranges[a] is None else ranges[a] for a in range(3)]
        i0, i1 = np.meshgrid(np.arange(rg[P][0], rg[P][1] + 1), np.arange(rg[PP][0], rg[PP][1] + 1), indexing="xy")
        pos = [None, None, None]
        pos[ny] = np.full(i0.size, line)
        pos[P] = i0.ravel()
        pos[PP] = i1.ravel()
        flat_n = pos[0] * Ny * Nz + pos[1] * Nz + pos[2]
        pos[ny] = np.full(i0.size, shift)
        flat_s = pos[0] * Ny * Nz + pos[1] * Nz + pos[2]
        out["normal_idx_nyP"].append(P * cs + flat_n)
        out["shifted_idx_nyP"].append(P * cs + flat_s)
        out["normal_idx_nyPP"].append(PP * cs + flat_n)
        out["shifted_idx_nyPP"].append(PP * cs + flat_s)
        out["coeff_nyP"].append(np.full(i0.size, coeff))
        out["coeff_nyPP"].append(np.full(i0.size, coeff))
    return {k: (np.concatenate(v).astype(np.float32) if k.startswith("coeff") else np.concatenate(v).astype(np.uint32))
            for k, v in out.items()}


# ---------------------------------------------------------------------------
# TFSF plane wave
# ---------------------------------------------------------------------------
# curl stencils: E_n at node p uses H terms (comp, offset, sign); H_n uses E terms
_E_CURL = {0: [(2, (0, 0, 0), 1), (2, (0, -1, 0), -1), (1, (0, 0, 0), -1), (1, (0, 0, -1), 1)],
           1: [(0, (0, 0, 0), 1), (0, (0, 0, -1), -1), (2, (0, 0, 0), -1), (2, (-1, 0, 0), 1)],
           2: [(1, (0, 0, 0), 1), (1, (-1, 0, 0), -1), (0, (0, 0, 0), -1), (0, (0, -1, 0), 1)]}
_H_CURL = {0: [(2, (0, 0, 0), 1), (2, (0, 1, 0), -1), (1, (0, 0, 0), -1), (1, (0, 0, 1), 1)],
           1: [(0, (0, 0, 0), 1), (0, (0, 0, 1), -1), (2, (0, 0, 0), -1), (2, (1, 0, 0), 1)],
           2: [(1, (0, 0, 0), 1), (1, (1, 0, 0), -1), (0, (0, 0, 0), -1), (0, (0, 1, 0), 1)]}


def tfsf_plane_wave(mesh, dT, lo, hi, k_hat, e_hat, coef_at, signal_len, E0=1.0):
    """TFSF injection points for a plane wave E = E0 e_hat g(t - k.(r-r0)/c)
    on the box of nodes [lo, hi] (total field inside).

    coef_at(kind, comp, flat_cell_idx) -> vi (kind 'E') or iv (kind 'H') of
    those edges.  Returns the reference's configureTFSF point lists."""
    k_hat = np.asarray(k_hat, float) / np.linalg.norm(k_hat)
    e_hat = np.asarray(e_hat, float)
    h_hat = np.cross(k_hat, e_hat)
    Nx, Ny, Nz = mesh.shape
    cs = Nx * Ny * Nz
    lo, hi = np.asarray(lo), np.asarray(hi)
    # reference point: the box corner first reached by the wave, 2 cells upstream
    corners = np.array([[mesh.lines[a][[lo, hi][c[a]][a]] for a in range(3)] for c in
                        [(i, j, k) for i in (0, 1) for j in (0, 1) for k in (0, 1)]])
    dmin = np.min(np.diff(mesh.lines[0]))
    r0 = corners[np.argmin(corners @ k_hat)] - 2 * dmin * k_hat
    dl = [mesh.dl(n) for n in range(3)]
    dd = [mesh.dd(n) for n in range(3)]

    def inside_E(n, p):
        ok = np.ones(p[0].shape, bool)
        for a in range(3):
            top = hi[a] - 1 if a == n else hi[a]
            ok &= (p[a] >= lo[a]) & (p[a] <= top)
        return ok

    def inside_H(n, p):
        ok = np.ones(p[0].shape, bool)
        for a in range(3):
            top = hi[a] if a == n else hi[a] - 1
            ok &= (p[a] >= lo[a]) & (p[a] <= top)
        return ok

    def coords(kind, n, p):
        r = []
        for a in range(3):
            c = field_pos(mesh, n, kind, a)
            r.append(c[np.clip(p[a], 0, len(c) - 1)])
        return np.stack(r, axis=-1)

    # candidate nodes: the union of six slabs (thickness 3) around the box faces
    span = [np.arange(max(lo[a] - 2, 0), min(hi[a] + 3, mesh.shape[a])) for a in range(3)]
    flats = []
    for a in range(3):
        for c in (lo[a], hi[a]):
            rr = list(span)
            rr[a] = np.arange(max(c - 1, 0), min(c + 2, mesh.shape[a]))
            g = np.meshgrid(*rr, indexing="ij")
            flats.append((g[0] * Ny + g[1]).astype(np.int64).ravel() * Nz + g[2].ravel())
    flat_all = np.unique(np.concatenate(flats))
    P = [flat_all // (Ny * Nz), (flat_all // Nz) % Ny, flat_all % Nz]
    vpts, cpts = [], []
    for n in range(3):
        # E edges inside whose curl reads an H edge outside
        inE = inside_E(n, P)
        pe = [p[inE] for p in P]
        for (hc, off, s) in _E_CURL[n]:
            q = [pe[a] + off[a] for a in range(3)]
            valid = np.ones(pe[0].shape, bool)
            for a in range(3):
                valid &= (q[a] >= 0) & (q[a] < mesh.shape[a])
            out = valid & ~inside_H(hc, q)
            if not out.any() or abs(h_hat[hc]) < 1e-12:
                continue
            pe_o = [x[out] for x in pe]
            q_o = [x[out] for x in q]
            rH = coords("H", hc, q_o)
            tau = (rH - r0) @ k_hat / C0
            D = tau / dT - 0.5
            flat = pe_o[0] * Ny * Nz + pe_o[1] * Nz + pe_o[2]
            ampl = coef_at("E", n, flat) * s * (E0 / Z0) * h_hat[hc] * dd[hc][q_o[hc]]
            vpts.append((n * cs + flat, D, ampl))
        # H edges outside whose curl reads an E edge inside
        outH = ~inside_H(n, P)
        ph = [p[outH] for p in P]
        for (ec, off, s) in _H_CURL[n]:
            q = [ph[a] + off[a] for a in range(3)]
            valid = np.ones(ph[0].shape, bool)
            for a in range(3):
                valid &= (q[a] >= 0) & (q[a] < mesh.shape[a])
            inn = valid & inside_E(ec, q)
            if not inn.any() or abs(e_hat[ec]) < 1e-12:
                continue
            ph_i = [x[inn] for x in ph]
            q_i = [x[inn] for x in q]
            rE = coords("E", ec, q_i)
            tau = (rE - r0) @ k_hat / C0
            D = tau / dT - 1.0
            flat = ph_i[0] * Ny * Nz + ph_i[1] * Nz + ph_i[2]
            ampl = coef_at("H", n, flat) * (-s) * E0 * e_hat[ec] * dl[ec][q_i[ec]]
            cpts.append((n * cs + flat, D, ampl))

    def pack(lst):
        if not lst:
            return dict(field_idx=np.zeros(0, np.uint32), delay_int=np.zeros(0, np.uint32),
                        delay_frac=np.zeros(0, np.float32), amp=np.zeros(0, np.float32))
        idx = np.concatenate([a for a, _, _ in lst])
        D = np.concatenate([b for _, b, _ in lst])
        A = np.concatenate([c for _, _, c in lst])
        keep = A != 0
        idx, D, A = idx[keep], D[keep], A[keep]
        di = np.ceil(D)
        return dict(field_idx=idx.astype(np.uint32), delay_int=di.astype(np.uint32),
                    delay_frac=(di - D).astype(np.float32), amp=A.astype(np.float32))
    return pack(vpts), pack(cpts)


def tfsf_points_list(cols):
    """Column dict -> the reference's list of point objects."""
    return [dict(field_idx=int(a), delay_int=int(b), delay_frac=float(c), amp=float(d)) for a, b, c, d in
            zip(cols["field_idx"], cols["delay_int"], cols["delay_frac"], cols["amp"])]


# ---------------------------------------------------------------------------
# NF2FF surface (sim-engine.mjs:351-472, edge lengths :577-591)
# ---------------------------------------------------------------------------
def nf2ff_box(mesh, lo, hi):
    """Surface points, per-point metadata and edge lengths of the NF2FF box
    whose six faces sit on lines lo[a] and hi[a]."""
    pts, metas = [], []
    for d in range(3):
        for face, sign in ((lo[d], -1.0), (hi[d], 1.0)):
            rngs = [np.arange(lo[a], hi[a] + 1) if a != d else np.array([face]) for a in range(3)]
            g = np.meshgrid(*rngs, indexing="ij")
            p = np.stack([x.ravel() for x in g], axis=-1)
            pts.append(p)
            nP, nPP = (d + 1) % 3, (d + 2) % 3
            face_lines = [mesh.lines[a][rngs[a]] for a in range(3)]

            def el(lines):
                N = len(lines)
                L = np.zeros(N)
                if N == 1:
                    return L
                L[0] = 0.5 * abs(lines[1] - lines[0])
                L[1:-1] = 0.5 * np.abs(lines[2:] - lines[:-2])
                L[-1] = 0.5 * abs(lines[-1] - lines[-2])
                return L
            lp, lpp = el(face_lines[nP]), el(face_lines[nPP])
            m = np.zeros((len(p), 8))
            for a in range(3):
                m[:, a] = mesh.lines[a][p[:, a]]
            m[:, 3] = d
            m[:, 4] = sign
            m[:, 5] = lp[p[:, nP] - rngs[nP][0]] * lpp[p[:, nPP] - rngs[nPP][0]]
            metas.append(m)
    pts = np.concatenate(pts).astype(np.uint32)
    meta = np.concatenate(metas).astype(np.float32)
    primal, dual = [], []
    for n in range(3):
        L = mesh.lines[n]
        N = len(L)
        e = np.zeros(N)
        e[:-1] = np.diff(L)
        if N > 1:
            e[-1] = e[-2]
        dd_ = np.zeros(N)
        dd_[0] = 0.5 * e[0]
        dd_[1:-1] = 0.5 * (e[:-2] + e[1:-1])
        if N > 1:
            dd_[-1] = 0.5 * e[-2]
        primal.append(e.astype(np.float32))
        dual.append(dd_.astype(np.float32))
    return pts, meta, primal, dual


def rad_power(accE, accH, meta):
    """Radiated power through the surface (sim-engine.mjs:474-497)."""
    E = np.asarray(accE, np.float64).reshape(-1, 3, 2)
    H = np.asarray(accH, np.float64).reshape(-1, 3, 2)
    m = np.asarray(meta, np.float64).reshape(-1, 8)
    nd = m[:, 3].astype(int)
    nP, nPP = (nd + 1) % 3, (nd + 2) % 3
    r = np.arange(len(m))
    poy = (E[r, nP, 0] * H[r, nPP, 0] + E[r, nP, 1] * H[r, nPP, 1]) - (E[r, nPP, 0] * H[r, nP, 0] + E[r, nPP, 1] * H[r, nP, 1])
    return float(np.sum(0.5 * m[:, 5] * poy * m[:, 4]))


# ---------------------------------------------------------------------------
# probes (the reference's host-side gather and integral, sim-engine.mjs:188-261)
# ---------------------------------------------------------------------------
def voltage_probe(mesh, start, stop, weight=1.0, interval=1):
    return {"type": 0, "normDir": -1, "weight": weight, "processInterval": interval,
            "start": [int(v) for v in start], "stop": [int(v) for v in stop],
            "startInside": [True] * 3, "stopInside": [True] * 3}


def current_probe(mesh, start, stop, norm_dir, weight=1.0, interval=1):
    return {"type": 1, "normDir": int(norm_dir), "weight": weight, "processInterval": interval,
            "start": [int(v) for v in start], "stop": [int(v) for v in stop],
            "startInside": [True] * 3, "stopInside": [True] * 3}


def build_gather_indices(probes, grid):
    """Restates buildGatherIndices (scripts/lib/sim-engine.mjs:188-242)."""
    Nx, Ny, Nz = grid
    cs = Nx * Ny * Nz
    allidx, slices = [], []
    for p in probes:
        off = len(allidx)
        if p["type"] == 0:
            signs = []
            for n in range(3):
                lo, hi = min(p["start"][n], p["stop"][n]), max(p["start"][n], p["stop"][n])
                if lo == hi:
                    continue
                sign = 1 if p["start"][n] < p["stop"][n] else -1
                for pos in range(lo, hi):
                    xyz = list(p["start"])
                    xyz[n] = pos
                    allidx.append(n * cs + xyz[0] * Ny * Nz + xyz[1] * Nz + xyz[2])
                    signs.append(sign)
            slices.append({"offset": off, "count": len(allidx) - off, "type": "voltage", "signs": signs})
        else:
            s, t, si, so = p["start"], p["stop"], p["startInside"], p["stopInside"]
            edges = []
            add = lambda n, xyz, sg: edges.append((n, list(xyz), sg))
            nd = p["normDir"]
            if nd == 0:
                if so[0] and si[2]:
                    for i in range(s[1] + 1, t[1] + 1): add(1, [t[0], i, s[2]], 1)
                if so[0] and so[1]:
                    for i in range(s[2] + 1, t[2] + 1): add(2, [t[0], t[1], i], 1)
                if si[0] and so[2]:
                    for i in range(s[1] + 1, t[1] + 1): add(1, [s[0], i, t[2]], -1)
                if si[0] and si[1]:
                    for i in range(s[2] + 1, t[2] + 1): add(2, [s[0], s[1], i], -1)
            elif nd == 1:
                if si[0] and si[1]:
                    for i in range(s[2] + 1, t[2] + 1): add(2, [s[0], s[1], i], 1)
                if so[1] and so[2]:
                    for i in range(s[0] + 1, t[0] + 1): add(0, [i, t[1], t[2]], 1)
                if so[0] and so[1]:
                    for i in range(s[2] + 1, t[2] + 1): add(2, [t[0], t[1], i], -1)
                if si[1] and si[2]:
                    for i in range(s[0] + 1, t[0] + 1): add(0, [i, s[1], s[2]], -1)
            else:
                if si[1] and si[2]:
                    for i in range(s[0] + 1, t[0] + 1): add(0, [i, s[1], s[2]], 1)
                if so[0] and si[2]:
                    for i in range(s[1] + 1, t[1] + 1): add(1, [t[0], i, s[2]], 1)
                if so[1] and so[2]:
                    for i in range(s[0] + 1, t[0] + 1): add(0, [i, t[1], t[2]], -1)
                if si[0] and so[2]:
                    for i in range(s[1] + 1, t[1] + 1): add(1, [s[0], i, t[2]], -1)
            for n, xyz, sg in edges:
                allidx.append(n * cs + xyz[0] * Ny * Nz + xyz[1] * Nz + xyz[2])
            slices.append({"offset": off, "count": len(allidx) - off, "type": "current", "signs": [e[2] for e in edges]})
    return np.asarray(allidx, dtype=np.uint32), slices


def probe_integrals(gathered, probes, slices):
    """Restates computeProbeIntegrals (sim-engine.mjs:244-261) for all samples.
    gathered: (num_samples, 2*G) -> (num_samples, num_probes) float64."""
    g = np.asarray(gathered, np.float64).reshape(-1, np.asarray(gathered).shape[-1])
    out = np.zeros((g.shape[0], len(probes)))
    for p, (pr, sl) in enumerate(zip(probes, slices)):
        col = 0 if sl["type"] == "voltage" else 1
        for i in range(sl["count"]):
            out[:, p] += g[:, (sl["offset"] + i) * 2 + col] * sl["signs"][i]
        out[:, p] *= pr["weight"]
    return out
