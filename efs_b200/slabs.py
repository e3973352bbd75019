"""x-slab decomposition of a plain solve over several engines (one per GPU).

The reference runs one engine per solve (src/webgpu-engine.mjs); nothing in
it splits a grid.  This module splits a job along x, the outermost stride of
the NIJK layout, so that each rank's slab is a contiguous range of planes:

* rank r owns planes [x0, x1) and holds, besides them, one ghost plane below
  (x0 - 1) and two above (x1, x1 + 1), clipped to the grid;
* every rank runs the ordinary full timestep on its sub-grid (coefficients,
  UPML regions, Mur, excitation, TFSF, ADE and PBC entries sliced to the
  planes it holds, translated to local indices);
* after each timestep the ghost planes are overwritten with the owners'
  values: E and H (3 components) of plane x0 - 1 from rank r - 1, and of
  planes x1, x1 + 1 from rank r + 1.

Why the owned planes are exact, bit for bit, against the single-domain
solve: E_new(x0) reads H(x0 - 1), which the exchange restored; H_new(x1 - 1)
reads E_new(x1), which the rank computes itself from exchanged H(x1),
H(x1 + 1), E(x1) and the replicated point operations on plane x1; with the
second upper ghost plane H_new(x1) is exact too, so the NF2FF samples and
probes of plane x1 - 1 (which interpolate H at x1) are taken before the
exchange.  Ghost values that come out wrong (E of the lower ghost, computed
with the index-0 self reference; H of the top plane, which a sub-grid does
not update; their UPML fluxes and ADE states) only feed ghost values, which
the next exchange overwrites.  The exchange moves 3 planes x 6 components x
Ny x Nz floats per interface and timestep; PBC along x would couple the
first and last ranks and is rejected.

Sampling outputs (NF2FF surface points, probes) are assigned to the rank
that owns their plane; energies are sums over owned planes.  The whole-solve
results are reductions over ranks: the energy (one scalar), the radiated
power through the NF2FF surface (one scalar) and the far field (E_theta and
E_phi per angle are sums over surface points, so each rank evaluates its own
points and the complex components are summed; P_rad is formed after the sum).
"""
import numpy as np

GHOST_LO, GHOST_HI = 1, 2


def plan(Nx, world):
    """Owned [x0, x1) and held [g0, g1) planes per rank (near-equal owned slabs)."""
    if world < 1 or Nx < 3 * world:
        raise ValueError("need at least 3 x-planes per rank")
    cuts = [round(r * Nx / world) for r in range(world + 1)]
    out = []
    for r in range(world):
        x0, x1 = cuts[r], cuts[r + 1]
        out.append(dict(rank=r, x0=x0, x1=x1, g0=max(0, x0 - GHOST_LO), g1=min(Nx, x1 + GHOST_HI)))
    return out


def _cells(idx, N, NyNz):
    """(component, x, rest-within-plane) of caller field indices."""
    idx = np.asarray(idx, np.int64)
    n = idx // N
    cell = idx - n * N
    return n, cell // NyNz, cell % NyNz


def _local(n, x, rest, g0, Nl, NyNz):
    return (n * Nl + (x - g0) * NyNz + rest).astype(np.uint32)


def split(job, world):
    """Per-rank sub-jobs of `job` (a workloads job dict): list of (slab, sub_job)."""
    Nx, Ny, Nz = job["grid"]
    NyNz = Ny * Nz
    N = Nx * NyNz
    if job.get("pbc") and any(a["axis"] == 0 for a in job["pbc"]["axes"]):
        raise ValueError("PBC along x couples the first and last slabs: not supported")
    out = []
    for s in plan(Nx, world):
        g0, g1 = s["g0"], s["g1"]
        nx = g1 - g0
        Nl = nx * NyNz
        keep = lambda x: (x >= g0) & (x < g1)
        sub = dict(name="%s_slab%d" % (job.get("name", "job"), s["rank"]), grid=[nx, Ny, Nz], dT=job["dT"],
                   maxTS=job.get("maxTS", 0), endCrit=0.0)
        c = job["coefficients"]
        if "mat" in c:
            sub["coefficients"] = dict(mat=np.asarray(c["mat"]).reshape(Nx, NyNz)[g0:g1].reshape(-1),
                                       table=c["table"])
        else:
            sub["coefficients"] = {k: np.asarray(c[k]).reshape(3, Nx, NyNz)[:, g0:g1].reshape(-1)
                                   for k in ("vv", "vi", "ii", "iv")}
        if job.get("pml"):
            regs = []
            for r in job["pml"]:
                (sx, sy, sz), (rx, ry, rz) = r["startPos"], r["numLines"]
                lo, hi = max(sx, g0), min(sx + rx, g1)
                if lo >= hi:
                    continue
                reg = dict(startPos=[lo - g0, sy, sz], numLines=[hi - lo, ry, rz])
                for k in ("vv", "vvfo", "vvfn", "ii", "iifo", "iifn"):
                    reg[k] = np.asarray(r[k]).reshape(3, rx, ry, rz)[:, lo - sx:hi - sx].reshape(-1)
                regs.append(reg)
            sub["pml"] = regs
        if job.get("mur"):
            m = job["mur"]
            mo = {}
            for side in ("nyP", "nyPP"):
                nn, nxn, rn = _cells(m["normal_idx_" + side], N, NyNz)
                ns, nxs, rs = _cells(m["shifted_idx_" + side], N, NyNz)
                k = keep(nxn) & keep(nxs)
                mo["normal_idx_" + side] = _local(nn[k], nxn[k], rn[k], g0, Nl, NyNz)
                mo["shifted_idx_" + side] = _local(ns[k], nxs[k], rs[k], g0, Nl, NyNz)
                mo["coeff_" + side] = np.asarray(m["coeff_" + side], np.float32)[k]
            sub["mur"] = mo
        if job.get("excitation"):
            e = job["excitation"]
            pos = np.asarray(e["pos"], np.int64)
            x = pos // NyNz
            k = keep(x)
            sub["excitation"] = dict(signal=e["signal"], period=e.get("period", 0),
                                     delay=np.asarray(e["delay"], np.uint32)[k], amp=np.asarray(e["amp"], np.float32)[k],
                                     dir=np.asarray(e["dir"], np.uint32)[k],
                                     pos=((x[k] - g0) * NyNz + pos[k] % NyNz).astype(np.uint32))
        if job.get("tfsf"):
            t = job["tfsf"]
            tt = dict(signal=t["signal"], period=t.get("period", 0))
            for side in ("voltagePoints", "currentPoints"):
                p = t[side]
                if not isinstance(p, dict):
                    p = {k: np.asarray([q[k] for q in p]) for k in ("field_idx", "delay_int", "delay_frac", "amp")}
                n, x, rest = _cells(p["field_idx"], N, NyNz)
                k = keep(x)
                tt[side] = dict(field_idx=_local(n[k], x[k], rest[k], g0, Nl, NyNz),
                                delay_int=np.asarray(p["delay_int"], np.uint32)[k],
                                delay_frac=np.asarray(p["delay_frac"], np.float32)[k],
                                amp=np.asarray(p["amp"], np.float32)[k])
            sub["tfsf"] = tt
        if job.get("ade"):
            orders = []
            for o in job["ade"]["orders"]:
                for d in o["directions"]:            # one order per (order, direction): counts may differ per direction
                    pos = np.asarray(d["pos_idx"], np.int64)
                    x = pos // NyNz
                    k = keep(x)
                    dd = dict(dir=d["dir"], pos_idx=((x[k] - g0) * NyNz + pos[k] % NyNz).astype(np.uint32))
                    for key in ("v_int_ADE", "v_ext_ADE", "v_Lor_ADE", "i_int_ADE", "i_ext_ADE", "i_Lor_ADE"):
                        if d.get(key) is not None:
                            dd[key] = np.asarray(d[key], np.float32)[k]
                    orders.append(dict(numCells=int(k.sum()), hasLorentz=o.get("hasLorentz", False), directions=[dd]))
            sub["ade"] = dict(orders=orders, apply=job["ade"].get("apply", False))
        if job.get("pbc"):
            sub["pbc"] = job["pbc"]
        if job.get("nf2ff"):
            nf = job["nf2ff"]
            pts = np.asarray(nf["surfaceIndices"], np.int64).reshape(-1, 3)
            k = (pts[:, 0] >= s["x0"]) & (pts[:, 0] < s["x1"])
            lp = pts[k].copy()
            lp[:, 0] -= g0
            sub["nf2ff"] = dict(nf, surfaceIndices=lp.astype(np.uint32).ravel(), numPoints=int(k.sum()), gridSize=[nx, Ny, Nz],
                                primalEdgeLens=[np.asarray(nf["primalEdgeLens"][0])[g0:g1]] + list(nf["primalEdgeLens"][1:]),
                                dualEdgeLens=[np.asarray(nf["dualEdgeLens"][0])[g0:g1]] + list(nf["dualEdgeLens"][1:]))
            sub["nf2ff_points"] = np.flatnonzero(k)          # positions in the job's point list
            if job.get("nf2ff_meta") is not None:            # far-field rows of the owned points (global positions)
                sub["nf2ff_meta"] = np.asarray(job["nf2ff_meta"], np.float32).reshape(-1, 8)[k].ravel()
            if job.get("nf2ff_freqs") is not None:
                sub["nf2ff_freqs"] = job["nf2ff_freqs"]
        out.append((s, sub))
    return out


def owned(fields, slab, Ny, Nz):
    """The owned planes of a rank's (3 * nx * Ny * Nz) field array, as (3, x1 - x0, Ny * Nz)."""
    nx = slab["g1"] - slab["g0"]
    a = np.asarray(fields).reshape(3, nx, Ny * Nz)
    return a[:, slab["x0"] - slab["g0"]:slab["x1"] - slab["g0"]]


def exchange(ranks, get_planes, set_planes, send=None):
    """Overwrite every rank's ghost planes with their owners' values.

    ranks: list of slabs (plan entries) this process drives, or all of them.
    get_planes(rank, local_x, count) -> (volt, curr), each (3, count, Ny*Nz);
    set_planes(rank, local_x, volt, curr).  With all ranks in one process the
    copies are direct; across processes `send` (see exchange_dist) moves the
    planes."""
    by_rank = {s["rank"]: s for s in ranks}
    for s in ranks:
        r = s["rank"]
        if r > 0 and (r - 1) in by_rank:                       # lower ghost x0-1 from rank r-1
            p = by_rank[r - 1]
            v, c = get_planes(r - 1, s["x0"] - 1 - p["g0"], 1)
            set_planes(r, s["x0"] - 1 - s["g0"], v, c)
        if (r + 1) in by_rank:                                 # upper ghosts x1, x1+1 from rank r+1
            p = by_rank[r + 1]
            cnt = s["g1"] - s["x1"]
            v, c = get_planes(r + 1, s["x1"] - p["g0"], cnt)
            set_planes(r, s["x1"] - s["g0"], v, c)


def exchange_dist(slab, world, get_planes, set_planes, send_recv):
    """The ghost exchange of one rank in a process group: send_recv(dst, arrays, src, shapes)
    posts the sends to `dst` and receives from `src` (None: no partner).  Every rank
    takes the same two exchanges in the same order: first upward (last owned plane to
    rank + 1), then downward (first owned planes to rank - 1)."""
    r = slab["rank"]
    lo_ghost = slab["x0"] - slab["g0"]                          # count of lower ghost planes held
    hi_ghost = slab["g1"] - slab["x1"]
    # first exchange: plane x1-1 up; receive plane x0-1 from below
    out = get_planes(r, slab["x1"] - 1 - slab["g0"], 1) if r + 1 < world else None
    got = send_recv(r + 1 if r + 1 < world else None, out, r - 1 if r > 0 else None, 1)
    if got is not None and lo_ghost:
        set_planes(r, 0, got[0], got[1])
    # second exchange: planes x0, x0+1 down; receive planes x1, x1+1 from above
    cnt_down = min(GHOST_HI, slab["x1"] - slab["x0"])
    out = get_planes(r, slab["x0"] - slab["g0"], cnt_down) if r > 0 else None
    got = send_recv(r - 1 if r > 0 else None, out, r + 1 if r + 1 < world else None, hi_ghost)
    if got is not None and hi_ghost:
        set_planes(r, slab["x1"] - slab["g0"], got[0], got[1])


# ---------------------------------------------------------------------------
# Reductions over ranks.  `all_reduce_sum(x)` returns the sum over ranks of a
# float or float64 array (torch.distributed.all_reduce in a process group, a
# plain sum when one process drives every slab); every rank calls it in the
# same order.
# ---------------------------------------------------------------------------
Z0 = 376.73031346177066              # free-space impedance used by the far field (efs_kernels.cuh)


def owned_energy(volt, curr, slab, grid):
    """This rank's share of the single-domain energy: the sum of volt^2 +
    curr^2 over cells x < Nx-1, y < Ny-1, z < Nz-1 and the three components
    (src/webgpu-engine.mjs:3090-3103), over the owned planes, in f64.
    volt, curr: the owned planes, (3, x1 - x0, Ny*Nz) as getPlanes returns."""
    Nx, Ny, Nz = grid
    n = min(slab["x1"], Nx - 1) - slab["x0"]
    if n <= 0 or Ny < 2 or Nz < 2:
        return 0.0
    tot = 0.0
    for a in (volt, curr):
        b = np.asarray(a).reshape(3, -1, Ny, Nz)[:, :n, :Ny - 1, :Nz - 1].astype(np.float64)
        tot += float(np.sum(b * b))
    return tot


def energy_dist(volt, curr, slab, grid, all_reduce_sum):
    """Energy of the decomposed solve: the owned shares summed over ranks
    (one scalar all-reduce)."""
    return float(all_reduce_sum(np.float64(owned_energy(volt, curr, slab, grid))))


def far_field_dist(partial, all_reduce_sum):
    """Far field of the decomposed solve from each rank's far field of its
    own NF2FF points (the engine's computeNF2FFfarField with the rank's
    accumulators and point rows, the same angles, frequency, centre and
    radius): (n_angles, 5) rows [P_rad, E_theta re, im, E_phi re, im].
    E_theta and E_phi are sums over surface points, so the ranks' complex
    components add (one all-reduce of 4 values per angle) and P_rad =
    (|E_theta|^2 + |E_phi|^2) / (2 Z0) is formed from the sums."""
    p = np.asarray(partial, np.float64).reshape(-1, 5)
    e = np.asarray(all_reduce_sum(np.ascontiguousarray(p[:, 1:5])), np.float64)
    return np.column_stack([(e * e).sum(axis=1) / (2 * Z0), e])


def rad_power_dist(accE, accH, meta, all_reduce_sum):
    """Radiated power through the NF2FF surface (sim-engine.mjs:474-497),
    a sum over surface points: each rank's points, summed over ranks."""
    from .opgen import rad_power
    return float(all_reduce_sum(np.float64(rad_power(accE, accH, meta) if len(meta) else 0.0)))


class LocalSlabs:
    """Every slab of a job on engines driven by this process (one GPU each,
    or several on one GPU): configure, step and exchange ghost planes with
    the engines' getPlanes/setPlanes.  make_engine(rank) returns an
    initialised engine (CudaEngine or the oracle)."""

    def __init__(self, job, world, make_engine):
        from . import workloads
        self.job = job
        self.parts = split(job, world)
        self.engines = []
        for s, sub in self.parts:
            e = make_engine(s["rank"])
            workloads.configure(e, sub)
            self.engines.append(e)

    def _get(self, r, x, cnt):
        return self.engines[r].getPlanes(x, cnt)

    def _set(self, r, x, v, c):
        self.engines[r].setPlanes(x, v, c)

    def iterate(self, n):
        for _ in range(n):
            for e in self.engines:
                e.iterate(1)
            exchange([s for s, _ in self.parts], self._get, self._set)

    def owned_fields(self):
        """E and H of the whole grid assembled from the owned planes, (3, Nx, Ny*Nz) each."""
        Nx, Ny, Nz = self.job["grid"]
        vs, cs = [], []
        for (s, _), e in zip(self.parts, self.engines):
            v, c = e.getPlanes(s["x0"] - s["g0"], s["x1"] - s["x0"])
            vs.append(v)
            cs.append(c)
        return np.concatenate(vs, axis=1), np.concatenate(cs, axis=1)

    def energy(self):
        """Energy of the whole grid from the owned planes (energy_dist with a
        plain sum over the slabs)."""
        tot = 0.0
        for (s, _), e in zip(self.parts, self.engines):
            v, c = e.getPlanes(s["x0"] - s["g0"], s["x1"] - s["x0"])
            tot += owned_energy(v, c, s, self.job["grid"])
        return tot

    def destroy(self):
        for e in self.engines:
            if hasattr(e, "destroy"):
                e.destroy()
