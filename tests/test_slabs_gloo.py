"""x-slab decomposition of a plain solve (efs_b200.slabs) on the CPU: each
rank steps its slab (owned planes plus ghost planes) on the f32 oracle and the
ghost planes are exchanged after every timestep; the owned planes and the
NF2FF accumulators of the owned surface points must equal the single-domain
solve bit for bit (without the exchange they do not).  Two jobs: the large plain workload at 40^3
(boxes, Mur on +-x/+-y, UPML on +-z, TFSF, NF2FF with 3 frequencies) and the
dispersive workload at 36x24x28 (UPML on all faces, so the x slabs cut UPML
regions; Drude/Lorentz spheres with the ADE apply step; TFSF at 30 degrees).
World size 2 over gloo (send/recv between processes) and world size 3 in one
process (the middle rank has both neighbours).  The whole-solve results are
reductions over the ranks (efs_b200.slabs: energy, radiated power and far
field, summed by all-reduce over gloo or by a plain sum in one process) and
must equal the single-domain values up to f64 summation order."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

STEPS = 25


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _job(name):
    from efs_b200 import workloads
    if name == "plain":
        return dict(workloads.large_plain(40, tfsf_inset=8, nf2ff_inset=5, steps=200, chunk=8, pml=4), probes=[])
    return workloads.dispersive(grid=(36, 24, 28), pml=3, chunk=6, steps=200, tfsf_inset=6, nf2ff_inset=4, workers=1)


def _single(job):
    from efs_b200 import workloads
    from oracle.oracle import OracleEngine
    o = OracleEngine(mode="f32")
    workloads.configure(o, job)
    o.iterate(STEPS)
    return o


def _planes_io(engines, Ny, Nz):
    def get(r, x, cnt):
        f = engines[r].getFields()
        nx = len(f["volt"]) // (3 * Ny * Nz)
        v = np.asarray(f["volt"], np.float32).reshape(3, nx, Ny * Nz)[:, x:x + cnt].copy()
        c = np.asarray(f["curr"], np.float32).reshape(3, nx, Ny * Nz)[:, x:x + cnt].copy()
        return v, c

    def put(r, x, v, c):
        f = engines[r].getFields()
        nx = len(f["volt"]) // (3 * Ny * Nz)
        vv = np.asarray(f["volt"], np.float32).reshape(3, nx, Ny * Nz).copy()
        cc = np.asarray(f["curr"], np.float32).reshape(3, nx, Ny * Nz).copy()
        vv[:, x:x + v.shape[1]] = v
        cc[:, x:x + c.shape[1]] = c
        engines[r].uploadFields(vv.reshape(-1), cc.reshape(-1))
    return get, put


def _check(job, slabs, results):
    """results[r] = (owned volt, owned curr, nf2ff E, nf2ff H, ade volt state)."""
    o = _single(job)
    Nx, Ny, Nz = job["grid"]
    vol = np.concatenate([results[s["rank"]][0] for s in slabs], axis=1)
    cur = np.concatenate([results[s["rank"]][1] for s in slabs], axis=1)
    assert np.array_equal(vol.view(np.uint32), np.asarray(o.volt, np.float32).reshape(3, Nx, Ny * Nz).view(np.uint32))
    assert np.array_equal(cur.view(np.uint32), np.asarray(o.curr, np.float32).reshape(3, Nx, Ny * Nz).view(np.uint32))
    if job.get("nf2ff"):
        acc = o.readNF2FFAccumulation(True)
        nfreq = len(job["nf2ff"]["omegas"])
        npts = job["nf2ff"]["numPoints"]
        E = np.asarray(acc["accumE"], np.float32).reshape(nfreq, npts, 6)
        H = np.asarray(acc["accumH"], np.float32).reshape(nfreq, npts, 6)
        seen = 0
        for s in slabs:
            idx, e, h = results[s["rank"]][2:5]
            assert np.array_equal(e.reshape(nfreq, -1, 6).view(np.uint32), E[:, idx].view(np.uint32))
            assert np.array_equal(h.reshape(nfreq, -1, 6).view(np.uint32), H[:, idx].view(np.uint32))
            seen += len(idx)
        assert seen == npts


ANGLES = (np.deg2rad(np.arange(0.0, 181.0, 30.0)).astype(np.float32),
          np.deg2rad(np.arange(0.0, 360.0, 45.0)).astype(np.float32))


def _partials(o, s, sub, get):
    """This rank's owned planes, far field of its own NF2FF points at
    frequency 0 and its NF2FF accumulators/rows (for the radiated power)."""
    from oracle.oracle import far_field
    v, c = get(s["rank"], s["x0"] - s["g0"], s["x1"] - s["x0"])
    A = ANGLES[0].size * ANGLES[1].size
    if sub.get("nf2ff") and sub["nf2ff"]["numPoints"]:
        acc = o.readNF2FFAccumulation(True)
        aE, aH = np.asarray(acc["accumE"])[0], np.asarray(acc["accumH"])[0]
        ff = far_field(aE, aH, sub["nf2ff_meta"], *ANGLES, sub["nf2ff_freqs"][0])
        meta = np.asarray(sub["nf2ff_meta"], np.float32)
    else:
        aE = aH = meta = np.zeros(0, np.float32)
        ff = np.zeros((A, 5))
    return v, c, ff, aE, aH, meta


def _check_reductions(job, reduced):
    """reduced = (energy, far field (A, 5), radiated power) of the slabs
    against the single-domain oracle: f64 sums in another order."""
    from efs_b200 import opgen
    from oracle.oracle import far_field
    o = _single(job)
    energy, ff, prad = reduced
    assert abs(energy - o.energy()) <= 1e-12 * abs(o.energy()), (energy, o.energy())
    acc = o.readNF2FFAccumulation(True)
    aE, aH = np.asarray(acc["accumE"])[0], np.asarray(acc["accumH"])[0]
    ref = far_field(aE, aH, job["nf2ff_meta"], *ANGLES, job["nf2ff_freqs"][0])
    scale = np.abs(ref[:, 1:]).max()
    assert np.abs(ff[:, 1:] - ref[:, 1:]).max() <= 1e-9 * scale
    assert np.abs(ff[:, 0] - ref[:, 0]).max() <= 1e-9 * ref[:, 0].max()
    p_ref = opgen.rad_power(aE, aH, job["nf2ff_meta"])
    assert abs(prad - p_ref) <= 1e-9 * abs(p_ref), (prad, p_ref)


def _rank_results(o, s, sub, Ny, Nz):
    from efs_b200 import slabs
    f = o.getFields()
    out = [slabs.owned(np.asarray(f["volt"], np.float32), s, Ny, Nz).copy(),
           slabs.owned(np.asarray(f["curr"], np.float32), s, Ny, Nz).copy()]
    if sub.get("nf2ff") and sub["nf2ff"]["numPoints"]:
        acc = o.readNF2FFAccumulation(True)
        out += [sub["nf2ff_points"], np.asarray(acc["accumE"], np.float32), np.asarray(acc["accumH"], np.float32)]
    else:
        out += [np.zeros(0, np.int64), np.zeros(0, np.float32), np.zeros(0, np.float32)]
    return out


@pytest.mark.parametrize("name", ["plain", "dispersive"])
def test_three_slabs_in_process(name):
    from efs_b200 import slabs, workloads
    from oracle.oracle import OracleEngine
    job = _job(name)
    Nx, Ny, Nz = job["grid"]
    parts = slabs.split(job, 3)
    engines = []
    for s, sub in parts:
        o = OracleEngine(mode="f32")
        workloads.configure(o, sub)
        engines.append(o)
    get, put = _planes_io(engines, Ny, Nz)
    for _ in range(STEPS):
        for o in engines:
            o.iterate(1)
        slabs.exchange([s for s, _ in parts], get, put)
    results = {s["rank"]: _rank_results(engines[s["rank"]], s, sub, Ny, Nz) for s, sub in parts}
    _check(job, [s for s, _ in parts], results)
    # whole-solve results as reductions over the slabs (a plain sum in one process)
    parts_r = [_partials(engines[s["rank"]], s, sub, get) for s, sub in parts]
    energy = sum(slabs.owned_energy(v, c, s, job["grid"]) for (s, _), (v, c, *_r) in zip(parts, parts_r))
    ff = slabs.far_field_dist(parts_r[0][2], lambda x: sum(np.asarray(p[2])[:, 1:5] for p in parts_r))
    prad = sum(slabs.rad_power_dist(p[3], p[4], p[5], lambda x: x) for p in parts_r)
    _check_reductions(job, (energy, ff, prad))


def _slab_rank(rank, world, port, outdir, name):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch
    from efs_b200 import replicas, slabs, workloads
    from oracle.oracle import OracleEngine
    dist = replicas.init_group("gloo", timeout_s=60)
    job = _job(name)
    Nx, Ny, Nz = job["grid"]
    s, sub = slabs.split(job, world)[rank]
    o = OracleEngine(mode="f32")
    workloads.configure(o, sub)
    get, put = _planes_io({rank: o}, Ny, Nz)

    def send_recv(dst, arrays, src, count):
        reqs = []
        if dst is not None:
            for a in arrays:
                reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(a)), dst))
        got = None
        if src is not None:
            bufs = [torch.zeros((3, count, Ny * Nz), dtype=torch.float32) for _ in range(2)]
            for b in bufs:
                dist.recv(b, src)
            got = [b.numpy() for b in bufs]
        for q in reqs:
            q.wait()
        return got

    for _ in range(STEPS):
        o.iterate(1)
        slabs.exchange_dist(s, world, get, put, send_recv)
    res = _rank_results(o, s, sub, Ny, Nz)
    np.savez(os.path.join(outdir, "rank%d.npz" % rank), *res)

    def all_reduce_sum(x):
        t = torch.from_numpy(np.array(x, np.float64).reshape(-1))
        dist.all_reduce(t)
        return t.numpy().reshape(np.shape(x))
    v, c, ff, aE, aH, meta = _partials(o, s, sub, get)
    energy = slabs.energy_dist(v, c, s, job["grid"], all_reduce_sum)
    ff = slabs.far_field_dist(ff, all_reduce_sum)
    prad = slabs.rad_power_dist(aE, aH, meta, all_reduce_sum)
    np.savez(os.path.join(outdir, "reduced%d.npz" % rank), energy=energy, ff=ff, prad=prad)
    dist.destroy_process_group()


@pytest.mark.parametrize("name", ["plain", "dispersive"])
def test_two_slabs_over_gloo(name):
    from efs_b200 import slabs
    out = tempfile.mkdtemp()
    mp.start_processes(_slab_rank, args=(2, _free_port(), out, name), nprocs=2, start_method="spawn", join=True)
    job = _job(name)
    parts = slabs.split(job, 2)
    results = {}
    for s, _ in parts:
        z = np.load(os.path.join(out, "rank%d.npz" % s["rank"]))
        results[s["rank"]] = [z["arr_%d" % i] for i in range(5)]
    _check(job, [s for s, _ in parts], results)
    red = [np.load(os.path.join(out, "reduced%d.npz" % s["rank"])) for s, _ in parts]
    for z in red[1:]:                      # every rank holds the same reduced results
        assert float(z["energy"]) == float(red[0]["energy"]) and np.array_equal(z["ff"], red[0]["ff"])
    _check_reductions(job, (float(red[0]["energy"]), red[0]["ff"], float(red[0]["prad"])))


def test_local_slabs_driver():
    """slabs.LocalSlabs (the in-process driver the GPU runs use) on the
    oracle: owned fields bit-exact against one domain, energy() equal up to
    f64 summation order."""
    from efs_b200 import slabs
    from oracle.oracle import OracleEngine
    job = _job("plain")
    Nx, Ny, Nz = job["grid"]
    ls = slabs.LocalSlabs(job, 3, lambda r: OracleEngine(mode="f32"))
    ls.iterate(STEPS)
    v, c = ls.owned_fields()
    o = _single(job)
    assert np.array_equal(v.view(np.uint32), np.asarray(o.volt, np.float32).reshape(3, Nx, Ny * Nz).view(np.uint32))
    assert np.array_equal(c.view(np.uint32), np.asarray(o.curr, np.float32).reshape(3, Nx, Ny * Nz).view(np.uint32))
    assert abs(ls.energy() - o.energy()) <= 1e-12 * o.energy()
    ls.destroy()
