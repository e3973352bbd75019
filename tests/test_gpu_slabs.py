"""x-slab decomposition on the CUDA engine (efs_b200.slabs.LocalSlabs): three
slab engines on one GPU, stepped one timestep at a time with the ghost planes
exchanged through efs_get_planes / efs_set_planes after each, against the
same job on one engine.  The assembled owned planes must equal the single
engine's fields bit for bit (the large plain workload at 40^3 and the
dispersive workload at 36x24x28 with the ADE apply step).  The engines run
one after another on one GPU (nothing waits on another engine); across GPUs
the same exchange moves the planes between devices."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _job(name):
    from efs_b200 import workloads
    if name == "plain":
        return dict(workloads.large_plain(40, tfsf_inset=8, nf2ff_inset=5, steps=200, chunk=8, pml=4), probes=[])
    return workloads.dispersive(grid=(36, 24, 28), pml=3, chunk=6, steps=200, tfsf_inset=6, nf2ff_inset=4, workers=1)


@pytest.mark.parametrize("name", ["plain", "dispersive"])
def test_three_slabs_equal_one_engine(cuda_engine_cls, name):
    from efs_b200 import slabs, workloads

    def make(_rank):
        e = cuda_engine_cls()
        assert e.initGPU()
        return e
    job = _job(name)
    Nx, Ny, Nz = job["grid"]
    run = slabs.LocalSlabs(job, 3, make)
    one = make(0)
    workloads.configure(one, job)
    for n in (1, 12, 17):
        run.iterate(n)
        one.iterate(n)
        v, c = run.owned_fields()
        f = one.getFields()
        assert np.array_equal(v.reshape(-1).view(np.uint32), np.asarray(f["volt"], np.float32).view(np.uint32))
        assert np.array_equal(c.reshape(-1).view(np.uint32), np.asarray(f["curr"], np.float32).view(np.uint32))
    run.destroy()
    one.destroy()


def test_planes_round_trip_device(cuda_engine_cls):
    """efs_get_planes / efs_set_planes into and out of device memory (torch
    CUDA tensors) on a grid with padded rows (Nz = 13)."""
    import torch
    N = (9, 7, 13)
    g = cuda_engine_cls()
    assert g.initGPU()
    t = 3 * N[0] * N[1] * N[2]
    r = np.random.default_rng(3)
    c = dict(vv=np.ones(t, np.float32), vi=np.full(t, 0.2, np.float32), ii=np.ones(t, np.float32),
             iv=np.full(t, 0.2, np.float32))
    g.init(N, c)
    v0, h0 = r.standard_normal(t).astype(np.float32), r.standard_normal(t).astype(np.float32)
    g.uploadFields(v0, h0)
    dv = torch.empty((3, 2, N[1] * N[2]), dtype=torch.float32, device="cuda")
    dc = torch.empty_like(dv)
    g.getPlanes(4, 2, out=(dv, dc))
    ref_v = v0.reshape(3, N[0], -1)[:, 4:6]
    assert np.array_equal(dv.cpu().numpy(), ref_v)
    dv2, dc2 = dv * 2, dc * 2
    torch.cuda.synchronize()                 # torch's stream finished the products before the engine's stream reads them
    g.setPlanes(1, dv2, dc2)
    f = g.getFields()
    got = np.asarray(f["volt"]).reshape(3, N[0], -1)
    assert np.array_equal(got[:, 1:3], 2 * ref_v)
    assert np.array_equal(got[:, 3:], v0.reshape(3, N[0], -1)[:, 3:])
    g.destroy()
