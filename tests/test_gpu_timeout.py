"""Failure detection on the device path: a bounded device wait that runs out.

Every mbarrier wait of the fused kernel is bounded (about 1 s).  The
diagnostic efs_debug_set_wait lowers that limit to 2 ms and leaves the loads
of one x-plane unissued, so every CTA that streams the plane gives up at it,
drains its other loads in flight (bounded again) and returns; the kernel
records the event in the engine's status word.  The next synchronising call
must return EFS_ERR_TIMEOUT, the CUDA context must stay usable (the same
engine steps again once the knob is reset), and a fresh engine on the same
device must then step bit for bit like the oracle.  Nothing here faults or
hangs a GPU: the waits give up by design.  (The reference only logs a lost
device, src/webgpu-engine.mjs:1129-1131.)
"""
import pytest

from test_gpu_parity import compare_fields, rand_coeffs, seed_fields
from oracle.oracle import OracleEngine

pytestmark = pytest.mark.gpu

EFS_ERR_TIMEOUT = 5


def test_wait_runs_out_and_device_recovers(cuda_engine_cls):
    from efs_b200.engine import EfsError
    N = (20, 18, 24)
    c = rand_coeffs(N, 50)
    g = cuda_engine_cls()
    assert g.initGPU()
    g.init(N, c)
    g.debugSetWait(2_000_000, skip_plane=5)
    g.iterate(1)
    with pytest.raises(EfsError) as err:
        g.sync()
    assert err.value.code == EFS_ERR_TIMEOUT
    g.sync()                                # the status was reported once and cleared
    g.debugSetWait()                        # default limit, every plane issued
    g.iterate(3)
    g.sync()
    assert g.numTS == 4
    g.destroy()

    fresh = cuda_engine_cls()
    assert fresh.initGPU()
    fresh.init(N, c)
    o = OracleEngine(N, c, mode="f32")
    seed_fields(fresh, o, N, 51)
    fresh.iterate(6)
    o.iterate(6)
    compare_fields(fresh, o, "after a timed-out wait on this device")
    fresh.destroy()
