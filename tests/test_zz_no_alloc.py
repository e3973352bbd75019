"""efs_energy_noalloc, the allocation-free energy entry point, against efs_energy.

Some callers cannot let the library allocate device memory once they are
running (a server that reserved its HBM budget up front, a host runtime that
owns every device allocation).  efs_energy_noalloc serves them with scratch
in a fixed array inside libefs.so.  These tests call it through the C ABI:
first on a fresh engine, before anything else could have allocated scratch
for it, checking that neither the engine's device bytes nor the device's free
memory change across the call; then against efs_energy (lagged == 0) to
1e-10 relative (both sum the same f32 per-cell terms in f64, in different
orders), twice in a row and again after the fields change, since every call
shares the same scratch array.  The file runs last so that a failure here
leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10


def energy_ref(g):
    v = C.c_double()
    assert g._lib.efs_energy(g.handle, 0, C.byref(v)) == 0, g._lib.efs_last_error(g.handle)
    return v.value


def energy_noalloc(g):
    v = C.c_double()
    rc = g._lib.efs_energy_noalloc(g.handle, C.byref(v))
    assert rc == 0, g._lib.efs_last_error(g.handle)
    return v.value


def make_engine(cls, N, seed):
    r = np.random.default_rng(seed)
    t = 3 * N[0] * N[1] * N[2]
    coeffs = dict(vv=(0.95 + 0.05 * r.random(t)).astype(np.float32), vi=(0.1 + 0.2 * r.random(t)).astype(np.float32),
                  ii=(0.97 + 0.03 * r.random(t)).astype(np.float32), iv=(0.1 + 0.2 * r.random(t)).astype(np.float32))
    g = cls()
    assert g.initGPU()
    g.init(N, coeffs)
    g.uploadFields(r.standard_normal(t).astype(np.float32), r.standard_normal(t).astype(np.float32))
    return g


def test_energy_noalloc_allocates_nothing(cuda_engine_cls):
    import torch
    warm = make_engine(cuda_engine_cls, (6, 6, 6), 3)
    try:
        energy_noalloc(warm)      # library code and the scratch address resident on this device
    finally:
        warm.destroy()
    g = make_engine(cuda_engine_cls, (40, 36, 44), 5)
    try:
        torch.cuda.synchronize()
        held, free = g.deviceBytes(), torch.cuda.mem_get_info()[0]
        got = energy_noalloc(g)   # first energy call of this engine: no efs_energy before it
        torch.cuda.synchronize()
        assert g.deviceBytes() == held
        assert torch.cuda.mem_get_info()[0] == free
        ref = energy_ref(g)
        assert abs(got - ref) <= TOL * abs(ref), (got, ref)
    finally:
        g.destroy()


# (3,3,3): one partial sum; (48,50,64): 145,089 interior cells, three partial
# sums, the last one partly filled; (4,2,43692): 131,073 = 2*65536+1 interior
# cells, the last partial sum a single cell; (8,1,1): no interior cells
@pytest.mark.parametrize("N", [(3, 3, 3), (48, 50, 64), (4, 2, 43692), (8, 1, 1)])
def test_energy_noalloc_matches_energy(cuda_engine_cls, N):
    g = make_engine(cuda_engine_cls, N, 7)
    try:
        for _ in range(2):                        # two states of the fields
            first, second = energy_noalloc(g), energy_noalloc(g)   # two calls in a row, before efs_energy
            ref = energy_ref(g)
            for got in (first, second):
                assert abs(got - ref) <= TOL * abs(ref), (N, got, ref)
            if ref == 0.0:
                assert first == second == 0.0
            g.iterate(5)                          # new fields; the shared scratch keeps the old sums
    finally:
        g.destroy()


def test_energy_noalloc_after_other_engines(cuda_engine_cls):
    """A second engine on the same device reuses the looked-up scratch address."""
    a = make_engine(cuda_engine_cls, (20, 22, 24), 11)
    b = make_engine(cuda_engine_cls, (30, 18, 26), 12)
    try:
        for g in (a, b, a):
            ref = energy_ref(g)
            assert abs(energy_noalloc(g) - ref) <= TOL * abs(ref)
    finally:
        a.destroy()
        b.destroy()
