"""LBM_MassMomentumNoAlloc: the allocation-free variant of the FP64
mass/momentum reduction, for callers that cannot call cudaMalloc (real-time
loops that must not stall on an allocation, applications whose device memory
belongs to another allocator).  Its scratch is a fixed __device__ array, so
this test checks, through the C ABI, that it reproduces
LBM_ComputeMassMomentum on two calls in a row (the array keeps the previous
call's contents), including a second, smaller field; that a field of many
65,536-cell chunks sums like NumPy's FP64 sum and that a following field of
fewer chunks reads none of the first field's partials; and that a field
beyond the stated maximum is rejected.  The file sorts last so a run that
stops at the first failure has run every other test already; it also passes
alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tests import scenarios as S

pytestmark = pytest.mark.gpu

RTOL = 1e-12          # FP64 sums of the same values in a different order
MAX_CELLS = 4096 * 65536


def _field(solver, dims, steps):
    sc = dict(dims=dims, visc=0.05, flags=dict(useMRT=1, periodicYZ=1),
              geometry=[("sphere", (-1.2, 0.1, 0.0, 0.5))])
    g = S.make_gpu(solver, sc)
    g.step(0.05, n=steps)
    ref = g.mass_momentum()          # the existing entry point
    soa = np.ascontiguousarray(g.populations().T)   # [19, n] float32
    return g, ref, soa


def _no_alloc(lib, soa, n):
    import torch
    dev = torch.from_numpy(np.ascontiguousarray(soa).reshape(-1)).cuda()
    torch.cuda.synchronize()
    out = np.zeros(4, np.float64)
    rc = lib.LBM_MassMomentumNoAlloc(ctypes.c_void_p(dev.data_ptr()), n,
                                     out.ctypes.data_as(ctypes.c_void_p), None)
    return rc, out


def test_no_alloc_matches_existing_entry_point(solver):
    lib = solver.load()
    g1, ref1, soa1 = _field(solver, (48, 24, 24), 40)
    g2, ref2, soa2 = _field(solver, (24, 16, 12), 7)
    rc, out1 = _no_alloc(lib, soa1, g1.n)
    assert rc == 0
    np.testing.assert_allclose(out1, ref1, rtol=RTOL, atol=1e-12)
    # second call, smaller field: stale partials of the first call must not leak
    rc, out2 = _no_alloc(lib, soa2, g2.n)
    assert rc == 0
    np.testing.assert_allclose(out2, ref2, rtol=RTOL, atol=1e-12)
    # and the first field again
    rc, out3 = _no_alloc(lib, soa1, g1.n)
    assert rc == 0
    np.testing.assert_array_equal(out3, out1)


def _numpy_sums(soa):
    """FP64 mass and momentum of an SoA field [19, n] (D3Q19 velocity set of
    simulation/shaders/lbm_collide.comp:33-52)."""
    ex = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], np.float64)
    ey = np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1], np.float64)
    ez = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1], np.float64)
    per_dir = soa.astype(np.float64).sum(axis=1)
    return np.array([per_dir.sum(), ex @ per_dir, ey @ per_dir, ez @ per_dir])


def test_no_alloc_many_chunks_then_fewer(solver):
    lib = solver.load()
    rng = np.random.default_rng(7)
    n_big = 3 * 65536 + 12345            # four chunks, the last one partial
    big = rng.uniform(0.0, 0.1, size=(19, n_big)).astype(np.float32)
    rc, out = _no_alloc(lib, big, n_big)
    assert rc == 0
    np.testing.assert_allclose(out, _numpy_sums(big), rtol=1e-12, atol=1e-9)
    # a field of fewer chunks right after: the totals must not include the
    # partials the previous call left in chunks 1..3
    n_small = 65536 + 999                 # two chunks
    small = rng.uniform(0.0, 0.1, size=(19, n_small)).astype(np.float32)
    rc, out2 = _no_alloc(lib, small, n_small)
    assert rc == 0
    np.testing.assert_allclose(out2, _numpy_sums(small), rtol=1e-12, atol=1e-9)
    # and one chunk
    n_one = 4099
    one = rng.uniform(0.0, 0.1, size=(19, n_one)).astype(np.float32)
    rc, out3 = _no_alloc(lib, one, n_one)
    assert rc == 0
    np.testing.assert_allclose(out3, _numpy_sums(one), rtol=1e-12, atol=1e-9)


def test_no_alloc_rejects_oversized_field(solver):
    import torch
    lib = solver.load()
    buf = torch.zeros(19 * 64, dtype=torch.float32, device="cuda")
    out = np.zeros(4, np.float64)
    rc = lib.LBM_MassMomentumNoAlloc(ctypes.c_void_p(buf.data_ptr()), MAX_CELLS + 1,
                                     out.ctypes.data_as(ctypes.c_void_p), None)
    assert rc == 1                   # LBM_ERR_INVALID_ARGUMENT, nothing launched
    assert np.all(out == 0)
