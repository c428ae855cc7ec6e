"""The TMA-staged step kernel (k_step_tma) against the direct kernel.

Both kernels run the same stream + collision code per cell; the staged one
only changes where the pulled populations are read from (shared-memory
boxes filled by bulk tensor copies instead of global loads).  Exact
arithmetic must therefore give byte-identical populations, forces and guard
counts.  The sizes are chosen so that tiles are partial in x, y and z, the
grid edges (wrap / clamp / own-value pulls) cut through staged tiles, and
Bouzidi links and solid cells sit inside staged tiles.  The oracle parity
tests run with staging on (the default), so they cover it against the CPU
oracle as well.
"""
import numpy as np
import pytest

from tests import scenarios as S

pytestmark = pytest.mark.gpu

OPS = {
    "bgk": dict(),
    "reg_smag": dict(useRegularized=1, useSmagorinsky=1, smagorinskyCs=0.17),
    "mrt_smag": dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1),
}


def _pair(solver, sc, storage):
    on = S.make_gpu(solver, sc, storage=storage)
    off = S.make_gpu(solver, sc, storage=storage)
    assert on.set_tma_staging(True), "staging unavailable for an aligned grid"
    assert not off.set_tma_staging(False)
    return on, off


def _assert_same(on, off):
    assert on.post_collision().tobytes() == off.post_collision().tobytes()
    np.testing.assert_array_equal(on.drag_force_decomposed(), off.drag_force_decomposed())
    assert on.guard_resets() == off.guard_resets()


@pytest.mark.parametrize("storage", ["fp32", "fp16", "bf16"])
@pytest.mark.parametrize("periodic", [0, 1])
@pytest.mark.parametrize("op", sorted(OPS))
def test_staged_equals_direct(solver, storage, periodic, op):
    # 72 x 37 x 19: three 32-wide tiles (the last partial), five 8-row tiles
    # (the last partial), three z segments (the last partial)
    sc = dict(dims=(72, 37, 19), visc=0.01, flags=dict(OPS[op], periodicYZ=periodic),
              geometry=[("sphere", (-0.6, 0.15, 0.05, 0.55)), ("ground", (-1.1,))])
    on, off = _pair(solver, sc, storage)
    for _ in range(3):
        on.step(0.06, 0.01, -0.005, n=15)
        off.step(0.06, 0.01, -0.005, n=15)
        _assert_same(on, off)
    on.close()
    off.close()


def test_staged_equals_direct_ahmed_mrt_smagorinsky(solver):
    from lattice_fluid_dynamics_b200 import geometry as G
    tris, bbox = G.ahmed_body()
    sc = dict(dims=(256, 128, 128), visc=1e-4, tau=G.reynolds_tau(0.05, 64.0, 5e4),
              flags=dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1, periodicYZ=1),
              geometry=[("mesh", (tris, bbox))])
    on, off = _pair(solver, sc, "fp32")
    on.step(0.05, n=64)
    off.step(0.05, n=64)
    _assert_same(on, off)


def test_fast_arithmetic_staged_close_to_direct(solver):
    # contracted FMAs may differ between the two kernels: close, not identical
    sc = dict(dims=(96, 48, 40), visc=0.005, flags=dict(useRegularized=1),
              geometry=[("sphere", (-0.5, 0.0, 0.0, 0.6))])
    on, off = _pair(solver, sc, "fp16")
    on.set(arithmetic=1)
    off.set(arithmetic=1)
    on.step(0.05, n=100)
    off.step(0.05, n=100)
    assert S.rel_err(on.post_collision(), off.post_collision(), floor=1e-3) < 1e-2


def test_unaligned_rows_fall_back(solver):
    # 42 FP32 elements per row is not a multiple of 16 bytes: no tensor map
    sc = dict(dims=(42, 16, 12), visc=0.02, geometry=[S.BOX])
    g = S.make_gpu(solver, sc)
    assert not g.set_tma_staging(True)
    g.step(0.05, n=10)
    g.check()
    fp64 = S.make_gpu(solver, dict(dims=(64, 16, 12), visc=0.02), storage="fp64")
    assert not fp64.set_tma_staging(True)


def test_stepn_graph_with_staging(solver):
    sc = dict(dims=(64, 32, 24), visc=0.02, flags=dict(useMRT=1),
              geometry=[("sphere", (-0.5, 0.0, 0.0, 0.5))])
    a, b = _pair(solver, sc, "fp32")
    a.step(0.05, n=70)          # LBM_StepN through captured graph chunks
    b.step_loop(0.05, n=70)     # one LBM_Step call per step
    _assert_same(a, b)
