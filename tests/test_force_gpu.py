"""The drag readback (LBM_ComputeDragForceDecomposed / LBM_ComputeDragForceF64)
against the oracle across the cases its kernel handles specially: a grid
without boundary links, repeated readbacks without a step in between (the
block partials and the ticket that the last block resets), a link list that
grows (more blocks, a larger partials buffer), readbacks after explicit,
fused and graph-replayed steps, and FP16 storage.  The integer sums are
bit-identical to the oracle's; the FP64 sums are added in a fixed order and
so repeat exactly."""
import numpy as np
import pytest

from tests import scenarios as S

pytestmark = pytest.mark.gpu


def _same_force(og, gg):
    np.testing.assert_array_equal(gg.drag_force_decomposed(), og.drag_force_decomposed())
    assert og.force_raw == list(gg.drag_force_f64()[1])


def test_no_links_reads_zero(oracle, solver):
    sc = dict(dims=(64, 32, 32), visc=0.02)
    og, gg = S.make_oracle(oracle, sc), S.make_gpu(solver, sc)
    og.step(0.05, n=5)
    gg.step(0.05, n=5)
    assert not gg.drag_force_decomposed().any()
    f64, raw = gg.drag_force_f64()
    assert not f64.any() and not raw.any()
    _same_force(og, gg)


def test_repeated_readbacks_and_growing_link_list(oracle, solver):
    sc = dict(dims=(96, 48, 48), visc=0.01, flags=dict(useRegularized=1, periodicYZ=1),
              geometry=[("sphere", (-1.2, 0.0, 0.0, 0.35))])
    og, gg = S.make_oracle(oracle, sc), S.make_gpu(solver, sc)
    og.step(0.05, 0.0, 0.0, n=1)      # explicit-f step
    gg.step(0.05, 0.0, 0.0, n=1)
    _same_force(og, gg)
    og.step(0.05, n=13)               # fused steps, odd count
    gg.step_loop(0.05, n=13)
    first = gg.drag_force_f64()
    for _ in range(4):                # no step in between: identical, FP64 included
        again = gg.drag_force_f64()
        assert again[0].tobytes() == first[0].tobytes()
        assert again[1].tolist() == first[1].tolist()
    _same_force(og, gg)
    nl0 = len(gg.links()[0])
    # a second, larger body: more boundary cells, more force blocks
    for t in (og, gg):
        t.set_solid_sphere(0.6, 0.2, -0.1, 0.8)
    assert len(gg.links()[0]) > nl0
    og.step(0.05, n=64)               # graph-replayed chunks on the GPU side
    gg.step(0.05, n=64)
    _same_force(og, gg)


def test_fp16_readback_repeats_and_tracks_fp32(oracle, solver):
    sc = dict(dims=(64, 32, 32), visc=0.02, geometry=[S.BOX])
    g16 = S.make_gpu(solver, sc, storage="fp16")
    g32 = S.make_gpu(solver, sc)
    g16.step(0.05, n=200)
    g32.step(0.05, n=200)
    a, b = g16.drag_force_f64(), g16.drag_force_f64()
    assert a[0].tobytes() == b[0].tobytes() and a[1].tolist() == b[1].tolist()
    f16, f32 = g16.drag_force_decomposed(), g32.drag_force_decomposed()
    assert abs(f16[0] - f32[0]) <= 2e-2 * abs(f32[0])
