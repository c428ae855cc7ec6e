"""Batched stepping (LBM_Batch*): every grid of a batch must end bit-identical
to the same grid stepped alone, whatever the mix of sizes, operators,
periodic flags, tile shapes and run lengths."""
from __future__ import annotations

import numpy as np
import pytest

from lattice_fluid_dynamics_b200 import capi, geometry
from tests import scenarios as S

MIX = [
    dict(dims=(40, 24, 16), visc=0.02, flags=dict(periodicYZ=1),
         geometry=[("sphere", (-2.0, 0.0, 0.0, 0.5))], U=0.05),
    dict(dims=(72, 20, 28), visc=0.01, flags=dict(useRegularized=1, periodicYZ=0),
         geometry=[S.BOX], U=0.04),
    dict(dims=(33, 17, 9), visc=0.05, flags=dict(useMRT=1, periodicYZ=1),
         geometry=[("sphere_halfway", (-1.0, 0.1, 0.0, 0.6)), ("ground", (-1.5,))], U=0.06),
    dict(dims=(64, 32, 32), visc=0.005, flags=dict(useMRT=1, useSmagorinsky=1,
                                                    smagorinskyCs=0.12, periodicYZ=1),
         geometry=[("mesh", geometry.uv_sphere(0.7, (-1.5, 0.0, 0.0), 12, 12))], U=0.05),
    dict(dims=(300, 8, 8), visc=0.1, flags=dict(periodicYZ=0), geometry=[], U=0.03),
]


# every NX even: the batch runs the paired (two cells per thread) kernels
MIX_EVEN = [dict(m, dims=(34, 18, 9)) if m["dims"] == (33, 17, 9) else m for m in MIX]
MIXES = {"odd": MIX, "even": MIX_EVEN}


def _make(solver, sc):
    g = S.make_gpu(solver, dict(sc, init=(sc["U"], 0.0, 0.0)))
    return g


def _inlets(mix):
    return np.array([[m["U"], 0.0, 0.0] for m in mix], np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("mix", sorted(MIXES))
@pytest.mark.parametrize("schedule", ["fused", "graph"])
@pytest.mark.parametrize("runs", [[70], [1, 1, 33], [3, 64, 5]])
def test_batch_matches_solo(solver, runs, schedule, mix):
    MIX = MIXES[mix]
    bg = [_make(solver, m) for m in MIX]
    sg = [_make(solver, m) for m in MIX]
    b = capi.Batch(bg)
    b.set_schedule(schedule)
    for n in runs:
        b.run(n, _inlets(MIX))
        for g, m in zip(sg, MIX):
            g.step(m["U"], n=n)
    for k, (g1, g2) in enumerate(zip(bg, sg)):
        assert np.array_equal(g1.populations(), g2.populations()), k
        assert np.array_equal(g1.velocity(), g2.velocity()), k
        assert np.array_equal(g1.drag_force_decomposed(), g2.drag_force_decomposed()), k
        assert g1.guard_resets() == g2.guard_resets()
    b.close()


@pytest.mark.gpu
def test_batch_matches_oracle(solver, oracle):
    sc = MIX[3]
    g = _make(solver, sc)
    o = S.make_oracle(oracle, dict(sc, init=(sc["U"], 0.0, 0.0)))
    b = capi.Batch([g])
    b.run(40, _inlets([sc]))
    o.step(sc["U"], n=40)
    assert np.array_equal(g.populations(), o.f)
    assert np.array_equal(g.drag_force_decomposed(), o.drag_force_decomposed())


@pytest.mark.gpu
@pytest.mark.parametrize("mix", sorted(MIXES))
@pytest.mark.parametrize("schedule", ["fused", "graph"])
@pytest.mark.parametrize("tile", [32, 64, 128, 256])
def test_tiles_do_not_change_results(solver, tile, schedule, mix):
    if mix == "even" and tile == 32:
        pytest.skip("the paired kernels' tiles are 64, 128 or 256 cells wide")
    MIX = MIXES[mix]
    bg = [_make(solver, m) for m in MIX]
    sg = [_make(solver, m) for m in MIX]
    b = capi.Batch(bg)
    b.set_schedule(schedule)
    for i in range(len(bg)):
        b.set_tile(i, tile)
        assert b.tile(i) == (tile, 256 // tile)
    b.run(37, _inlets(MIX))
    for g, m in zip(sg, MIX):
        g.step(m["U"], n=37)
    for g1, g2 in zip(bg, sg):
        assert np.array_equal(g1.populations(), g2.populations())


@pytest.mark.gpu
@pytest.mark.parametrize("mix", sorted(MIXES))
def test_autotune_leaves_state_and_interleaves_with_solo_calls(solver, mix):
    MIX = MIXES[mix]
    bg = [_make(solver, m) for m in MIX]
    sg = [_make(solver, m) for m in MIX]
    b = capi.Batch(bg)
    b.run(5, _inlets(MIX))
    before = [g.populations() for g in bg]
    b.autotune(3)
    assert b.schedule in ("fused", "graph")
    for g, f in zip(bg, before):
        assert np.array_equal(g.populations(), f)
    assert all(b.tile(i)[0] in (32, 64, 128, 256) for i in range(len(bg)))
    # a solo step on one member and a periodic-flag change between runs
    bg[0].step(MIX[0]["U"], n=3)
    bg[1].set(periodicYZ=1)
    b.run(40, _inlets(MIX))
    for g, m in zip(sg, MIX):
        g.step(m["U"], n=5)
    sg[0].step(MIX[0]["U"], n=3)
    sg[1].set(periodicYZ=1)
    for g, m in zip(sg, MIX):
        g.step(m["U"], n=40)
    for g1, g2 in zip(bg, sg):
        assert np.array_equal(g1.populations(), g2.populations())


@pytest.mark.gpu
def test_batch_rejects_bad_groups(solver):
    a = _make(solver, MIX[0])
    f16 = capi.Grid(16, 8, 8, 0.1, storage="fp16")
    f16.initialize_flow(0.05)
    with pytest.raises(RuntimeError):
        capi.Batch([a, f16])
    with pytest.raises(RuntimeError):
        capi.Batch([a, a])
    fresh = capi.Grid(16, 8, 8, 0.1)
    with pytest.raises(RuntimeError):
        capi.Batch([fresh])
    fast = _make(solver, MIX[1])
    fast.set(arithmetic=capi.LBM_ARITH_FAST)
    with pytest.raises(RuntimeError):
        capi.Batch([fast])


@pytest.mark.gpu
def test_sweep_small_is_identical_to_solo(solver):
    from lattice_fluid_dynamics_b200 import sweep
    res = sweep.run_sweep(count=6, steps=80, seed=1, autotune=True, solo=True)
    assert res["cd_identical"] == 6
    assert res["mlups"] > 0
    assert all(np.isfinite(p["cd"]) and p["cd"] > 0 for p in res["per_instance"])
