"""LBM_ARITH_FAST (contracted FMAs, approximate division / sqrt) against
the CPU oracle.  The fast step is not bit-identical to the oracle, and it
does NOT meet the hot path's parity bar (populations 1e-5, Cd/Cl 1e-4
relative): measured on B200, config 1 drifts to ~1e-3 in Cd over 1000
steps and config 2 to ~3e-3 in the populations over 200 steps.  That is
why LBM_ARITH_EXACT is the default.  These tests pin the drift to a
bounded level (the fast mode is still the same scheme) and print it."""
import numpy as np
import pytest

from tests import scenarios as S

pytestmark = pytest.mark.gpu


def _run(oracle, solver, sc, steps, every):
    og = S.make_oracle(oracle, sc)
    gg = S.make_gpu(solver, sc)
    gg.set(arithmetic=1)
    A = og.projected_area(0)
    worst_cd = worst_cl = 0.0
    for _ in range(steps // every):
        og.step(0.05, n=every)
        gg.step(0.05, n=every)
        fo, fg = og.drag_force_decomposed(), gg.drag_force_decomposed()
        q = 0.5 * 0.05 * 0.05 * A
        worst_cd = max(worst_cd, abs(fg[0] - fo[0]) / max(abs(fo[0]), 1e-12))
        worst_cl = max(worst_cl, abs(fg[1] - fo[1]) / q)
    pop = S.rel_err(gg.populations(), og.f)
    return pop, worst_cd, worst_cl


def test_fast_config1_bgk_1000_steps(oracle, solver):
    sc = dict(dims=(128, 64, 64), visc=(0.6 - 0.5) / 3, tau=0.6,
              geometry=[S.sphere_c1(halfway=True)])
    pop, cd, cl = _run(oracle, solver, sc, 1000, 10)
    print(f"fast config1: populations rel {pop:.2e}, Cd rel {cd:.2e}, Cl/Cd-scale {cl:.2e}")
    assert pop <= 1e-3 and cd <= 1e-2 and cl <= 1e-2


def test_fast_config2_mrt_smagorinsky(oracle, solver):
    from lattice_fluid_dynamics_b200 import geometry as G
    tris, bbox = G.ahmed_body()
    sc = dict(dims=(256, 128, 128), visc=1e-4, tau=G.reynolds_tau(0.05, 64.0, 5e4),
              flags=dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1, periodicYZ=1),
              geometry=[("mesh", (tris, bbox))])
    pop, cd, cl = _run(oracle, solver, sc, 200, 20)
    print(f"fast config2 (200 steps): populations rel {pop:.2e}, Cd rel {cd:.2e}, "
          f"Cl/Cd-scale {cl:.2e}")
    assert pop <= 5e-2 and cd <= 1e-2 and cl <= 1e-2
