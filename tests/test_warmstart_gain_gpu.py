"""What the trained warm-start network gains over the plain method.

The network is trained, by this library's own forward and backward kernels,
on snapshots that the plain solver produces for 64 random shapes (seed 2) at
64x32x32 (300 epochs); then, on 8 held-out shapes at 128x64x64, the number of steps until
the trailing-mean drag coefficient enters and stays within 0.5 % of its
converged value (the mean of a long cold run) is compared for (a) the plain
method, uniform flow at start, and (b) the same solver initialised from the
trained network's prediction (LBM_InitializeFromWarmNet, flux-corrected),
with the same FP32 storage, so the difference is the network's alone.  An
untrained network of the same architecture is evaluated beside it as a
control.  The test requires the trained warm start to need fewer steps than
the plain start in total and on the median shape, and prints every number.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FULL = (128, 64, 64)
HALF = tuple(v // 2 for v in FULL)
NET = tuple(v // 4 for v in FULL)


def _evaluate(net, shapes):
    from lattice_fluid_dynamics_b200 import warmstart as W
    return W.evaluate(net, shapes, FULL, sample=50, cold_steps=16000, avg_steps=1000,
                      ref_steps=3000, hold_steps=2000, variants=("warmc_fp32",))


def test_trained_warm_start_reaches_the_cd_band_sooner(solver):
    from lattice_fluid_dynamics_b200 import capi
    from lattice_fluid_dynamics_b200 import warmstart as W
    net = capi.WarmNet(*NET, max_batch=8, seed=2)
    info = {}
    # 56 training samples, batch 8: 7 Adam steps per epoch; 300 epochs get
    # past the 200-step learning-rate warm-up into the cosine decay
    hist = W.train_from_snapshots(net, count=64, val=8, seed=2, snapshot_dims=HALF,
                                  snapshot_steps=4000, epochs=300, batch=8, lr=1e-3, res=info)
    assert hist[-1]["train_loss"] < 0.5 * hist[0]["train_loss"], hist
    shapes = [W.random_union(2, 100000 + i) for i in range(8)]
    rows = _evaluate(net, shapes)
    untrained = capi.WarmNet(*NET, max_batch=8, seed=3)
    untrained.set_output_scaling(np.asarray(info["output_scaling"]["scale"], np.float32),
                                 np.asarray(info["output_scaling"]["shift"], np.float32))
    rows_u = _evaluate(untrained, shapes)
    cold, warm, ctrl = [], [], []
    for r, ru in zip(rows, rows_u):
        c, w, u = r["cold_fp32"]["steps"], r["warmc_fp32"]["steps"], ru["warmc_fp32"]["steps"]
        print(f"shape {r['index']}: Re {r['Re']:.0f}, Cd {r['cd_ref']:.4f}: steps to the 0.5 % "
              f"band cold {c}, trained warm {w} (fallback {r['warmc_fp32']['fallback']}), "
              f"untrained warm {u}")
        if c is not None and w is not None:
            cold.append(c)
            warm.append(w)
            ctrl.append(u if u is not None else 16000)
    print(f"trained on {info['trained_on']} snapshots (dropped {info['dataset_unstable']}), "
          f"final loss {hist[-1]['train_loss']:.4f}; shapes where both enter the band: "
          f"{len(cold)} of {len(rows)}")
    print(f"steps, total: cold {sum(cold)}, trained warm {sum(warm)}, untrained warm "
          f"{sum(ctrl)}; median: cold {np.median(cold)}, trained warm {np.median(warm)}, "
          f"untrained warm {np.median(ctrl)}")
    assert len(cold) >= 6
    assert sum(warm) < sum(cold)
    assert np.median(warm) < np.median(cold)
