"""The warm-start network on the GPU (tensor-core convolutions + element-wise
kernels + Adam) against the CPU oracle of the same network: forward
prediction, loss and the gradient of every layer's parameters, with the
oracle rounding to bfloat16 where the GPU stores bfloat16.  Tolerances:
prediction 2e-2 of its scale, loss 1e-2 relative, each layer's gradient
cosine similarity > 0.99 and norm within 5 %."""
from __future__ import annotations

import numpy as np
import pytest

from lattice_fluid_dynamics_b200 import capi
from oracle import nnoracle as no

DIMS = (1, 8, 8, 16)  # batch, nz, ny, nx


def _inputs(seed, dims=DIMS):
    rng = np.random.default_rng(seed)
    nb, nz, ny, nx = dims
    m = nb * nz * ny * nx
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    mask = (((x - nx / 3) ** 2 / 9 + (y - ny / 2) ** 2 / 4 + (z - nz / 2) ** 2 / 4) < 1.5)
    feats = np.zeros((nb, nz * ny * nx, 3), np.float32)
    feats[..., 0] = mask.reshape(-1).astype(np.float32)
    feats[..., 1] = rng.uniform(0.03, 0.08, (nb, 1))
    feats[..., 2] = rng.uniform(100, 1000, (nb, 1))
    target = rng.normal(0, 1, (nb, nz * ny * nx, 4)).astype(np.float32)
    return feats.reshape(m, 3), target.reshape(m, 4)


def _layer_slices():
    out, off = [], 0
    for cin, cout, _ in no.LAYERS:
        nw = cout * 27 * cin
        out.append((slice(off, off + nw), slice(off + nw, off + nw + cout)))
        off += nw + cout
    return out


@pytest.mark.gpu
def test_param_count_matches_oracle(solver):
    assert capi.WarmNet.param_count() == no.param_count()


@pytest.mark.gpu
@pytest.mark.parametrize("nb,grid", [(1, DIMS[1:]), (2, DIMS[1:]), (1, (8, 16, 16))])
def test_forward_and_gradients_match_oracle(solver, nb, grid):
    """(8, 16, 16) runs the finest level on the halo-tiled kernels (NY a
    multiple of 16), bias gradients folded into their weight gradients."""
    dims = (nb,) + tuple(grid)
    net = capi.WarmNet(dims[3], dims[2], dims[1], max_batch=nb, seed=3)
    p = net.params()
    # give the output layer a larger scale so the prediction is not tiny
    sl = _layer_slices()
    p[sl[15][0]] *= 10.0
    net.set_params(p)
    feats, target = _inputs(7 + nb, dims)
    pred = net.forward(feats).reshape(-1, 4)
    loss_o, pred_o, g_o = no.net(p, dims, feats, target, bf16_mode=True)
    scale = float(np.abs(pred_o).max())
    assert float(np.abs(pred - pred_o).max()) <= 2e-2 * scale
    loss, g = net.loss_grad(feats, target)
    assert loss == pytest.approx(loss_o, rel=1e-2)
    for l, (ws, bs) in enumerate(sl):
        for part in (ws, bs):
            a, b = g[part].astype(np.float64), g_o[part].astype(np.float64)
            nb_ = np.linalg.norm(b)
            if nb_ == 0:
                assert np.linalg.norm(a) == 0
                continue
            cos = float(a @ b / (np.linalg.norm(a) * nb_))
            assert cos > 0.99, (l, cos)
            assert abs(np.linalg.norm(a) / nb_ - 1) < 0.05, (l, np.linalg.norm(a) / nb_)


@pytest.mark.gpu
def test_training_reduces_loss(solver):
    """Adam on a fixed smooth target (a function of the mask and U): the loss
    falls by an order of magnitude."""
    dims = (2, 8, 8, 16)
    net = capi.WarmNet(16, 8, 8, max_batch=2, seed=1)
    feats, _ = _inputs(5, dims)
    m = feats.shape[0]
    fluid = 1.0 - feats[:, 0]
    target = np.stack([0.5 * fluid, fluid * (1 + feats[:, 1] * 5), 0.1 * fluid,
                       np.zeros(m)], 1).astype(np.float32)
    net.set_grad_clip(5.0)
    losses = [net.train_step(feats, target, 3e-3) for _ in range(150)]
    assert all(np.isfinite(losses))
    assert losses[-1] < 0.1 * losses[0], (losses[0], losses[-1])


@pytest.mark.gpu
def test_warm_initialisation_decodes_prediction(solver):
    """With all weights zero and output bias (0.5, 1, 0, 0) the prediction is
    constant: the grid starts at rho = 1 + 0.5 U^2, u = (U, 0, 0) in fluid
    cells and rho = 1, u = 0 in solid cells."""
    net = capi.WarmNet(16, 8, 8, max_batch=1, seed=0)
    p = np.zeros(net.param_count(), np.float32)
    sl = _layer_slices()
    p[sl[15][1]] = [0.5, 1.0, 0.0, 0.0]
    net.set_params(p)
    g = capi.Grid(64, 32, 32, 0.02)
    g.set_solid_sphere(-2.0, 0.0, 0.0, 0.5)
    U = 0.04
    assert capi.load().LBM_InitializeFromWarmNet(g.handle, net.handle, U, 300.0, 0) == 0
    vel = g.velocity()
    solid = g.solid()
    fl = solid == 0
    assert np.allclose(vel[fl, 0], U, rtol=1e-6) and np.allclose(vel[fl, 1:3], 0)
    assert np.allclose(vel[fl, 3], np.float32(1 + 0.5 * U * U), rtol=1e-6)
    assert np.all(vel[~fl, :3] == 0) and np.all(vel[~fl, 3] == 1)
    g.step(U, n=20)
    assert np.isfinite(g.drag_force_decomposed()).all()
    # output scaling: physical = shift + scale * output
    net.set_output_scaling([2.0, 0.5, 1.0, 1.0], [0.25, 0.5, 0.0, 0.0])
    assert capi.load().LBM_InitializeFromWarmNet(g.handle, net.handle, U, 300.0, 0) == 0
    vel = g.velocity()
    assert np.allclose(vel[fl, 0], U, rtol=1e-6)  # 0.5 + 0.5 * 1
    assert np.allclose(vel[fl, 3], np.float32(1 + 1.25 * U * U), rtol=1e-6)  # 0.25 + 2 * 0.5
    net.set_output_scaling([1.0] * 4, [0.0] * 4)
    # velocity only: density stays 1
    assert capi.load().LBM_InitializeFromWarmNet(g.handle, net.handle, U, 300.0, 1) == 0
    vel = g.velocity()
    assert np.allclose(vel[fl, 0], U, rtol=1e-6) and np.all(vel[:, 3] == 1)


@pytest.mark.gpu
def test_grid_features_and_targets(solver):
    torch = pytest.importorskip("torch")
    g = capi.Grid(32, 16, 16, 0.05)
    g.set_solid_aabb(-3.0, -1.0, -1.0, -2.0, 1.0, 1.0)
    g.initialize_flow(0.05)
    g.step(0.05, n=10)
    feat = torch.zeros((16 * 8 * 8, 3), dtype=torch.float32, device="cuda")
    tgt = torch.zeros((16 * 8 * 8, 4), dtype=torch.float32, device="cuda")
    L = capi.load()
    assert L.LBM_WarmNetGridFeatures(g.handle, 2, 0.05, 400.0, feat.data_ptr()) == 0
    assert L.LBM_WarmNetGridTargets(g.handle, 2, 0.05, tgt.data_ptr()) == 0
    solid = (g.solid() == 1).reshape(16, 16, 32).astype(np.float32)
    frac = solid.reshape(8, 2, 8, 2, 16, 2).mean(axis=(1, 3, 5)).reshape(-1)
    f = feat.cpu().numpy()
    assert np.array_equal(f[:, 0], frac.astype(np.float32))
    assert np.all(f[:, 1] == np.float32(0.05)) and np.all(f[:, 2] == 400.0)
    vel = g.velocity().reshape(16, 16, 32, 4).astype(np.float64)
    sm = (g.solid() != 0).reshape(16, 16, 32)
    q = np.stack([(vel[..., 3] - 1) / 0.05 ** 2, vel[..., 0] / 0.05, vel[..., 1] / 0.05,
                  vel[..., 2] / 0.05], -1)
    q[sm] = 0
    ref = q.reshape(8, 2, 8, 2, 16, 2, 4).mean(axis=(1, 3, 5)).reshape(-1, 4)
    assert np.allclose(tgt.cpu().numpy(), ref, rtol=1e-4, atol=1e-4)


@pytest.mark.gpu
def test_warm_initialisation_flux_correction(solver):
    """LBM_WARM_FLUX_CORRECT: every x-plane carries the inlet mass flux and
    the outlet plane's fluid density averages 1."""
    net = capi.WarmNet(16, 8, 8, max_batch=1, seed=4)  # untrained: an arbitrary field
    g = capi.Grid(64, 32, 32, 0.02)
    g.set_solid_sphere(-2.0, 0.0, 0.0, 0.6)
    U = 0.05
    assert capi.load().LBM_InitializeFromWarmNet(g.handle, net.handle, U, 300.0, 2) == 0
    vel = g.velocity().reshape(32, 32, 64, 4).astype(np.float64)
    solid = g.solid().reshape(32, 32, 64)
    flux = (vel[..., 3] * vel[..., 0]).sum(axis=(0, 1))
    assert np.allclose(flux, U * 32 * 32, rtol=2e-3)
    out = vel[:, :, -1, 3][solid[:, :, -1] == 0]
    assert abs(out.mean() - 1.0) < 1e-5
