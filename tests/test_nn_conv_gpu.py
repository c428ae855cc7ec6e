"""Tensor-core convolution kernels of the warm-start network (forward, input
gradient, weight gradient) against the CPU oracle on the same
bfloat16-representable inputs.  Tolerance: 1e-2 of the largest magnitude
(bfloat16 output rounding is 2^-9 relative; accumulation order differs)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from lattice_fluid_dynamics_b200 import capi
from oracle import nnoracle as no

torch = pytest.importorskip("torch")


def _dev_bf16(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).to("cuda").to(torch.bfloat16)


def _padded_weights(w, cout_pad, cin):
    """[cout][27 cin] -> bf16 [cout_pad][k_pad]"""
    kp = capi.load().LBM_NNKPad(cin)
    out = np.zeros((cout_pad, kp), np.float32)
    out[:w.shape[0], :w.shape[1]] = w
    return _dev_bf16(out)


def _close(a, b, tol=1e-2):
    scale = max(float(np.abs(b).max()), 1e-6)
    err = float(np.abs(a - b).max())
    assert err <= tol * scale, (err, scale)


CASES = [  # cin, cout, cout_pad, dims (nb, nz, ny, nx)
    (8, 16, 16, (1, 8, 8, 16)),
    (16, 32, 32, (2, 4, 8, 16)),
    (48, 16, 16, (1, 8, 8, 16)),
    (32, 64, 64, (1, 4, 8, 8)),
    (192, 64, 64, (1, 4, 4, 8)),
    (64, 128, 128, (2, 2, 4, 8)),
    (16, 4, 16, (1, 8, 8, 16)),
    (96, 32, 32, (1, 4, 8, 8)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,cout_pad,dims", CASES)
def test_conv_forward(solver, cin, cout, cout_pad, dims):
    L = capi.load()
    rng = np.random.default_rng(cin + cout)
    m = int(np.prod(dims))
    x = no.bf16(rng.normal(size=(m, cin)))
    w = no.bf16(rng.normal(size=(cout, 27 * cin)) / np.sqrt(27 * cin))
    b = rng.normal(size=cout_pad).astype(np.float32)
    b[cout:] = 0
    xd, wd = _dev_bf16(x), _padded_weights(w, cout_pad, cin)
    bd = torch.from_numpy(b).cuda()
    store = ((cout + 7) // 8) * 8
    for act in (0, 1):
        y = torch.zeros((m, cout_pad), dtype=torch.bfloat16, device="cuda")
        y32 = torch.zeros((m, cout_pad), dtype=torch.float32, device="cuda")
        rc = L.LBM_NNConvForward(xd.data_ptr(), cin, 0, cin, wd.data_ptr(), bd.data_ptr(),
                                 cout_pad, act, y.data_ptr(), y32.data_ptr(), cout_pad, 0, store,
                                 0, *dims, None)
        assert rc == 0
        assert L.LBM_NNTakeError() == 0
        ref = no.conv_fwd(x, cin, w, b[:cout], cout, dims)
        if act:
            ref = np.where(ref > 0, ref, 0.1 * ref)
        _close(y32.cpu().numpy()[:, :cout], ref, 1e-4)
        _close(y.float().cpu().numpy()[:, :cout], ref)


@pytest.mark.gpu
def test_conv_forward_slices(solver):
    """input and output as channel slices of wider buffers, fp32 accumulate"""
    L = capi.load()
    rng = np.random.default_rng(5)
    dims = (1, 4, 8, 16)
    m = int(np.prod(dims))
    wide = no.bf16(rng.normal(size=(m, 48)))
    w = no.bf16(rng.normal(size=(32, 27 * 16)) / 10)
    xd, wd = _dev_bf16(wide), _padded_weights(w, 32, 16)
    y32 = torch.ones((m, 64), dtype=torch.float32, device="cuda")
    assert L.LBM_NNConvForward(xd.data_ptr(), 48, 16, 16, wd.data_ptr(), None, 32, 0, None,
                               y32.data_ptr(), 64, 24, 32, 1, *dims, None) == 0
    ref = no.conv_fwd(wide, 16, w, None, 32, dims, xs=48, xo=16)
    out = y32.cpu().numpy()
    _close(out[:, 24:56] - 1.0, ref, 1e-4)
    assert np.all(out[:, :24] == 1.0) and np.all(out[:, 56:] == 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,cout_pad,dims", CASES)
def test_conv_input_gradient(solver, cin, cout, cout_pad, dims):
    L = capi.load()
    rng = np.random.default_rng(7 + cin)
    m = int(np.prod(dims))
    g = np.zeros((m, cout_pad), np.float32)
    g[:, :cout] = no.bf16(rng.normal(size=(m, cout)))
    w = no.bf16(rng.normal(size=(cout, 27 * cin)) / np.sqrt(27 * cin))
    wd = _padded_weights(w, cout_pad, cin)
    cin_pad = ((cin + 15) // 16) * 16
    wt = torch.zeros((cin_pad, L.LBM_NNKPad(cout_pad)), dtype=torch.bfloat16, device="cuda")
    assert L.LBM_NNWeightTranspose(wd.data_ptr(), cout_pad, cin, wt.data_ptr(), cin_pad,
                                   None) == 0
    gd = _dev_bf16(g)
    dx = torch.zeros((m, cin), dtype=torch.float32, device="cuda")
    assert L.LBM_NNConvForward(gd.data_ptr(), cout_pad, 0, cout_pad, wt.data_ptr(), None,
                               cin_pad, 0, None, dx.data_ptr(), cin, 0, cin, 0, *dims,
                               None) == 0
    assert L.LBM_NNTakeError() == 0
    ref = no.conv_dgrad(g[:, :cout], cout, w, cin, dims)
    _close(dx.cpu().numpy(), ref, 1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,cout_pad,dims", [c for c in CASES if c[2] in (16, 32, 64, 128)])
@pytest.mark.parametrize("chunks", [1, 3])
def test_conv_weight_gradient(solver, cin, cout, cout_pad, dims, chunks):
    L = capi.load()
    rng = np.random.default_rng(11 + cin + cout)
    m = int(np.prod(dims))
    x = no.bf16(rng.normal(size=(m, cin)))
    g = np.zeros((m, cout_pad), np.float32)
    g[:, :cout] = no.bf16(rng.normal(size=(m, cout)))
    xd, gd = _dev_bf16(x), _dev_bf16(g)
    cstore = ((cout + 7) // 8) * 8
    ws_bytes = L.LBM_NNWgradWorkspaceBytes(cin, cout_pad, *dims, chunks)
    ws = torch.zeros(ws_bytes // 4, dtype=torch.float32, device="cuda")
    dw = torch.full((cstore, 27 * cin), 0.5, dtype=torch.float32, device="cuda")
    assert L.LBM_NNConvWeightGrad(xd.data_ptr(), cin, 0, cin, gd.data_ptr(), cout_pad, cstore,
                                  cout_pad, dw.data_ptr(), 0, ws.data_ptr(), ws_bytes, chunks,
                                  *dims, None) == 0
    assert L.LBM_NNTakeError() == 0
    ref, _ = no.conv_wgrad(x, cin, g[:, :cout], cout, dims)
    _close(dw.cpu().numpy()[:cout], ref, 1e-4)
    # accumulate mode adds
    assert L.LBM_NNConvWeightGrad(xd.data_ptr(), cin, 0, cin, gd.data_ptr(), cout_pad, cstore,
                                  cout_pad, dw.data_ptr(), 1, ws.data_ptr(), ws_bytes, chunks,
                                  *dims, None) == 0
    _close(dw.cpu().numpy()[:cout], 2 * ref, 1e-4)


HALO_CASES = [  # shapes the halo-tiled forward kernel takes: cin % 16, NX % 8, NY % 16
    (16, 16, 16, (2, 3, 16, 16)),
    (48, 16, 16, (1, 2, 32, 8)),
    (16, 32, 32, (1, 3, 16, 24)),
    (96, 32, 32, (2, 2, 16, 8)),
    (16, 48, 48, (1, 2, 16, 16)),
    (32, 64, 64, (1, 2, 16, 8)),
    (32, 96, 96, (1, 1, 32, 16)),
    (16, 4, 16, (1, 4, 16, 8)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,cout_pad,dims", HALO_CASES)
def test_conv_forward_halo(solver, cin, cout, cout_pad, dims):
    """The halo-tiled kernel against the oracle and against the gather
    kernel on the same inputs, with the output as a slice of a wider
    buffer and the input a channel slice as well."""
    L = capi.load()
    rng = np.random.default_rng(3 * cin + cout)
    m = int(np.prod(dims))
    xs, xo = cin + 16, 16
    wide = no.bf16(rng.normal(size=(m, xs)))
    w = no.bf16(rng.normal(size=(cout, 27 * cin)) / np.sqrt(27 * cin))
    b = rng.normal(size=cout_pad).astype(np.float32)
    b[cout:] = 0
    xd, wd = _dev_bf16(wide), _padded_weights(w, cout_pad, cin)
    bd = torch.from_numpy(b).cuda()
    store = ((cout + 7) // 8) * 8
    ys, yo = cout_pad + 8, 8
    ref = no.conv_fwd(wide, cin, w, b[:cout], cout, dims, xs=xs, xo=xo)
    ref = np.where(ref > 0, ref, 0.1 * ref)
    outs = {}
    try:
        for path in (0, 1, 2, 3):
            assert L.LBM_NNSetConvPath(path) == 0
            y = torch.full((m, ys), 7.0, dtype=torch.bfloat16, device="cuda")
            y32 = torch.full((m, ys), 7.0, dtype=torch.float32, device="cuda")
            rc = L.LBM_NNConvForward(xd.data_ptr(), xs, xo, cin, wd.data_ptr(), bd.data_ptr(),
                                     cout_pad, 1, y.data_ptr(), y32.data_ptr(), ys, yo, store, 0,
                                     *dims, None)
            assert rc == 0
            assert L.LBM_NNTakeError() == 0
            o32 = y32.cpu().numpy()
            _close(o32[:, yo:yo + cout], ref, 1e-4)
            _close(y.float().cpu().numpy()[:, yo:yo + cout], ref)
            assert np.all(o32[:, :yo] == 7.0) and np.all(o32[:, yo + store:] == 7.0)
            outs[path] = o32
    finally:
        L.LBM_NNSetConvPath(0)
    # the kernels accumulate the same products in FP32, in different orders
    _close(outs[0][:, yo:yo + cout], outs[1][:, yo:yo + cout], 1e-5)
    _close(outs[2][:, yo:yo + cout], outs[1][:, yo:yo + cout], 1e-5)
    _close(outs[3][:, yo:yo + cout], outs[1][:, yo:yo + cout], 1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,cout_pad,dims", [c for c in HALO_CASES if c[2] % 16 == 0])
def test_conv_input_gradient_halo(solver, cin, cout, cout_pad, dims):
    """The input gradient through the halo kernel: the gradient buffer has
    cout_pad (a multiple of 16) channels; output channels cin."""
    L = capi.load()
    rng = np.random.default_rng(17 + cin + cout)
    m = int(np.prod(dims))
    g = np.zeros((m, cout_pad), np.float32)
    g[:, :cout] = no.bf16(rng.normal(size=(m, cout)))
    w = no.bf16(rng.normal(size=(cout, 27 * cin)) / np.sqrt(27 * cin))
    wd = _padded_weights(w, cout_pad, cin)
    cin_pad = ((cin + 15) // 16) * 16
    wt = torch.zeros((cin_pad, L.LBM_NNKPad(cout_pad)), dtype=torch.bfloat16, device="cuda")
    assert L.LBM_NNWeightTranspose(wd.data_ptr(), cout_pad, cin, wt.data_ptr(), cin_pad,
                                   None) == 0
    gd = _dev_bf16(g)
    ref = no.conv_dgrad(g[:, :cout], cout, w, cin, dims)
    try:
        for path in (0, 3):
            assert L.LBM_NNSetConvPath(path) == 0
            dx = torch.zeros((m, cin), dtype=torch.float32, device="cuda")
            assert L.LBM_NNConvForward(gd.data_ptr(), cout_pad, 0, cout_pad, wt.data_ptr(), None,
                                       cin_pad, 0, None, dx.data_ptr(), cin, 0, cin, 0, *dims,
                                       None) == 0
            assert L.LBM_NNTakeError() == 0
            _close(dx.cpu().numpy(), ref, 1e-4)
    finally:
        L.LBM_NNSetConvPath(0)


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,cout_pad,dims",
                         [c for c in HALO_CASES if c[2] in (16, 32, 64)] +
                         [(16, 128, 128, (1, 2, 16, 8)), (32, 16, 16, (4, 8, 32, 16))])
def test_conv_weight_gradient_paths(solver, cin, cout, cout_pad, dims):
    """The weight gradient with MN-major operands (default) against the
    oracle and against the gather kernel, with the input a channel slice of
    a wider buffer."""
    L = capi.load()
    rng = np.random.default_rng(23 + cin + cout)
    m = int(np.prod(dims))
    xs, xo = cin + 16, 16
    wide = no.bf16(rng.normal(size=(m, xs)))
    g = np.zeros((m, cout_pad), np.float32)
    g[:, :cout] = no.bf16(rng.normal(size=(m, cout)))
    xd, gd = _dev_bf16(wide), _dev_bf16(g)
    cstore = ((cout + 7) // 8) * 8
    ws_bytes = L.LBM_NNWgradWorkspaceBytes(cin, cout_pad, *dims, 1)
    ws = torch.zeros(ws_bytes // 4, dtype=torch.float32, device="cuda")
    ref, _ = no.conv_wgrad(np.ascontiguousarray(wide[:, xo:xo + cin]), cin, g[:, :cout], cout,
                           dims)
    outs = {}
    try:
        for path in (0, 1):
            assert L.LBM_NNSetConvPath(path) == 0
            dw = torch.full((cstore, 27 * cin), 0.5, dtype=torch.float32, device="cuda")
            assert L.LBM_NNConvWeightGrad(xd.data_ptr(), xs, xo, cin, gd.data_ptr(), cout_pad,
                                          cstore, cout_pad, dw.data_ptr(), 0, ws.data_ptr(),
                                          ws_bytes, 1, *dims, None) == 0
            assert L.LBM_NNTakeError() == 0
            outs[path] = dw.cpu().numpy()[:cout]
            _close(outs[path], ref, 1e-4)
    finally:
        L.LBM_NNSetConvPath(0)
    _close(outs[0], outs[1], 1e-5)


def test_nn_argument_checks_cpu():
    L = capi.load()
    assert L.LBM_NNKPad(8) == 256 and L.LBM_NNKPad(16) == 512 and L.LBM_NNKPad(192) == 5248
    # misaligned channel counts are rejected before any device work
    assert L.LBM_NNConvForward(1, 12, 0, 12, 1, None, 16, 0, 1, None, 16, 0, 16, 0,
                               1, 8, 8, 8, None) == 1
    assert L.LBM_NNConvWeightGrad(1, 8, 0, 8, 1, 16, 12, 16, 1, 0, 1, 1 << 30, 1,
                                  1, 8, 8, 8, None) == 1
    assert L.LBM_NNSetConvPath(4) == 1 and L.LBM_NNSetConvPath(0) == 0
