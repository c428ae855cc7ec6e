"""The warm-start network oracle checks itself: convolution adjoints by the
dot-product identity and the whole network's gradient by central finite
differences (FP32 storage, no bfloat16 rounding)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import nnoracle as no

DIMS = (1, 8, 8, 16)  # nb, nz, ny, nx


def _params(seed):
    rng = np.random.default_rng(seed)
    out = []
    for cin, cout, _ in no.LAYERS:
        out.append(rng.uniform(-1, 1, cout * 27 * cin) * np.sqrt(6.0 / (27 * cin)))
        out.append(rng.uniform(-0.1, 0.1, cout))
    return np.concatenate(out).astype(np.float32)


def _inputs(seed, dims=DIMS):
    rng = np.random.default_rng(seed)
    m = int(np.prod(dims))
    feats = np.stack([(rng.random(m) < 0.2).astype(np.float32),
                      np.full(m, 0.05, np.float32), np.full(m, 500.0, np.float32)], 1)
    target = rng.normal(0, 1, (m, 4)).astype(np.float32)
    return feats, target


def test_param_count():
    assert no.param_count() == sum(c * 27 * i + c for i, c, _ in no.LAYERS)
    assert 1.8e6 < no.param_count() < 2.1e6


@pytest.mark.parametrize("cin,cout", [(8, 16), (16, 32), (48, 16)])
def test_conv_adjoints(cin, cout):
    rng = np.random.default_rng(cin * cout)
    dims = (2, 4, 6, 8)
    m = int(np.prod(dims))
    x = rng.normal(size=(m, cin)).astype(np.float32)
    w = rng.normal(size=(cout, 27 * cin)).astype(np.float32)
    g = rng.normal(size=(m, cout)).astype(np.float32)
    y = no.conv_fwd(x, cin, w, None, cout, dims)
    dx = no.conv_dgrad(g, cout, w, cin, dims)
    dw, db = no.conv_wgrad(x, cin, g, cout, dims)
    lhs = float(np.sum(y.astype(np.float64) * g))
    assert lhs == pytest.approx(float(np.sum(x.astype(np.float64) * dx)), rel=1e-4)
    assert lhs == pytest.approx(float(np.sum(w.astype(np.float64) * dw)), rel=1e-4)
    assert np.allclose(db, g.sum(0), rtol=1e-4, atol=1e-3)


def test_conv_known_answer():
    # a single centre tap of weight 1 is the identity; the +x tap shifts
    dims = (1, 3, 3, 4)
    m = int(np.prod(dims))
    x = np.arange(m * 8, dtype=np.float32).reshape(m, 8)
    w = np.zeros((8, 27 * 8), np.float32)
    for c in range(8):
        w[c, 13 * 8 + c] = 1.0
    assert np.array_equal(no.conv_fwd(x, 8, w, None, 8, dims), x)
    w[:] = 0
    w[0, 14 * 8 + 0] = 1.0  # tap (0, 0, +1): y[x] = x[x + 1]
    y = no.conv_fwd(x, 8, w, None, 8, dims).reshape(3, 3, 4, 8)
    xx = x.reshape(3, 3, 4, 8)
    assert np.array_equal(y[:, :, :3, 0], xx[:, :, 1:, 0]) and np.all(y[:, :, 3, 0] == 0)


def test_network_gradient_finite_differences():
    p = _params(1)
    feats, target = _inputs(2)
    loss, _, g = no.net(p, DIMS, feats, target, bf16_mode=False)
    assert np.isfinite(loss) and g is not None
    rng = np.random.default_rng(3)
    # parameters of the first, a middle and the last layer, plus biases
    offsets, off = [], 0
    for cin, cout, _ in no.LAYERS:
        offsets.append(off)
        off += cout * 27 * cin + cout
    picks = []
    for layer in (0, 1, 7, 9, 13, 15):
        cin, cout, _ = no.LAYERS[layer]
        base = offsets[layer]
        picks += list(base + rng.integers(0, cout * 27 * cin, 3))
        picks.append(base + cout * 27 * cin + int(rng.integers(0, cout)))
    gmax = np.abs(g).max()
    for i in picks:
        h = 2e-3 * max(1.0, abs(float(p[i])))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (no.net(pp, DIMS, feats, target, False, False)[0] -
              no.net(pm, DIMS, feats, target, False, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 2e-2 * gmax + 5e-2 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.3, 1e-40], np.float32)
    r = no.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125)
    assert all(no.lib().nno_bf16(float(a)) == b for a, b in zip(v, r))
