"""The super-resolution upscaler's host pieces, without a GPU: the LTWS
weight format (simulation/src/superres.c:43-101) written and read back, the
reference's shipped model read by the same reader (where the reference tree
is present), and the oracle's trilinear skip and denormalisation on fields
whose answer is known."""
import os

import numpy as np
import pytest

from oracle import sr_oracle as so

REF_ASSETS = "/root/reference/simulation/assets"


def test_ltws_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.03, so.NWEIGHTS).astype(np.float32)
    path = str(tmp_path / "m.bin")
    so.write_ltws(path, w)
    got, shapes = so.read_ltws(path)
    assert shapes == so.SHAPES
    np.testing.assert_array_equal(got, w)
    assert os.path.getsize(path) == 12 + sum(4 + 4 * len(s) for s in so.SHAPES) + 4 * so.NWEIGHTS


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_ASSETS, "sr_model.bin")),
                    reason="the reference's shipped model is read only where its tree is")
def test_reference_model_format():
    w, shapes = so.read_ltws(os.path.join(REF_ASSETS, "sr_model.bin"))
    # the order compute_offsets assumes (superres.c:130-166): b0, W0, b1, W1, ...
    assert shapes == so.SHAPES and w.size == so.NWEIGHTS
    norm = np.fromfile(os.path.join(REF_ASSETS, "sr_model_norm.bin"), np.float32)
    assert norm.size == 8 and np.all(norm[4:] > 0)


def test_constant_field_zero_network():
    """With zero weights and biases the correction is 0, and the trilinear
    skip of a constant field is that constant in every fine cell."""
    dims = (5, 4, 3)
    c = np.tile(np.float32([0.04, -0.01, 0.002, 1.01]), (60, 1))
    fine, corr = so.upscale(c, dims, np.zeros(so.NWEIGHTS, np.float32), [0.01, 0, 0, 1],
                            [0.02, 0.01, 0.01, 0.005])
    assert fine.shape == (8 * 60, 4) and np.all(corr == 0)
    np.testing.assert_allclose(fine, np.tile(c[:1], (480, 1)), rtol=0, atol=2e-7)


def test_bias_only_network_adds_denormalised_bias():
    """W = 0: every fine cell gets skip + b3 (per sub-cell and channel),
    scaled by std."""
    dims = (3, 3, 2)
    w = np.zeros(so.NWEIGHTS, np.float32)
    b3 = np.arange(32, dtype=np.float32) * 0.01
    off = so.NWEIGHTS - 32 * 128 - 32
    w[off:off + 32] = b3
    c = np.zeros((18, 4), np.float32)
    fine, _ = so.upscale(c, dims, w, [0, 0, 0, 0], [2, 2, 2, 2])
    f = fine.reshape(4, 6, 6, 4)
    for s in range(8):
        dx, dy, dz = s & 1, (s >> 1) & 1, s >> 2
        np.testing.assert_allclose(f[dz::2, dy::2, dx::2], np.broadcast_to(2 * b3[4 * s:4 * s + 4],
                                                                           (2, 3, 3, 4)))
