"""The tensor-core super-resolution upscaler (LBM_SuperRes*) against the CPU
oracle of simulation/shaders/superres_upscale.comp (oracle/sr_oracle.py).

The kernel multiplies BF16 operands with FP32 accumulation.  Against the
oracle with the same BF16 operand rounding the outputs agree to FP32
summation-order noise plus, rarely, one BF16 step of a hidden activation:
|error| <= 5e-3 x max |correction|.  Against the oracle's plain FP32 network
(the shader's arithmetic) the BF16 operands cost more: <= 5e-2 x max
|correction|.  The trilinear skip and the denormalisation are FP32 on both
sides."""
import numpy as np
import pytest

from oracle import sr_oracle as so

pytestmark = pytest.mark.gpu


def _weights(seed, scale=0.04):
    rng = np.random.default_rng(seed)
    return rng.uniform(-scale, scale, so.NWEIGHTS).astype(np.float32)


def _run(solver, dims, w, mean, std, field):
    import torch
    from lattice_fluid_dynamics_b200 import capi
    sr = capi.SuperRes(*dims, weights=w, mean=mean, std=std)
    dev = torch.from_numpy(np.ascontiguousarray(field, np.float32)).cuda()
    torch.cuda.synchronize()
    sr.upscale(dev.data_ptr())
    out = sr.fine()
    assert sr.fine_size() == tuple(2 * d for d in dims)
    sr.close()
    return out


def _check(out, field, dims, w, mean, std):
    ref16, corr = so.upscale(field, dims, w, mean, std, bf16_operands=True)
    ref32, _ = so.upscale(field, dims, w, mean, std)
    scale = float(np.abs(corr).max()) * np.asarray(std, np.float32).max()
    e16 = float(np.abs(out - ref16).max())
    e32 = float(np.abs(out - ref32).max())
    print(f"dims {dims}: max |correction| x std {scale:.4g}; error vs BF16-operand oracle "
          f"{e16:.3g}, vs FP32 oracle {e32:.3g}")
    assert e16 <= 5e-3 * scale + 1e-6
    assert e32 <= 5e-2 * scale + 1e-6


@pytest.mark.parametrize("dims", [(20, 12, 9), (8, 8, 8), (3, 2, 1)])
def test_upscale_matches_oracle(solver, dims):
    rng = np.random.default_rng(sum(dims))
    n = int(np.prod(dims))
    field = np.column_stack([rng.normal(0.05, 0.02, n), rng.normal(0, 0.01, n),
                             rng.normal(0, 0.01, n), rng.normal(1.0, 0.003, n)])
    mean, std = [0.05, 0.0, 0.0, 1.0], [0.02, 0.01, 0.01, 0.003]
    w = _weights(1)
    out = _run(solver, dims, w, mean, std, field)
    _check(out, field, dims, w, mean, std)


def test_weights_file_and_flow_field(solver, tmp_path):
    """LBM_SuperResCreate reading an LTWS file and a normaliser file gives
    what the array constructor gives, on the velocity field of a grid."""
    from lattice_fluid_dynamics_b200 import capi
    from tests import scenarios as S
    g = S.make_gpu(solver, dict(dims=(24, 16, 12), visc=0.02, flags=dict(periodicYZ=1),
                                geometry=[("sphere", (-1.5, 0.0, 0.0, 0.6))]))
    g.step(0.05, n=30)
    field = g.velocity().reshape(-1, 4)
    w = _weights(2)
    mean, std = np.float32([0.04, 0.0, 0.0, 1.0]), np.float32([0.02, 0.01, 0.01, 0.01])
    wpath, npath = str(tmp_path / "sr.bin"), str(tmp_path / "norm.bin")
    so.write_ltws(wpath, w)
    np.concatenate([mean, std]).tofile(npath)
    sr = capi.SuperRes(24, 16, 12, weights_path=wpath, norm_path=npath)
    sr.upscale(g.velocity_device_ptr())
    out_file = sr.fine()
    sr.close()
    out_arr = _run(solver, (24, 16, 12), w, mean, std, field)
    np.testing.assert_array_equal(out_file, out_arr)
    _check(out_arr, field, (24, 16, 12), w, mean, std)
    g.close()


def test_bad_weights_rejected(solver, tmp_path):
    from lattice_fluid_dynamics_b200 import capi
    path = str(tmp_path / "short.bin")
    so.write_ltws(path, np.zeros(100, np.float32), shapes=[(100,)])
    with pytest.raises(RuntimeError):
        capi.SuperRes(4, 4, 4, weights_path=path)
    with pytest.raises(RuntimeError):
        capi.SuperRes(4, 4, 4, weights_path=str(tmp_path / "missing.bin"))
