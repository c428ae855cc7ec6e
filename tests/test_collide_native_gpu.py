"""Collision arithmetic on the device: the paired-FP32 build of every
collision operator must be bit-identical to the one-scalar-operation
build (tests/native/collide_check.cu)."""
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
OPS = ["BGK", "REG", "MRT", "BGK+Smag", "REG+Smag", "MRT+Smag"]


def _build(tmp, tag, extra):
    exe = str(tmp / f"collide_check_{tag}")
    subprocess.run([NVCC, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "--fmad=false", *extra, "-o", exe,
                    os.path.join(HERE, "native", "collide_check.cu")], check=True)
    return exe


def test_paired_collision_bitexact(tmp_path):
    n = 1 << 20
    outs = {}
    for tag, extra in (("paired", []), ("scalar", ["-DLBM_NO_PAIRED"])):
        exe = _build(tmp_path, tag, extra)
        path = str(tmp_path / f"{tag}.bin")
        r = subprocess.run([exe, path, str(n)], capture_output=True, text=True)
        print(tag, r.stdout.strip())
        assert r.returncode == 0, r.stderr
        outs[tag] = np.fromfile(path, np.float32).reshape(6, n, 19)
    a, b = outs["paired"].view(np.uint32), outs["scalar"].view(np.uint32)
    report = []
    for k, name in enumerate(OPS):
        diff = np.any(a[k] != b[k], axis=1)
        report.append(f"{name}: {int(diff.sum())} of {n} states differ")
        if diff.any():
            i = int(np.argmax(diff))
            cols = np.nonzero(a[k, i] != b[k, i])[0]
            report.append(f"   first state {i}, directions {cols.tolist()}: "
                          f"{outs['paired'][k, i, cols]} vs {outs['scalar'][k, i, cols]}")
    print("\n".join(report))
    assert np.array_equal(a, b), "\n".join(report)
