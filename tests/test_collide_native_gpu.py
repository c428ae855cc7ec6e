"""Collision arithmetic on the device: the paired-FP32 build of every
collision operator must be bit-identical to the one-scalar-operation
build, and the two-cells-per-thread collision of the paired step kernel to
the one-cell collision, on 2^20 random states including inlet / outlet
cells and guard resets (tests/native/collide_check.cu); and the device's equilibrium and MRT
transforms must reproduce, bit for bit, the reference's own C mirrors of
them (simulation/test/test_lbm.c:43-187) on the 2^20 seeded states of
tests/golden/ref_math.json."""
import json
import os
import subprocess
import sys

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
        outs[tag] = np.fromfile(path, np.float32).reshape(12, n, 19)
    a, b = outs["paired"].view(np.uint32), outs["scalar"].view(np.uint32)
    report = []
    for k, name in enumerate(OPS):
        # two cells per thread (paired f32x2 across cells) vs one cell per thread
        d2 = np.any(a[6 + k] != a[k], axis=1)
        report.append(f"{name}: two-cell collision differs from one-cell in {int(d2.sum())} "
                      f"of {n} states")
        if d2.any():
            i = int(np.argmax(d2))
            cols = np.nonzero(a[6 + k, i] != a[k, i])[0]
            report.append(f"   first state {i}, directions {cols.tolist()}: "
                          f"{outs['paired'][6 + k, i, cols]} vs {outs['paired'][k, i, cols]}")
    for k, name in enumerate(OPS + [o + " (two-cell)" for o in OPS]):
        diff = np.any(a[k] != b[k], axis=1)
        report.append(f"{name}: {int(diff.sum())} of {n} states differ")
        if diff.any():
            i = int(np.argmax(diff))
            cols = np.nonzero(a[k, i] != b[k, i])[0]
            report.append(f"   first state {i}, directions {cols.tolist()}: "
                          f"{outs['paired'][k, i, cols]} vs {outs['scalar'][k, i, cols]}")
    print("\n".join(report))
    assert np.array_equal(a, b), "\n".join(report)
    assert np.array_equal(a[6:], a[:6]), "\n".join(report)


def test_device_math_equals_reference_c(tmp_path):
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_ref_math as rm
    with open(os.path.join(HERE, "golden", "ref_math.json")) as fh:
        golden = json.load(fh)
    state, fi, m = rm.inputs(golden["seed"], golden["n"])
    n = state.shape[0]
    paths = [str(tmp_path / f"{k}.bin") for k in ("state", "fi", "m", "out")]
    for arr, path in zip((state, fi, m), paths):
        np.ascontiguousarray(arr).tofile(path)
    exe = _build(tmp_path, "paired", [])
    r = subprocess.run([exe, "--math", *paths[:3], str(n), paths[3]], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(paths[3], np.float32).reshape(7, n, 19)
    want = golden["sha256"]
    got = {"feq (one direction at a time)": rm.digest(out[0]),
           "equilibria (the step's)": rm.digest(out[1]),
           "forward_mrt": rm.digest(out[2]), "inverse_mrt": rm.digest(out[3]),
           "equilibria (two-cell step)": rm.digest(out[4]),
           "forward_mrt (two-cell step)": rm.digest(out[5]),
           "inverse_mrt (two-cell step)": rm.digest(out[6])}
    expect = {"feq (one direction at a time)": want["feq"], "equilibria (the step's)": want["feq"],
              "forward_mrt": want["forward_mrt"], "inverse_mrt": want["inverse_mrt"],
              "equilibria (two-cell step)": want["feq"],
              "forward_mrt (two-cell step)": want["forward_mrt"],
              "inverse_mrt (two-cell step)": want["inverse_mrt"]}
    report = []
    for name in got:
        if got[name] != expect[name]:
            report.append(f"{name}: digest differs from the reference's")
    if report:
        # locate the first differing rows against the oracle, which is pinned
        # to the same digests on the CPU
        from oracle import pyoracle
        import ctypes as C
        lib = pyoracle.lib()
        for nm in rm.ORACLE_NAMES:
            getattr(lib, nm).argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
        feq, fwd, inv = rm.outputs(lib, rm.ORACLE_NAMES, state, fi, m)
        for k, ref in zip(range(7), (feq, feq, fwd, inv, feq, fwd, inv)):
            bad = np.nonzero(np.any(out[k].view(np.uint32) != ref.view(np.uint32), axis=1))[0]
            if bad.size:
                i = int(bad[0])
                report.append(f"output {k}: {bad.size} rows differ; row {i}: "
                              f"{out[k][i].tolist()} vs {ref[i].tolist()}")
    assert not report, "\n".join(report)
