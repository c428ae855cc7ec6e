"""The solver divides by compile-time constants with Markstein's
three-operation sequence instead of an IEEE division (see cdiv in
csrc/lbm_d3q19.cuh).  This test rebuilds the checker in tests/native and
confirms, on a strided sample of all 2^32 single-precision inputs, that the
sequence returns the IEEE quotient for every input with
2^-100 <= |x| <= 2^100 (the solver sends every other input to the IEEE
division).  Setting LBM_CDIV_STRIDE=1 checks all 2^32 inputs.
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))

# every divisor the FP32 collision divides by: cs2, 2 cs2^2, 2 cs2 (in float)
# and the MRT row norms (lbm_collide.comp:188-206)
DIVISORS = ["0.333333343", "0.222222254", "0.666666687", "19", "2394", "252", "10",
            "40", "36", "72", "12", "24"]


def test_markstein_constant_division(tmp_path):
    exe = str(tmp_path / "cdiv_check")
    subprocess.run(["gcc", "-O3", "-march=native", "-ffp-contract=off", "-o", exe,
                    os.path.join(HERE, "native", "cdiv_check.c"), "-lm"], check=True)
    stride = os.environ.get("LBM_CDIV_STRIDE", "4099")
    r = subprocess.run([exe, stride, *DIVISORS], capture_output=True, text=True)
    print(r.stdout)
    assert r.returncode == 0, r.stdout
    for line in r.stdout.splitlines():
        assert "in[2^-100,2^100]=0 " in line, line


def test_speed_guard_threshold():
    """The stability guard's length(u) > 0.4 (lbm_collide.comp:429-430) is
    evaluated as u2 > 0x3e23d70b: sqrt is correctly rounded and monotone, so
    checking every float in [0.1, 0.2] (below it sqrt(x) <= 0.317, above it
    sqrt(x) >= 0.447) proves the equivalence for all non-negative floats."""
    import numpy as np
    lo = np.float32(0.1).view(np.uint32)
    hi = np.float32(0.2).view(np.uint32)
    x = np.arange(lo, hi + 1, dtype=np.uint32).view(np.float32)
    T = np.uint32(0x3E23D70B).view(np.float32)
    np.testing.assert_array_equal(np.sqrt(x) > np.float32(0.4), x > T)
