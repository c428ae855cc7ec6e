"""The oracle's collision arithmetic against the reference's own C.

simulation/test/test_lbm.c:43-187 holds the reference's CPU mirrors of its
collision shader's arithmetic (weights, feq, cpu_forwardMRT,
cpu_inverseMRT).  tests/golden/make_ref_math.py ran them, compiled from the
reference tree (oracle/Makefile `ref`), on 2^20 seeded states and recorded
the SHA-256 of every output array.  Here the oracle (oracle/oracle_core.inc)
must reproduce each digest bit for bit; where oracle/_ref/libref_math.so is
present the oracle is also run beside the reference itself on fresh seeds.
"""
import ctypes as C
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_ref_math as rm  # noqa: E402

with open(os.path.join(HERE, "golden", "ref_math.json")) as _fh:
    GOLDEN = json.load(_fh)


def _oracle_lib(oracle):
    lib = oracle.lib()
    for name in rm.ORACLE_NAMES:
        getattr(lib, name).argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
    return lib


def _first_mismatch(a, b):
    bad = np.nonzero(np.any(a.view(np.uint32) != b.view(np.uint32), axis=1))[0]
    if bad.size == 0:
        return None
    k = int(bad[0])
    return f"{bad.size} rows differ; first row {k}: {a[k].tolist()} vs {b[k].tolist()}"


def test_oracle_reproduces_reference_digests(oracle):
    lib = _oracle_lib(oracle)
    state, fi, m = rm.inputs(GOLDEN["seed"], GOLDEN["n"])
    feq, fwd, inv = rm.outputs(lib, rm.ORACLE_NAMES, state, fi, m)
    assert [float(oracle.lib().or_weight_f32(i)) for i in range(19)] == GOLDEN["weights"]
    got = {"feq": rm.digest(feq), "forward_mrt": rm.digest(fwd), "inverse_mrt": rm.digest(inv)}
    for k in (0, 1, 2):
        s = GOLDEN["samples"][str(k)]
        np.testing.assert_array_equal(feq[k], np.float32(s["feq"]))
        np.testing.assert_array_equal(fwd[k], np.float32(s["forward_mrt"]))
        np.testing.assert_array_equal(inv[k], np.float32(s["inverse_mrt"]))
    assert got == GOLDEN["sha256"]


@pytest.mark.skipif(not os.path.exists(rm.REF_LIB),
                    reason="oracle/_ref/libref_math.so is built only where the reference tree is")
@pytest.mark.parametrize("seed", [1])
def test_oracle_equals_reference_live(oracle, seed):
    ref = rm.load_ref()
    lib = _oracle_lib(oracle)
    state, fi, m = rm.inputs(seed, 1 << 20)
    for name, a, b in zip(("feq", "forward_mrt", "inverse_mrt"),
                          rm.outputs(lib, rm.ORACLE_NAMES, state, fi, m),
                          rm.outputs(ref, rm.REF_NAMES, state, fi, m)):
        assert _first_mismatch(a, b) is None, (name, _first_mismatch(a, b))


@pytest.mark.skipif(not os.path.exists(rm.REF_LIB),
                    reason="oracle/_ref/libref_math.so is built only where the reference tree is")
def test_golden_digests_come_from_the_reference():
    ref = rm.load_ref()
    state, fi, m = rm.inputs(GOLDEN["seed"], GOLDEN["n"])
    feq, fwd, inv = rm.outputs(ref, rm.REF_NAMES, state, fi, m)
    assert {"feq": rm.digest(feq), "forward_mrt": rm.digest(fwd),
            "inverse_mrt": rm.digest(inv)} == GOLDEN["sha256"]
