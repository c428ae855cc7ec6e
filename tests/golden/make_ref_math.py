"""Fixture pinning the collision arithmetic to the reference's own C.

The reference ships plain-C mirrors of its collision shader's arithmetic in
simulation/test/test_lbm.c:43-187 (weights, velocity set, feq,
cpu_forwardMRT, cpu_inverseMRT).  ``make -C oracle ref
REFSIM=<reference>/simulation`` cuts that block out of the test file and
compiles it, with -ffp-contract=off, into oracle/_ref/libref_math.so.  This
script runs it on a seeded set of 2^20 states (``inputs`` below, shared by
the tests) and records the SHA-256 of each output array, plus a few sample
rows, in tests/golden/ref_math.json.  The tests then require the oracle
(CPU) and the CUDA kernels (GPU) to reproduce those digests bit for bit,
without needing the reference tree at run time.

Input domain (the solver's): rho in [0.3, 2]; velocity components in
[-0.25, 0.25], some exactly 0 and some tiny (down to 1e-36); populations
near w_i rho; moment vectors with m_0 = rho in [0.3, 2] and the other
moments spread over eight decades, some tiny.

Run:  python tests/golden/make_ref_math.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_math.so")
OUT = os.path.join(HERE, "ref_math.json")
SEED = 20261204
N = 1 << 20

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)


def inputs(seed: int = SEED, n: int = N):
    """(state [n, 4], fi [n, 19], m [n, 19]) float32, deterministic in seed."""
    rng = np.random.default_rng(seed)
    rho = rng.uniform(0.3, 2.0, n)
    u = rng.uniform(-0.25, 0.25, (n, 3))
    kind = rng.integers(0, 100, n)
    comp = rng.integers(0, 3, n)
    rows = np.arange(n)
    zero = kind < 5                       # one component exactly zero
    u[rows[zero], comp[zero]] = 0.0
    tiny = (kind >= 5) & (kind < 7)       # one tiny component
    mag = 10.0 ** rng.uniform(-36, -20, n)
    sgn = np.where(rng.integers(0, 2, n) == 0, -1.0, 1.0)
    u[rows[tiny], comp[tiny]] = (sgn * mag)[tiny]
    u[kind == 7] = 0.0                    # at rest
    state = np.column_stack([rho, u]).astype(np.float32)

    fi = (W[None, :] * rho[:, None] * (1.0 + rng.uniform(-0.4, 0.4, (n, 19)))).astype(np.float32)
    fz = rng.integers(0, 100, n) < 2
    fi[fz, rng.integers(0, 19, int(fz.sum()))] = 0.0

    m = rng.uniform(-1.0, 1.0, (n, 19)) * 10.0 ** rng.uniform(-8, 0, (n, 19)) * rho[:, None]
    m[:, 0] = rho
    mt = rng.integers(0, 100, (n, 19)) < 2
    mt[:, 0] = False
    m[mt] = (rng.uniform(-1, 1, int(mt.sum())) * 1e-35)
    return state, fi, m.astype(np.float32)


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


def load_ref(path: str = REF_LIB) -> C.CDLL:
    lib = C.CDLL(path)
    for name in ("ref_feq_batch", "ref_forward_mrt_batch", "ref_inverse_mrt_batch"):
        getattr(lib, name).argtypes = [C.c_int64, C.c_void_p, C.c_void_p]
    lib.ref_weight.restype = C.c_float
    lib.ref_weight.argtypes = [C.c_int]
    return lib


def run_batch(fn, n: int, inp: np.ndarray) -> np.ndarray:
    out = np.empty((n, 19), np.float32)
    inp = np.ascontiguousarray(inp)
    fn(n, inp.ctypes.data, out.ctypes.data)
    return out


def outputs(lib, names, state, fi, m):
    """(feq, forward, inverse) of one library whose batch functions are
    named by `names`."""
    n = state.shape[0]
    return (run_batch(getattr(lib, names[0]), n, state),
            run_batch(getattr(lib, names[1]), n, fi),
            run_batch(getattr(lib, names[2]), n, m))


REF_NAMES = ("ref_feq_batch", "ref_forward_mrt_batch", "ref_inverse_mrt_batch")
ORACLE_NAMES = ("or_feq_batch_f32", "or_mrt_forward_batch_f32", "or_mrt_inverse_batch_f32")


def main() -> int:
    if not os.path.exists(REF_LIB):
        sys.exit(f"{REF_LIB} missing: run `make -C oracle ref REFSIM=<reference>/simulation`")
    lib = load_ref()
    state, fi, m = inputs()
    feq, fwd, inv = outputs(lib, REF_NAMES, state, fi, m)
    doc = {
        "source": "simulation/test/test_lbm.c:43-187 (feq, cpu_forwardMRT, cpu_inverseMRT), "
                  "compiled by `make -C oracle ref` with -ffp-contract=off",
        "generator": "tests/golden/make_ref_math.py inputs()",
        "seed": SEED, "n": N,
        "weights": [float(lib.ref_weight(i)) for i in range(19)],
        "sha256": {"feq": digest(feq), "forward_mrt": digest(fwd), "inverse_mrt": digest(inv)},
        "samples": {str(k): {"state": state[k].tolist(), "feq": feq[k].tolist(),
                             "fi": fi[k].tolist(), "forward_mrt": fwd[k].tolist(),
                             "m": m[k].tolist(), "inverse_mrt": inv[k].tolist()}
                    for k in (0, 1, 2)},
    }
    with open(OUT, "w") as fh:
        json.dump(doc, fh, indent=1)
    print(f"wrote {OUT}: {doc['sha256']}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
