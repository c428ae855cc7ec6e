"""CPU oracle of the super-resolution upscaler (TEST INFRASTRUCTURE ONLY).

A numpy restatement of simulation/shaders/superres_upscale.comp:141-216
(gatherPatch, trilinearSkip, the 108 -> 128 -> 128 -> 128 -> 32 MLP,
denormalisation) and of the LTWS weight reader of simulation/src/superres.c:
43-101.  Only the tests import it; the library never does.

Arithmetic: the patch, skip and output in float32 with the shader's operation
order; the dense layers accumulate in float64 (the shader sums in float32
sequentially; float64 is the sum it approximates).  With bf16=True the
layer inputs and the weights are first rounded to bfloat16 -- the operands
the tensor-core kernel multiplies -- so the comparison with the GPU isolates
its FP32 accumulation.
"""
from __future__ import annotations

import struct

import numpy as np

H, KIN, NOUT = 128, 108, 32
SHAPES = [(H,), (H, KIN), (H,), (H, H), (H,), (H, H), (NOUT,), (NOUT, H)]
NWEIGHTS = sum(int(np.prod(s)) for s in SHAPES)  # 51,104


def read_ltws(path: str):
    """(values float32, shapes) of an LTWS file: magic 'LTWS' as a
    little-endian uint32, version, parameter count, then per parameter its
    rank, extents and float32 values (superres.c:43-101)."""
    b = open(path, "rb").read()
    magic, _version, count = struct.unpack_from("<III", b, 0)
    if magic != 0x4C545753:
        raise ValueError("bad LTWS magic")
    off, vals, shapes = 12, [], []
    for _ in range(count):
        (rank,) = struct.unpack_from("<I", b, off)
        off += 4
        dims = struct.unpack_from("<" + "I" * rank, b, off)
        off += 4 * rank
        n = int(np.prod(dims)) if rank else 1
        vals.append(np.frombuffer(b, np.float32, n, off))
        off += 4 * n
        shapes.append(tuple(dims))
    return np.concatenate(vals), shapes


def write_ltws(path: str, weights: np.ndarray, shapes=SHAPES, version: int = 1) -> None:
    """The inverse of read_ltws for a flat weight vector in file order."""
    w = np.asarray(weights, np.float32)
    with open(path, "wb") as fh:
        fh.write(struct.pack("<III", 0x4C545753, version, len(shapes)))
        off = 0
        for s in shapes:
            n = int(np.prod(s))
            fh.write(struct.pack("<I", len(s)) + struct.pack("<" + "I" * len(s), *s))
            fh.write(w[off:off + n].tobytes())
            off += n


def split(weights: np.ndarray):
    """b0, W0, b1, W1, b2, W2, b3, W3 from the flat vector (the order of
    compute_offsets, superres.c:130-166)."""
    out, off = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(weights[off:off + n], np.float32).reshape(s))
        off += n
    return out


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 to bfloat16 (nearest, ties to even), as float32."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def upscale(coarse: np.ndarray, dims, weights: np.ndarray, mean, std, bf16_operands=False):
    """Fine field [8 n, 4] (x fastest, fine dims 2x) from the coarse field
    [n, 4] of dims (cx, cy, cz)."""
    cx, cy, cz = dims
    v = np.asarray(coarse, np.float32).reshape(cz, cy, cx, 4)
    mean = np.asarray(mean, np.float32)
    std = np.asarray(std, np.float32)
    norm = (v - mean) / std  # normalize_ch (:58-60)
    zi, yi, xi = np.meshgrid(np.arange(cz), np.arange(cy), np.arange(cx), indexing="ij")

    def at(dx, dy, dz):  # sampleCoarse with clamping (:48-54)
        return norm[np.clip(zi + dz, 0, cz - 1), np.clip(yi + dy, 0, cy - 1),
                    np.clip(xi + dx, 0, cx - 1)]

    patch = np.concatenate([at(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1)
                            for dx in (-1, 0, 1)], axis=-1).reshape(-1, KIN)
    # trilinearSkip (:95-129), float32 in the shader's order
    skip = np.zeros((cz * cy * cx, 8, 4), np.float32)
    for s in range(8):
        dx, dy, dz = s & 1, (s >> 1) & 1, s >> 2
        f = [np.float32(0.25) + np.float32(0.5) * np.float32(d) for d in (dx, dy, dz)]
        val = np.zeros((cz, cy, cx, 4), np.float32)
        for c in range(8):
            ccx, ccy, ccz = c & 1, (c >> 1) & 1, c >> 2
            wz = f[2] if ccz else np.float32(1) - f[2]
            wy = f[1] if ccy else np.float32(1) - f[1]
            wx = f[0] if ccx else np.float32(1) - f[0]
            w = np.float32(np.float32(wz * wy) * wx)
            val = (val + w * at(ccx, ccy, ccz)).astype(np.float32)
        skip[:, s] = val.reshape(-1, 4)
    b0, W0, b1, W1, b2, W2, b3, W3 = split(weights)
    rnd = bf16 if bf16_operands else (lambda a: np.asarray(a, np.float32))
    h = patch
    for b, W in ((b0, W0), (b1, W1), (b2, W2)):
        h = np.maximum(rnd(h).astype(np.float64) @ rnd(W).astype(np.float64).T + b, 0.0)
        h = h.astype(np.float32)
    corr = (rnd(h).astype(np.float64) @ rnd(W3).astype(np.float64).T + b3).astype(np.float32)
    out = ((skip + corr.reshape(-1, 8, 4)) * std + mean).astype(np.float32)
    # scatter the 2 x 2 x 2 sub-cells into the fine grid (:193-214)
    fine = np.zeros((2 * cz, 2 * cy, 2 * cx, 4), np.float32)
    o = out.reshape(cz, cy, cx, 8, 4)
    for s in range(8):
        dx, dy, dz = s & 1, (s >> 1) & 1, s >> 2
        fine[dz::2, dy::2, dx::2] = o[:, :, :, s]
    return fine.reshape(-1, 4), corr
