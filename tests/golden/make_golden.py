"""Generate the golden fixtures for OBJ ingestion and Strouhal extraction.

The expected outputs come from the reference's own C sources, compiled by
``make -C oracle ref REFSIM=<reference>/simulation`` into ``oracle/_ref/libref_host.so`` from
simulation/obj-file-loader/lib/model_loader.c, simulation/src/model_bounds.c
and simulation/src/drag_metrics.c (only possible where the reference tree is
present).  The inputs are synthetic: small OBJ files written below that
exercise the loader's corner cases (quads and n-gons truncated to their first
three references, v/vt/vn, v//vn and v/vt tokens, comments, vt/vn lines,
out-of-range and negative indices, tabs) and seeded Cl series.

The placement main.c applies between loading and bounds (simulation/src/
main.c:250-349) is not a callable function in the reference, so it is
restated here in float32 with libm's cosf/sinf; the reference's
computeModelBounds and createTriangleBuffer are then called with those
parameters.

Run:  python tests/golden/make_golden.py   (writes tests/golden/obj/*.obj and
tests/golden/host_golden.json)
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OBJ_DIR = os.path.join(HERE, "obj")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
OUT = os.path.join(HERE, "host_golden.json")


class RefModel(C.Structure):
    _fields_ = [("vertices", C.POINTER(C.c_float)), ("faces", C.POINTER(C.c_int)),
                ("vertexCount", C.c_int), ("faceCount", C.c_int)]


class RefBounds(C.Structure):
    _fields_ = [(n, C.c_float) for n in
                ("minX", "minY", "minZ", "maxX", "maxY", "maxZ",
                 "centerX", "centerY", "centerZ")]


def load_ref():
    if not os.path.exists(REF_LIB):
        sys.exit(f"{REF_LIB} missing: run `make -C oracle ref REFSIM=<reference>/simulation` where the reference tree exists")
    lib = C.CDLL(REF_LIB)
    lib.loadOBJ.restype = RefModel
    lib.loadOBJ.argtypes = [C.c_char_p]
    lib.freeModel.argtypes = [C.POINTER(RefModel)]
    lib.computeModelBounds.restype = RefBounds
    lib.computeModelBounds.argtypes = [C.POINTER(RefModel)] + [C.c_float] * 5
    lib.createTriangleBuffer.restype = C.POINTER(C.c_float)
    lib.createTriangleBuffer.argtypes = [C.POINTER(RefModel)] + [C.c_float] * 5 + [C.POINTER(C.c_int)]
    lib.compute_strouhal.restype = None
    lib.compute_strouhal.argtypes = [C.POINTER(C.c_float), C.c_int, C.c_int, C.c_float, C.c_float]
    return lib


# --------------------------------------------------------------------------
# synthetic OBJ inputs


def obj_cube_quads() -> str:
    """Unit cube with quad faces in mixed token formats: the loader keeps only
    the first three references of every face."""
    v = [(x, y, z) for x in (0.0, 1.0) for y in (0.0, 1.0) for z in (0.0, 1.0)]
    lines = ["# cube with quads", "o cube"]
    lines += [f"v {x:.6f} {y:.6f} {z:.6f}" for x, y, z in v]
    lines += ["vt 0 0", "vt 1 0", "vn 0 0 1"]
    quads = [(1, 2, 4, 3), (5, 7, 8, 6), (1, 5, 6, 2), (3, 4, 8, 7), (1, 3, 7, 5), (2, 6, 8, 4)]
    fmts = ["{}", "{}/1", "{}/1/1", "{}//1", "{}/2/1", "{}"]
    for q, fm in zip(quads, fmts):
        lines.append("f " + " ".join(fm.format(i) for i in q))
    lines.append("f\t1 2\t3")         # tab separators
    lines.append("f 1 2 3 4 5 6")     # hexagon: first three kept
    lines.append("f 1 2 99")          # out of range: skipped by the triangle buffer
    lines.append("f -1 -2 -3")        # relative indices: skipped (negative)
    lines.append("f 0 1 2")           # index 0: skipped
    return "\n".join(lines) + "\n"


def obj_ellipsoid(nt: int, npz: int, radii, center, seed: int) -> str:
    """Jittered UV ellipsoid (triangles only)."""
    rng = np.random.default_rng(seed)
    a, b, c = radii
    verts = []
    for i in range(nt + 1):
        th = math.pi * i / nt
        for j in range(npz):
            ph = 2 * math.pi * j / npz
            r = 1.0 + 0.02 * rng.standard_normal()
            verts.append((center[0] + a * r * math.sin(th) * math.cos(ph),
                          center[1] + b * r * math.cos(th),
                          center[2] + c * r * math.sin(th) * math.sin(ph)))
    faces = []
    for i in range(nt):
        for j in range(npz):
            p0 = i * npz + j + 1
            p1 = i * npz + (j + 1) % npz + 1
            p2 = (i + 1) * npz + j + 1
            p3 = (i + 1) * npz + (j + 1) % npz + 1
            faces += [(p0, p2, p1), (p1, p2, p3)]
    lines = [f"v {x:.7g} {y:.7g} {z:.7g}" for x, y, z in verts]
    lines += [f"f {p} {q} {r}" for p, q, r in faces]
    return "\n".join(lines) + "\n"


CASES = {
    "cube_quads": obj_cube_quads,
    # longest extent along x: no rotation
    "ellipsoid_x": lambda: obj_ellipsoid(10, 14, (3.0, 0.8, 1.1), (5.0, -2.0, 1.0), 1),
    # longest extent along z: rotated 90 degrees about y
    "ellipsoid_z": lambda: obj_ellipsoid(12, 16, (0.9, 1.2, 4.0), (-3.0, 0.5, 7.0), 2),
}


# --------------------------------------------------------------------------
# main.c:250-349 placement, restated in float32


def place(verts: np.ndarray, scale_cli: float = 0.0):
    libm = C.CDLL("libm.so.6")
    libm.cosf.restype = libm.sinf.restype = C.c_float
    libm.cosf.argtypes = libm.sinf.argtypes = [C.c_float]
    f32 = np.float32
    mn = verts.min(axis=0)
    mx = verts.max(axis=0)
    c = ((mn + mx) * f32(0.5)).astype(f32)
    ext = (mx - mn).astype(f32)
    max_dim = f32(max(ext[0], max(ext[1], ext[2])))
    s = f32(scale_cli) if scale_cli > 0 else f32(f32(2.4) / max_dim)
    off = [f32(-c[k] * s) for k in range(3)]
    xs = (verts[:, 0] * s + off[0]).astype(f32)
    zs = (verts[:, 2] * s + off[2]).astype(f32)
    rot = f32(90.0) if f32(zs.max() - zs.min()) > f32(xs.max() - xs.min()) else f32(0.0)
    rad = f32(f32(rot * f32(math.pi)) / f32(180.0))
    off[0] = f32(off[0] + f32(f32(-2.0) * f32(libm.cosf(rad))))
    off[2] = f32(off[2] + f32(f32(2.0) * f32(libm.sinf(rad))))
    return float(s), [float(o) for o in off], float(rot)


def strouhal_ref(lib, series: np.ndarray, substeps: int, L: float, U: float) -> str:
    """Run the reference's compute_strouhal and capture the line it prints."""
    arr = np.ascontiguousarray(series, np.float32)
    libc = C.CDLL(None)
    sys.stdout.flush()
    libc.fflush(None)
    saved = os.dup(1)
    with tempfile.TemporaryFile() as tmp:
        os.dup2(tmp.fileno(), 1)
        try:
            lib.compute_strouhal(arr.ctypes.data_as(C.POINTER(C.c_float)), len(arr), substeps,
                                 L, U)
            libc.fflush(None)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        tmp.seek(0)
        return tmp.read().decode().strip()


def main():
    lib = load_ref()
    os.makedirs(OBJ_DIR, exist_ok=True)
    golden = {"obj": {}, "strouhal": []}
    for name, make in CASES.items():
        path = os.path.join(OBJ_DIR, name + ".obj")
        with open(path, "w") as fh:
            fh.write(make())
        m = lib.loadOBJ(path.encode())
        nv, nf = m.vertexCount, m.faceCount
        verts = np.ctypeslib.as_array(m.vertices, (nv, 3)).copy()
        faces = np.ctypeslib.as_array(m.faces, (nf, 3)).copy()
        s, off, rot = place(verts)
        b = lib.computeModelBounds(C.byref(m), s, off[0], off[1], off[2], rot)
        cnt = C.c_int()
        tp = lib.createTriangleBuffer(C.byref(m), s, off[0], off[1], off[2], rot, C.byref(cnt))
        tris = np.ctypeslib.as_array(tp, (cnt.value, 12)).copy()
        C.CDLL(None).free(C.cast(tp, C.c_void_p))
        # an explicit scale and a non-trivial angle exercise the general rotation
        cnt2 = C.c_int()
        tp2 = lib.createTriangleBuffer(C.byref(m), 0.37, 0.25, -0.5, 1.5, 33.0, C.byref(cnt2))
        tris2 = np.ctypeslib.as_array(tp2, (cnt2.value, 12)).copy()
        C.CDLL(None).free(C.cast(tp2, C.c_void_p))
        b2 = lib.computeModelBounds(C.byref(m), 0.37, 0.25, -0.5, 1.5, 33.0)
        lib.freeModel(C.byref(m))
        golden["obj"][name] = {
            "vertexCount": nv, "faceCount": nf,
            "vertices_hex": verts.astype("<f4").tobytes().hex(),
            "faces": faces.tolist(),
            "placement": {"scale": s, "offset": off, "rotationY": rot},
            "bounds_hex": np.array([getattr(b, f) for f, _ in RefBounds._fields_],
                                   "<f4").tobytes().hex(),
            "triangles_hex": tris.astype("<f4").tobytes().hex(),
            "triangleCount": int(cnt.value),
            "general": {"scale": 0.37, "offset": [0.25, -0.5, 1.5], "rotationY": 33.0,
                        "bounds_hex": np.array([getattr(b2, f) for f, _ in RefBounds._fields_],
                                               "<f4").tobytes().hex(),
                        "triangles_hex": tris2.astype("<f4").tobytes().hex()},
        }
    rng = np.random.default_rng(7)
    for n, substeps, period, L, U in [(11, 1, 8.0, 24.0, 0.05), (12, 1, 5.0, 24.0, 0.05),
                                      (100, 10, 9.0, 24.5, 0.05), (257, 4, 13.5, 40.0, 0.05),
                                      (64, 20, 3.0, 12.0, 0.08), (150, 1, 1e9, 24.0, 0.0)]:
        t = np.arange(n, dtype=np.float64)
        cl = 0.3 * np.sin(2 * np.pi * t / period) + 0.05 * rng.standard_normal(n) + 0.1
        cl = cl.astype(np.float32)
        line = strouhal_ref(lib, cl, substeps, L, U)
        golden["strouhal"].append({"cl_hex": cl.astype("<f4").tobytes().hex(),
                                   "substeps": substeps, "L": L, "U": U, "printed": line})
    with open(OUT, "w") as fh:
        json.dump(golden, fh, indent=1)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
