"""Deterministic geometry for the solver's workloads.

``ahmed_body`` builds the triangle buffer that ``LBM_SetSolidMesh``
consumes (12 floats per triangle, the GPUTriangle layout of
simulation/lib/model_bounds.h:14-18) for an Ahmed-style bluff body: a
1.044 x 0.389 x 0.288 box whose four front edges are rounded (radius
0.100) and whose rear top carries a 25 degree slant (0.222 long along the
slant).  The body is convex, so its surface is the radial graph
r(theta, phi) around the centroid; the mesher samples that graph on a
(theta, phi) lattice by bisection and triangulates it into a closed mesh
(2 * n_phi * (n_theta - 1) triangles; the defaults give 19,800).  The
body is placed like simulation/src/main.c:289-349 places a model: scaled
to the requested length and centred at world (-2, 0, 0).

``sweep_shapes`` draws the uneven-size batched sweep of spheres,
ellipsoids and slanted boxes from a seed.
"""
from __future__ import annotations

import math

import numpy as np

AHMED_L, AHMED_W, AHMED_H = 1.044, 0.389, 0.288
AHMED_R = 0.100
AHMED_SLANT_LEN = 0.222


def _ahmed_inside(p: np.ndarray, slant_deg: float) -> np.ndarray:
    """Inside test in body coordinates: x in [0, L] (front at 0), |y| <= W/2,
    z in [0, H]."""
    L, W, H, r = AHMED_L, AHMED_W, AHMED_H, AHMED_R
    x, y, z = p[..., 0], p[..., 1], p[..., 2]
    box = (x >= r) & (x <= L) & (np.abs(y) <= W / 2) & (z >= 0) & (z <= H)
    dy = np.maximum(np.abs(y) - (W / 2 - r), 0.0)
    dz = np.maximum(np.maximum(r - z, z - (H - r)), 0.0)
    cap = (x >= 0) & (x < r) & ((r - x) ** 2 + dy ** 2 + dz ** 2 <= r * r)
    t = math.tan(math.radians(slant_deg))
    xs = L - AHMED_SLANT_LEN * math.cos(math.radians(slant_deg))
    slant_ok = z <= H - np.maximum(x - xs, 0.0) * t
    return (box | cap) & slant_ok


def ahmed_body(length: float = 2.0, center=(-2.0, 0.0, 0.0), n_theta: int = 100,
               n_phi: int = 100, slant_deg: float = 25.0):
    """Return (triangles float32 [n, 12], bbox (minX, minY, minZ, maxX, maxY,
    maxZ)) of the Ahmed-style body scaled to `length` world units along x
    and centred (bounding-box centre) at `center`."""
    c0 = np.array([AHMED_L * 0.45, 0.0, AHMED_H * 0.45])  # interior point
    th = np.linspace(0.0, math.pi, n_theta + 1)            # from -x (front) to +x
    ph = np.linspace(0.0, 2 * math.pi, n_phi, endpoint=False)
    T, P = np.meshgrid(th[1:-1], ph, indexing="ij")
    dirs = np.stack([-np.cos(T), np.sin(T) * np.cos(P), np.sin(T) * np.sin(P)], -1)
    dirs = np.concatenate([dirs.reshape(-1, 3), [[-1.0, 0, 0]], [[1.0, 0, 0]]])
    lo = np.zeros(len(dirs))
    hi = np.full(len(dirs), 2.0)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        ins = _ahmed_inside(c0 + dirs * mid[:, None], slant_deg)
        lo = np.where(ins, mid, lo)
        hi = np.where(ins, hi, mid)
    verts = c0 + dirs * lo[:, None]
    nr = n_theta - 1
    front, rear = nr * n_phi, nr * n_phi + 1

    def vid(i, j):
        return i * n_phi + (j % n_phi)

    tris = []
    for j in range(n_phi):
        tris.append((front, vid(0, j + 1), vid(0, j)))
        tris.append((rear, vid(nr - 1, j), vid(nr - 1, j + 1)))
    for i in range(nr - 1):
        for j in range(n_phi):
            a, b = vid(i, j), vid(i, j + 1)
            c, d = vid(i + 1, j), vid(i + 1, j + 1)
            tris.append((a, b, d))
            tris.append((a, d, c))
    tri = np.asarray(tris, np.int64)
    # scale and place (bounding-box centre at `center`)
    s = length / AHMED_L
    v = verts * s
    bmin, bmax = v.min(0), v.max(0)
    v = v - 0.5 * (bmin + bmax) + np.asarray(center)
    v = v.astype(np.float32)
    out = np.zeros((len(tri), 12), np.float32)
    out[:, 0:3] = v[tri[:, 0]]
    out[:, 4:7] = v[tri[:, 1]]
    out[:, 8:11] = v[tri[:, 2]]
    bb = v.min(0), v.max(0)
    bbox = (float(bb[0][0]), float(bb[0][1]), float(bb[0][2]),
            float(bb[1][0]), float(bb[1][1]), float(bb[1][2]))
    return out, bbox


def uv_sphere(radius: float, center=(0.0, 0.0, 0.0), n_theta: int = 32, n_phi: int = 32):
    """Closed UV sphere as a triangle buffer (12 floats per triangle)."""
    th = np.linspace(0.0, math.pi, n_theta + 1)[1:-1]
    ph = np.linspace(0.0, 2 * math.pi, n_phi, endpoint=False)
    T, P = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.cos(T), np.sin(T) * np.cos(P), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    d = np.concatenate([d, [[1.0, 0, 0]], [[-1.0, 0, 0]]])
    v = (np.asarray(center) + radius * d).astype(np.float32)
    nr = n_theta - 1
    p0, p1 = nr * n_phi, nr * n_phi + 1
    tris = []
    for j in range(n_phi):
        jn = (j + 1) % n_phi
        tris.append((p0, jn, j))
        tris.append((p1, (nr - 1) * n_phi + j, (nr - 1) * n_phi + jn))
    for i in range(nr - 1):
        for j in range(n_phi):
            jn = (j + 1) % n_phi
            a, b, c, e = i * n_phi + j, i * n_phi + jn, (i + 1) * n_phi + j, (i + 1) * n_phi + jn
            tris.append((a, b, e))
            tris.append((a, e, c))
    tri = np.asarray(tris)
    out = np.zeros((len(tri), 12), np.float32)
    out[:, 0:3] = v[tri[:, 0]]
    out[:, 4:7] = v[tri[:, 1]]
    out[:, 8:11] = v[tri[:, 2]]
    lo, hi = v.min(0), v.max(0)
    return out, (float(lo[0]), float(lo[1]), float(lo[2]), float(hi[0]), float(hi[1]),
                 float(hi[2]))


def reynolds_tau(U: float, length_cells: float, Re: float) -> float:
    """tau = 3 nu + 1/2 with nu = U L / Re (simulation/src/main.c:447-448)."""
    return 3.0 * (U * length_cells / Re) + 0.5


def write_obj(tris: np.ndarray, path: str) -> None:
    """Write a triangle buffer (12 floats per triangle) as a Wavefront OBJ,
    three vertices per face, printed with enough digits that every float32
    coordinate reads back exactly."""
    t = np.asarray(tris, np.float32).reshape(-1, 12)
    with open(path, "w") as fh:
        for row in t:
            for k in range(3):
                x, y, z = (float(v) for v in row[4 * k:4 * k + 3])
                fh.write(f"v {x:.9g} {y:.9g} {z:.9g}\n")
        for i in range(len(t)):
            fh.write(f"f {3 * i + 1} {3 * i + 2} {3 * i + 3}\n")
