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

``sweep_instances`` draws the uneven-size batched sweep of spheres,
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


def _cells_to_world(v: np.ndarray, dims) -> np.ndarray:
    """Cell coordinates -> the reference's world coordinates: x = c / (NX/8) - 4,
    y = c / (NY/4) - 2, z = c / (NZ/4) - 2 (simulation/src/lbm.c:353-362)."""
    nx, ny, nz = dims
    s = np.array([nx / 8.0, ny / 4.0, nz / 4.0])
    return v / s - np.array([4.0, 2.0, 2.0])


def _tris_from(verts: np.ndarray, faces) -> np.ndarray:
    f = np.asarray(faces, np.int64)
    out = np.zeros((len(f), 12), np.float32)
    v = verts.astype(np.float32)
    out[:, 0:3] = v[f[:, 0]]
    out[:, 4:7] = v[f[:, 1]]
    out[:, 8:11] = v[f[:, 2]]
    return out


def ellipsoid_cells(center, axes, n_theta: int = 24, n_phi: int = 24):
    """Closed ellipsoid mesh in cell coordinates; `axes` are full lengths."""
    th = np.linspace(0.0, math.pi, n_theta + 1)[1:-1]
    ph = np.linspace(0.0, 2 * math.pi, n_phi, endpoint=False)
    T, P = np.meshgrid(th, ph, indexing="ij")
    d = np.stack([np.cos(T), np.sin(T) * np.cos(P), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    d = np.concatenate([d, [[1.0, 0, 0]], [[-1.0, 0, 0]]])
    v = np.asarray(center) + 0.5 * np.asarray(axes) * d
    nr = n_theta - 1
    p0, p1 = nr * n_phi, nr * n_phi + 1
    faces = []
    for j in range(n_phi):
        jn = (j + 1) % n_phi
        faces.append((p0, jn, j))
        faces.append((p1, (nr - 1) * n_phi + j, (nr - 1) * n_phi + jn))
    for i in range(nr - 1):
        for j in range(n_phi):
            jn = (j + 1) % n_phi
            a, b, c, e = i * n_phi + j, i * n_phi + jn, (i + 1) * n_phi + j, (i + 1) * n_phi + jn
            faces.append((a, b, e))
            faces.append((a, e, c))
    return v, faces


def slanted_box_cells(center, size, slant_deg: float):
    """Box of `size` (L, W, H) cells whose rear top edge is lowered by a slant
    of `slant_deg` over the rear half of its length; 12 triangles."""
    L, W, H = size
    cx, cy, cz = center
    x0, x1 = cx - L / 2, cx + L / 2
    y0, y1 = cy - W / 2, cy + W / 2
    z0, z1 = cz - H / 2, cz + H / 2
    drop = min(0.5 * L * math.tan(math.radians(slant_deg)), 0.8 * H)
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1 - drop], [x1, y1, z1 - drop], [x0, y1, z1]])
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (1, 2, 6, 5), (0, 4, 7, 3)]
    faces = []
    for a, b, c, d in quads:
        faces += [(a, b, c), (a, c, d)]
    return v, faces


def sweep_instances(seed: int = 1, count: int = 64):
    """The batched parameter sweep: `count` instances drawn from `seed`.

    Grid sizes uniform between 64^3 and 192x96x96 (multiples of 8); one body
    per grid -- a sphere, an ellipsoid (axes 6-20 cells) or a slanted box
    (sides 6-20 cells, slant 15-35 degrees) -- centred at 30 % of the length
    and mid-height; U ~ U[0.02, 0.10], Re ~ U[100, 2000] with the body length
    in cells as the length scale; BGK or regularized collision; periodic
    y/z.  Each instance is a dict with dims, kind, triangles (world
    coordinates) and bbox, U, Re, length, op ("bgk" | "reg")."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        nx = 64 + 8 * int(rng.integers(0, 17))
        ny = 64 + 8 * int(rng.integers(0, 5))
        nz = 64 + 8 * int(rng.integers(0, 5))
        kind = ("sphere", "ellipsoid", "slanted_box")[int(rng.integers(0, 3))]
        c = (0.3 * nx, 0.5 * ny, 0.5 * nz)
        if kind == "sphere":
            d = float(rng.uniform(6, 20))
            axes = (d, d, d)
            v, f = ellipsoid_cells(c, axes)
        elif kind == "ellipsoid":
            axes = tuple(float(a) for a in rng.uniform(6, 20, 3))
            v, f = ellipsoid_cells(c, axes)
        else:
            axes = tuple(float(a) for a in rng.uniform(6, 20, 3))
            v, f = slanted_box_cells(c, axes, float(rng.uniform(15, 35)))
        w = _cells_to_world(v, (nx, ny, nz))
        tris = _tris_from(w, f)
        lo, hi = w.min(0), w.max(0)
        bbox = tuple(float(x) for x in (*lo, *hi))
        U = float(rng.uniform(0.02, 0.10))
        Re = float(rng.uniform(100, 2000))
        op = "bgk" if rng.integers(0, 2) == 0 else "reg"
        out.append(dict(index=k, dims=(nx, ny, nz), kind=kind, axes=axes, triangles=tris,
                        bbox=bbox, U=U, Re=Re, length=float(axes[0]), op=op))
    return out
