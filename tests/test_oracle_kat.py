"""Pins of the CPU oracle against the reference's own tests.

simulation/test/test_lbm.c holds the only known-answer tests of the path:
the pure-math tests (:191-232 weights and equilibrium, :303-366 MRT
transforms) and the GL solver tests whose assertions are physical bounds
(:234-301, :368-592).  The GL tests cannot run here (no graphics stack), so
their scenarios are replayed on the oracle with the same assertions.
"""
import numpy as np
import pytest

from tests import scenarios as S

EX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0]
EY = [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1]
EZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1]


# ---------------- test_lbm.c:191-232 ----------------
def test_weights_sum_to_one(oracle):
    s = np.float32(0)
    for i in range(19):
        s = np.float32(s + np.float32(oracle.weight32(i)))
    assert abs(float(s) - 1.0) <= 1e-6


def test_equilibrium_conserves_density(oracle):
    rho, u = 1.5, (0.05, 0.01, -0.02)
    s = sum(oracle.feq32(i, rho, *u) for i in range(19))
    assert abs(s - rho) <= 1e-5


def test_equilibrium_conserves_momentum(oracle):
    rho, u = 1.2, (0.08, -0.03, 0.04)
    m = np.zeros(3)
    for i in range(19):
        fi = oracle.feq32(i, rho, *u)
        m += fi * np.array([EX[i], EY[i], EZ[i]])
    np.testing.assert_allclose(m, rho * np.array(u), atol=1e-5)


def test_equilibrium_at_rest(oracle):
    for i in range(19):
        assert abs(oracle.feq32(i, 1.0, 0, 0, 0) - oracle.weight32(i)) <= 1e-6


def test_fp64_equilibrium_consistent(oracle):
    for i in range(19):
        assert abs(oracle.feq64(i, 1.1, 0.04, 0.01, -0.02)
                   - oracle.feq32(i, 1.1, 0.04, 0.01, -0.02)) < 1e-7


# ---------------- test_lbm.c:303-366 ----------------
def _feq_vec(oracle, rho, u):
    return np.array([oracle.feq32(i, rho, *u) for i in range(19)], np.float32)


def test_mrt_moment_roundtrip(oracle):
    fi = _feq_vec(oracle, 1.3, (0.06, -0.02, 0.03))
    back = oracle.mrt_inverse(oracle.mrt_forward(fi))
    np.testing.assert_allclose(back, fi, atol=1e-5)


def test_mrt_conserved_moments(oracle):
    rho, u = 1.4, (0.05, -0.01, 0.02)
    m = oracle.mrt_forward(_feq_vec(oracle, rho, u))
    assert abs(m[0] - rho) <= 1e-5
    assert abs(m[3] - rho * u[0]) <= 1e-5
    assert abs(m[5] - rho * u[1]) <= 1e-5
    assert abs(m[7] - rho * u[2]) <= 1e-5


def test_mrt_equilibrium_fixedpoint(oracle):
    rho, u = 1.1, (0.04, 0.01, -0.02)
    m = oracle.mrt_forward(_feq_vec(oracle, rho, u))
    meq = oracle.mrt_meq(rho, *u)
    np.testing.assert_allclose(m, meq, atol=1e-4)


# ---------------- test_lbm.c:234-301 ----------------
def test_grid_create_tau(oracle):
    g = oracle.OracleGrid(16, 8, 8, 0.1)
    assert abs(g.tau - (0.5 + 3 * 0.1)) <= 1e-4
    lo = oracle.OracleGrid(8, 4, 4, 0.0)
    hi = oracle.OracleGrid(8, 4, 4, 1.0)
    assert lo.tau == np.float32(0.52) and hi.tau == 2.0      # lbm.c:56-60


def test_solid_aabb_marks_cells(oracle):
    g = oracle.OracleGrid(16, 8, 8, 0.1)
    g.set_solid_aabb(-0.5, -0.25, -0.25, 0.5, 0.25, 0.25)
    c = int((g.solid != 0).sum())
    assert 0 < c < g.n


def test_aabb_index_math_independent(oracle):
    """lbm.c:353-394 recomputed independently in numpy float32."""
    nx, ny, nz = 32, 16, 16
    b = (-0.7, -0.33, -0.41, 0.55, 0.29, 0.12)
    g = oracle.OracleGrid(nx, ny, nz, 0.1)
    g.set_solid_aabb(*b)
    f = np.float32
    sx, sy, sz = f(nx) / f(8), f(ny) / f(4), f(nz) / f(4)
    lo = [int((f(b[0]) + f(4)) * sx), int((f(b[1]) + f(2)) * sy), int((f(b[2]) + f(2)) * sz)]
    hi = [int((f(b[3]) + f(4)) * sx), int((f(b[4]) + f(2)) * sy), int((f(b[5]) + f(2)) * sz)]
    ref = np.zeros((nz, ny, nx), np.int32)
    ref[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = 1
    np.testing.assert_array_equal(g.solid, ref.reshape(-1))
    # every q >= 0 entry is a fluid->solid link with q = 0.5, and vice versa
    s = ref
    q = g.q.reshape(nz, ny, nx, 19)
    for i in range(1, 19):
        nb = np.zeros_like(s)
        zs, ys, xs = np.meshgrid(range(nz), range(ny), range(nx), indexing="ij")
        mx, my, mz = xs + EX[i], ys + EY[i], zs + EZ[i]
        inb = (mx >= 0) & (mx < nx) & (my >= 0) & (my < ny) & (mz >= 0) & (mz < nz)
        nb[inb] = s[mz[inb], my[inb], mx[inb]]
        expect = (s != 1) & (nb == 1)
        np.testing.assert_array_equal(q[..., i] >= 0, expect)
        assert np.all(q[..., i][expect] == np.float32(0.5))


def test_sphere_q_against_float64_geometry(oracle):
    """Analytic ray-sphere q (lbm.c:502-524) agrees with a float64
    evaluation of the same geometry to float32 accuracy."""
    nx, ny, nz = 64, 32, 32
    cx, cy, cz, r = -1.3, 0.07, -0.11, 0.5
    g = oracle.OracleGrid(nx, ny, nz, 0.1)
    g.set_solid_sphere(cx, cy, cz, r)
    sc = np.array([nx / 8, ny / 4, nz / 4])
    cell, d, q = g.links()
    x = cell % nx
    y = (cell // nx) % ny
    z = cell // (nx * ny)
    w = (np.stack([x, y, z], 1) + 0.5) / sc - np.array([4, 2, 2])
    e = np.stack([np.array(EX)[d], np.array(EY)[d], np.array(EZ)[d]], 1) / sc
    o = w - np.array([cx, cy, cz])
    a = (e * e).sum(1)
    b = 2 * (o * e).sum(1)
    c = (o * o).sum(1) - r * r
    disc = b * b - 4 * a * c
    t = np.where(disc >= 0, (-b - np.sqrt(np.maximum(disc, 0))) / (2 * a), 0.5)
    t = np.where((t > 0) & (t <= 1), t, 0.5)
    t = np.clip(t, 0.01, 0.99)
    assert len(q) > 100
    assert np.max(np.abs(q - t)) < 5e-4


def test_flow_init_and_step_nonzero_drag(oracle):
    """test_lbm.c:271-301"""
    g = oracle.OracleGrid(16, 8, 8, 0.1)
    g.set_solid_aabb(-0.3, -0.15, -0.15, 0.3, 0.15, 0.15)
    g.initialize_flow(0.05)
    g.step(0.05, n=10)
    assert abs(g.drag_force_decomposed()[0]) > 1e-10
    g.step(0.05, n=990)
    assert abs(g.drag_force_decomposed()[0]) > 1e-10
    cd = g.drag_coefficient(0.05, 4.0)
    assert 0 < cd < 1000


def test_mrt_and_smagorinsky_steps(oracle):
    """test_lbm.c:368-401"""
    g = oracle.OracleGrid(16, 8, 8, 0.1)
    g.set(useMRT=1)
    g.set_solid_aabb(-0.3, -0.15, -0.15, 0.3, 0.15, 0.15)
    g.initialize_flow(0.05)
    g.step(0.05, n=10)
    assert abs(g.drag_force_decomposed()[0]) > 1e-10
    h = oracle.OracleGrid(16, 8, 8, 0.01)
    h.set(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1)
    h.set_solid_aabb(-0.3, -0.15, -0.15, 0.3, 0.15, 0.15)
    h.initialize_flow(0.05)
    h.step(0.05, n=20)
    assert np.isfinite(h.f).all()


def test_ground_plane_counts_and_drag(oracle):
    """test_lbm.c:549-592"""
    g = oracle.OracleGrid(32, 16, 16, 0.1)
    g.set_solid_aabb(-0.3, -0.15, -0.15, 0.3, 0.15, 0.15)
    g.add_ground_plane(-0.15)
    s = g.solid
    assert (s == 1).sum() > 0 and (s == 2).sum() > 0 and (s == 0).sum() > 0
    g.initialize_flow(0.05)
    g.step(0.05, n=20)
    assert abs(g.drag_force_decomposed()[0]) > 1e-10


def test_box_cd_convergence(oracle):
    """test_lbm.c:458-547 (128x64x64, Re = 50, MRT + Smagorinsky): five Cd
    samples 100 steps apart after 2500 steps, all positive, max/min < 10."""
    oracle.set_threads(0)
    U = 0.05
    g = oracle.OracleGrid(128, 64, 64, (U * 16.0) / 50.0)
    g.set(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1)
    g.set_solid_aabb(-0.3, -0.15, -0.15, 0.3, 0.15, 0.15)
    A = g.projected_area(0)
    g.initialize_flow(U)
    g.step(U, n=2500)
    dynP = 0.5 * U * U
    cds = []
    for _ in range(5):
        g.step(U, n=100)
        cds.append(abs(g.drag_force_decomposed()[0]) / (dynP * A))
    assert min(cds) > 0
    assert max(cds) / max(min(cds), 0.001) < 10


def test_sphere_cd_re100(oracle):
    """test_lbm.c:403-456: 128x64x64 sphere D = 1 (16 cells), Re = 100,
    4000 steps, 0.5 < Cd < 3.5."""
    U = 0.05
    visc = (U * 16.0) / 100.0
    g = oracle.OracleGrid(128, 64, 64, visc)
    g.set_solid_sphere(0.0, 0.0, 0.0, 0.5)
    A = g.projected_area(0)
    g.initialize_flow(U)
    g.step(U, n=4000)
    cd = g.drag_coefficient(U, A)
    print(f"oracle sphere Cd(Re=100) = {cd:.3f}")
    assert 0.5 < cd < 3.5


# ---------------- particles and export ----------------
def test_particle_seed_in_inlet_plane(oracle):
    p = oracle.particles_seed_inlet(50000, 0)
    assert np.all(p[:, 0] == -4.0)
    assert p[:, 1].min() >= -2 and p[:, 1].max() < 2
    assert abs(p[:, 1].mean()) < 0.02 and abs(p[:, 2].mean()) < 0.02
    assert np.all(p[:, 7] == 1.0)


def test_particle_uniform_flow(oracle):
    """Trilinear sampling of a uniform field returns it exactly: the
    particle velocity relaxes toward 2 u (particle_lbm.comp:219-226)."""
    nx, ny, nz = 16, 8, 8
    vel = np.zeros((nx * ny * nz, 4), np.float32)
    vel[:, 0] = 0.05
    vel[:, 3] = 1.0
    p = oracle.particles_seed_inlet(100, 3)
    for _ in range(2000):
        oracle.particles_step(vel, (nx, ny, nz), p, 0.016, 3)
    np.testing.assert_allclose(p[:, 4], 0.1, rtol=1e-4)


def test_vti_layout(oracle, tmp_path):
    nx, ny, nz = 4, 3, 2
    vel = np.arange(4 * nx * ny * nz, dtype=np.float32).reshape(-1, 4)
    solid = (np.arange(nx * ny * nz) % 3).astype(np.int32)
    path = str(tmp_path / "a.vti")
    assert oracle.write_vti(path, (nx, ny, nz), vel, solid)
    raw = open(path, "rb").read()
    marker = b'<AppendedData encoding="raw">\n_'
    blob = raw[raw.index(marker) + len(marker):]
    n = nx * ny * nz
    assert int(np.frombuffer(blob[:8], "<u8")[0]) == 12 * n
    v = np.frombuffer(blob[8:8 + 12 * n], "<f4").reshape(n, 3)
    np.testing.assert_array_equal(v, vel[:, :3])
    off = 8 + 12 * n
    assert int(np.frombuffer(blob[off:off + 8], "<u8")[0]) == 4 * n
    np.testing.assert_array_equal(np.frombuffer(blob[off + 8:off + 8 + 4 * n], "<f4"), vel[:, 3])
    assert b'WholeExtent="0 4 0 3 0 2"' in raw
