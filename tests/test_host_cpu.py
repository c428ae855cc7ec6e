"""Host-side driver pieces of the C ABI against the reference's own C code.

The fixtures in tests/golden/host_golden.json were produced by the
reference's loadOBJ, computeModelBounds, createTriangleBuffer
(simulation/obj-file-loader/lib/model_loader.c, simulation/src/model_bounds.c)
and compute_strouhal (simulation/src/drag_metrics.c), compiled from their
sources by ``make -C oracle ref REFSIM=<reference>/simulation``; tests/golden/make_golden.py regenerates
them.  Comparisons are bit-exact (float bytes, printed strings).  When
oracle/_ref/libref_host.so is present the live reference is also run on
freshly generated meshes.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np
import pytest

import lattice_fluid_dynamics_b200 as lfd
from lattice_fluid_dynamics_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
with open(os.path.join(GOLDEN, "host_golden.json")) as _fh:
    G = json.load(_fh)


def _f32(hexstr: str) -> np.ndarray:
    return np.frombuffer(bytes.fromhex(hexstr), "<f4")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    lfd.load()


@pytest.mark.parametrize("name", sorted(G["obj"]))
def test_load_obj_matches_reference(name):
    ref = G["obj"][name]
    m = capi.Model(os.path.join(GOLDEN, "obj", name + ".obj"))
    assert m.vertex_count == ref["vertexCount"]
    assert m.face_count == ref["faceCount"]
    assert m.vertices().astype("<f4").tobytes() == bytes.fromhex(ref["vertices_hex"])
    assert m.faces().tolist() == ref["faces"]


@pytest.mark.parametrize("name", sorted(G["obj"]))
def test_placement_bounds_triangles_match_reference(name):
    ref = G["obj"][name]
    m = capi.Model(os.path.join(GOLDEN, "obj", name + ".obj"))
    s, off, rot = m.place()
    p = ref["placement"]
    assert np.float32(s) == np.float32(p["scale"])
    assert np.array_equal(np.float32(off), np.float32(p["offset"]))
    assert rot == p["rotationY"]
    assert m.bounds(s, off, rot).tobytes() == _f32(ref["bounds_hex"]).tobytes()
    tris = m.triangles(s, off, rot)
    assert tris.shape[0] == ref["triangleCount"]
    assert tris.tobytes() == _f32(ref["triangles_hex"]).tobytes()
    gen = ref["general"]
    t2 = m.triangles(gen["scale"], gen["offset"], gen["rotationY"])
    assert t2.tobytes() == _f32(gen["triangles_hex"]).tobytes()
    b2 = m.bounds(gen["scale"], gen["offset"], gen["rotationY"])
    assert b2.tobytes() == _f32(gen["bounds_hex"]).tobytes()


def test_quads_truncated_and_bad_faces_skipped():
    m = capi.Model(os.path.join(GOLDEN, "obj", "cube_quads.obj"))
    faces = m.faces()
    # "f 1 2 3 4 5 6" keeps 1 2 3; the tab-separated face line is not a face
    assert [1, 2, 3] in faces.tolist()
    tris = m.triangles(1.0, (0.0, 0.0, 0.0), 0.0)
    bad = sum(1 for f in faces if min(f) < 1 or max(f) > m.vertex_count)
    assert tris.shape[0] == m.face_count - bad == 7


def test_missing_file_raises(tmp_path):
    with pytest.raises(OSError):
        capi.Model(str(tmp_path / "nope.obj"))


def test_empty_model(tmp_path):
    p = tmp_path / "empty.obj"
    p.write_text("# nothing\n")
    m = capi.Model(str(p))
    assert m.vertex_count == 0 and m.face_count == 0
    assert m.triangles(1.0, (0, 0, 0), 0.0).shape == (0, 12)
    # computeModelBounds' default box (model_bounds.c:154-160)
    assert m.bounds(1.0, (0, 0, 0), 0.0).tolist() == [-0.5] * 3 + [0.5] * 3 + [0.0] * 3
    with pytest.raises(ValueError):
        m.place()


@pytest.mark.parametrize("case", range(len(G["strouhal"])))
def test_strouhal_matches_reference(case):
    ref = G["strouhal"][case]
    cl = _f32(ref["cl_hex"])
    st, f = capi.strouhal(cl, ref["substeps"], ref["L"], ref["U"])
    if len(cl) < 12:
        assert ref["printed"] == "" and st == 0.0 and f == 0.0
        return
    line = "St=%.4f (f=%.6f, L=%.1f, U=%.3f)" % (st, f, np.float32(ref["L"]),
                                                 np.float32(ref["U"]))
    assert line == ref["printed"]


def test_strouhal_finds_shedding_frequency():
    # a pure tone on an exact DFT bin is found exactly
    n_total, substeps, interval = 400, 2, 20
    start = n_total * 35 // 100
    n = n_total - start
    k = 13
    t = np.arange(n_total)
    cl = np.sin(2 * np.pi * k * (t - start) / n).astype(np.float32)
    st, f = capi.strouhal(cl, substeps, 30.0, 0.05, interval)
    fs = 1.0 / (interval * substeps)
    assert f == pytest.approx(k * fs / n, rel=1e-6)
    assert st == pytest.approx(f * 30.0 / 0.05, rel=1e-6)


@pytest.mark.parametrize("U,L,Re", [(0.05, 24.0, 200.0), (0.05, 24.0, 10000.0),
                                    (0.05, 60.0, 50.0), (0.08, 33.3, 1234.5)])
def test_reynolds_to_tau(U, L, Re):
    tau, nu, re, clamped = capi.reynolds_to_tau(U, L, Re)
    f32 = np.float32
    nu_ref = f32(f32(U) * f32(L)) / f32(Re)
    tau_ref = f32(f32(3.0) * nu_ref) + f32(0.5)
    if tau_ref < f32(0.52):
        assert clamped
        nu_ref = f32(f32(f32(0.52) - f32(0.5)) / f32(3.0))
        assert tau == f32(0.52) and nu == nu_ref
        assert re == f32(f32(f32(U) * f32(L)) / nu_ref)
    else:
        assert not clamped and tau == tau_ref and nu == nu_ref and re == f32(Re)


REF_LIB = os.path.join(HERE, "..", "oracle", "_ref", "libref_host.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference host library not built")
def test_live_reference_random_meshes(tmp_path):
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden as mg

    lib = mg.load_ref()
    rng = np.random.default_rng(11)
    for trial in range(4):
        radii = tuple(rng.uniform(0.3, 5.0, 3))
        center = tuple(rng.uniform(-10, 10, 3))
        path = tmp_path / f"m{trial}.obj"
        path.write_text(mg.obj_ellipsoid(int(rng.integers(3, 12)), int(rng.integers(3, 12)),
                                         radii, center, trial))
        rm = lib.loadOBJ(str(path).encode())
        m = capi.Model(str(path))
        rv = np.ctypeslib.as_array(rm.vertices, (rm.vertexCount, 3))
        assert np.array_equal(rv, m.vertices())
        s, off, rot = m.place()
        ps, poff, prot = mg.place(m.vertices())
        assert (s, list(off), rot) == (ps, poff, prot)
        ang = float(rng.uniform(0, 360))
        cnt = C.c_int()
        tp = lib.createTriangleBuffer(C.byref(rm), s, *off, ang, C.byref(cnt))
        rt = np.ctypeslib.as_array(tp, (cnt.value, 12)).copy()
        C.CDLL(None).free(C.cast(tp, C.c_void_p))
        assert np.array_equal(rt, m.triangles(s, off, ang))
        lib.freeModel(C.byref(rm))
