"""The batched-sweep instance generator (host only)."""
from __future__ import annotations

from collections import Counter

import numpy as np

from lattice_fluid_dynamics_b200 import geometry


def _closed(tris: np.ndarray) -> bool:
    """Every edge of a closed triangle mesh is shared by exactly two faces."""
    edges = Counter()
    v = tris.reshape(-1, 3, 4)[:, :, :3]
    for t in v:
        for a, b in ((0, 1), (1, 2), (2, 0)):
            e = tuple(sorted((tuple(t[a]), tuple(t[b]))))
            edges[e] += 1
    return all(c == 2 for c in edges.values())


def test_sweep_instances_deterministic_and_in_range():
    a = geometry.sweep_instances(1, 64)
    b = geometry.sweep_instances(1, 64)
    assert len(a) == 64
    for x, y in zip(a, b):
        assert x["dims"] == y["dims"] and np.array_equal(x["triangles"], y["triangles"])
    for i in a:
        nx, ny, nz = i["dims"]
        assert 64 <= nx <= 192 and 64 <= ny <= 96 and 64 <= nz <= 96
        assert nx % 8 == ny % 8 == nz % 8 == 0
        assert 0.02 <= i["U"] <= 0.10 and 100 <= i["Re"] <= 2000
        assert all(6 <= ax <= 20 for ax in i["axes"])
        assert i["op"] in ("bgk", "reg") and i["kind"] in ("sphere", "ellipsoid", "slanted_box")
        lo = np.array(i["bbox"][:3])
        hi = np.array(i["bbox"][3:])
        assert np.all(lo > [-4, -2, -2]) and np.all(hi < [4, 2, 2])
    kinds = Counter(i["kind"] for i in a)
    assert len(kinds) == 3
    assert geometry.sweep_instances(2, 4)[0]["dims"] != a[0]["dims"] or \
        not np.array_equal(geometry.sweep_instances(2, 4)[0]["triangles"], a[0]["triangles"])


def test_sweep_meshes_closed():
    for i in geometry.sweep_instances(1, 12):
        assert _closed(i["triangles"]), i["kind"]


def test_warmstart_shapes_closed_disjoint_deterministic():
    from lattice_fluid_dynamics_b200 import warmstart as ws
    for i in range(24):
        a = ws.random_union(2, i)
        b = ws.random_union(2, i)
        assert np.array_equal(a["triangles"], b["triangles"]) and a["U"] == b["U"]
        assert _closed(a["triangles"])
        lo, hi = np.array(a["bbox"][:3]), np.array(a["bbox"][3:])
        assert np.all(lo > [-4, -2, -2]) and np.all(hi < [0, 2, 2])
        assert 0.04 <= a["U"] <= 0.08 and 20 <= a["Re"] <= 100
    assert not np.array_equal(ws.random_union(2, 0)["triangles"],
                              ws.random_union(2, 100000)["triangles"])


def test_warmstart_entry_and_summaries():
    from lattice_fluid_dynamics_b200 import warmstart as W
    # trailing mean and the first sample after which it stays in the band
    avg = W.smoothed([1.0, 1.0, 2.0, 2.0, 2.0], 2)
    assert np.allclose(avg, [1.0, 1.0, 1.5, 2.0, 2.0])
    assert W.entry_index(avg, 2.0) == 3
    assert W.entry_index(avg, 2.0, band=0.3) == 2
    assert W.entry_index([1.0, 1.0, 3.0], 1.0) is None   # leaves the band at the end
    assert W.entry_index([1.0, 1.0], 1.0) == 0
    rows = [
        {"cold_fp32": {"steps": 4000, "wall_s": 0.4}, "cold_fp16_ref": {"steps": 3000, "wall_s": 0.3},
         "warmc_fp16": {"steps": None, "wall_s": None, "steps16": 1000, "wall_s16": 0.1}},
        {"cold_fp32": {"steps": 9000, "wall_s": 0.9}, "cold_fp16_ref": {"steps": 8000, "wall_s": 0.8},
         "warmc_fp16": {"steps": 2000, "wall_s": 0.2, "steps16": 2000, "wall_s16": 0.2}},
    ]
    s32 = W.summarize(rows, "warmc_fp16")
    assert s32["both_converged"] == 1 and s32["wall_ratio_total"] == 0.2 / 0.9
    s16 = W.summarize_fp16(rows, "warmc_fp16")
    assert s16["both_converged"] == 2
    assert abs(s16["wall_ratio_total"] - 0.3 / 1.1) < 1e-12
    assert s16["steps_ratio_total"] == 3000 / 11000
    assert s16["faster_fraction"] == 1.0
