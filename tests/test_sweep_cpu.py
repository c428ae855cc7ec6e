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


def test_sweep_shards_partition_and_balance():
    from lattice_fluid_dynamics_b200 import sweep
    dims = [i["dims"] for i in geometry.sweep_instances(1, 64)]
    for world in (1, 2, 3, 4, 8):
        parts = [sweep.shard(dims, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))                      # every instance exactly once
        loads = [sum(int(np.prod(dims[k])) for k in p) for p in parts]
        assert max(loads) <= 1.05 * min(loads)              # near-equal lattice updates
        assert parts == [sweep.shard(dims, world, r) for r in range(world)]  # deterministic


def _fake_rank_result(rank, idx, ms):
    return {"instances": len(idx), "steps": 100, "seed": 1, "storage": "fp32",
            "cells_total": 1000 * len(idx), "ms": ms, "mlups": 0.0,
            "gb_per_s": 10.0 * (rank + 1), "schedule": "graph", "cd_identical": len(idx),
            "per_instance": [{"index": k, "cd": 0.1 * k} for k in idx]}


def test_sweep_merge_ranks():
    from lattice_fluid_dynamics_b200 import sweep
    parts = [[0, 3], [1, 2, 4]]
    res = sweep.merge_ranks([_fake_rank_result(r, p, 50.0 + 10 * r) for r, p in enumerate(parts)])
    assert res["instances"] == 5 and res["ranks"] == 2 and res["ms"] == 60.0
    assert [p["index"] for p in res["per_instance"]] == [0, 1, 2, 3, 4]
    assert res["mlups"] == 5000 * 100 / 0.060 / 1e6
    assert res["cd_identical"] == 5


def _gather_rank(rank, world, port, out):
    import os
    import torch.distributed as dist
    from lattice_fluid_dynamics_b200 import sweep
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dims = [i["dims"] for i in geometry.sweep_instances(1, 64)]
        mine = sweep.shard(dims, world, rank)
        got = [None] * world
        dist.all_gather_object(got, _fake_rank_result(rank, mine, 40.0 + rank))
        if rank == 0:
            res = sweep.merge_ranks(got)
            out.put((res["instances"], [p["index"] for p in res["per_instance"]], res["ms"]))
    finally:
        dist.destroy_process_group()


def test_sweep_two_gloo_ranks_gather():
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    n, order, ms = q.get(timeout=240)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert n == 64 and order == list(range(64)) and ms == 41.0
