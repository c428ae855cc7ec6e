"""Batched parameter sweep: many small wind-tunnel grids in one launch per step.

The reference runs one grid per process (simulation/src/main.c), so a sweep
over bodies and Reynolds numbers is a loop of separate runs, each too small
to fill a GPU.  Here the instances drawn by ``geometry.sweep_instances``
(64 grids from 64^3 to 192x96x96, spheres / ellipsoids / slanted boxes, BGK
or regularized, U and Re drawn per instance) are grouped in one LBMBatch:
every lattice step of all of them is a single kernel launch, replayed from a
CUDA graph, with a tile width chosen per grid by LBM_BatchAutotune.

``run_sweep`` reports the aggregate MLUPS, each instance's drag coefficient,
its chosen tile, and -- with ``solo=True`` -- the same instances stepped one
grid at a time (LBM_StepN), whose Cd must be identical.

    python -m lattice_fluid_dynamics_b200.sweep --count 64 --steps 3000

Under torchrun (one process per GPU) every rank takes its share of the
instances (``shard``: a near-equal number of lattice updates each), runs it
as its own batch with no collective on the data path, and rank 0 gathers the
per-instance results; the aggregate MLUPS counts every rank's updates over
the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

from . import capi, geometry


def build_grid(inst: dict, storage: str = "fp32", tau_clamp: bool = False) -> capi.Grid:
    """One instance through the reference's API: mesh body, periodic y/z,
    uniform inlet flow.  tau = 3 U L / Re + 1/2 is set directly, so the
    instance runs at the Reynolds number it was drawn with (the sweep's
    contract: tau set for Re in [100, 2000]); with tau_clamp the viscosity
    goes through the reference driver's rule instead, whose 0.52 tau floor
    (simulation/src/main.c:447-460) lowers the Re that runs."""
    nx, ny, nz = inst["dims"]
    _, nu, _, _ = capi.reynolds_to_tau(inst["U"], inst["length"], inst["Re"])
    g = capi.Grid(nx, ny, nz, nu, storage=storage)
    g.set(useRegularized=1 if inst["op"] == "reg" else 0, periodicYZ=1)
    if not tau_clamp:
        g.set(tau=geometry.reynolds_tau(inst["U"], inst["length"], inst["Re"]))
    g.set_solid_mesh(inst["triangles"], inst["bbox"])
    g.initialize_flow(inst["U"])
    return g


def drag_coefficient(g: capi.Grid, U: float, area: float) -> float:
    return float(g.drag_coefficient(U, area))


def _timed(stream_ptr: int, fn) -> float:
    """Milliseconds of fn() on the given CUDA stream, by CUDA events."""
    import torch
    stream = torch.cuda.ExternalStream(stream_ptr)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def shard(dims, world: int, rank: int) -> list:
    """Indices of the instances rank `rank` of `world` runs: largest grids
    first, each to the rank with the fewest cells so far (ties: lowest
    rank), so every rank gets a near-equal share of lattice updates."""
    load = [0] * world
    owner = [0] * len(dims)
    sizes = [int(np.prod(d)) for d in dims]
    for k in sorted(range(len(dims)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda j: (load[j], j))
        owner[k] = r
        load[r] += sizes[k]
    return [k for k in range(len(dims)) if owner[k] == rank]


def merge_ranks(results: list) -> dict:
    """One sweep result from the per-rank results of a sharded sweep: the
    instances in index order, updates of every rank over the slowest rank's
    time."""
    first = results[0]
    ms = max(r["ms"] for r in results)
    cells = sum(r["cells_total"] for r in results)
    total = cells * first["steps"]
    out = {k: first[k] for k in ("steps", "seed", "storage", "tau_clamp") if k in first}
    out.update({
        "instances": sum(r["instances"] for r in results), "ranks": len(results),
        "cells_total": cells, "ms": ms, "mlups": total / (ms * 1e-3) / 1e6,
        "gb_per_s": sum(r["gb_per_s"] * r["ms"] for r in results) / ms,
        "per_rank_ms": [r["ms"] for r in results],
        "schedule": [r["schedule"] for r in results],
        "per_instance": sorted((p for r in results for p in r["per_instance"]),
                               key=lambda p: p["index"]),
    })
    if all("cd_identical" in r for r in results):
        out["cd_identical"] = sum(r["cd_identical"] for r in results)
    return out


def run_sweep(count: int = 64, steps: int = 3000, seed: int = 1, autotune: bool = True,
              solo: bool = True, storage: str = "fp32", warmup: int = 0,
              indices=None, tau_clamp: bool = False, schedule: str | None = None) -> dict:
    """The sweep of `count` instances from `seed`, or of the subset
    `indices` of them (a rank's shard); per-instance results keep the
    instance's index in the full sweep."""
    insts = geometry.sweep_instances(seed, count)
    index = list(range(count)) if indices is None else list(indices)
    insts = [insts[k] for k in index]
    count = len(insts)
    t0 = time.perf_counter()
    grids = [build_grid(i, storage, tau_clamp) for i in insts]
    setup_s = time.perf_counter() - t0
    areas = [g.projected_area(0) for g in grids]
    cells = np.array([np.prod(i["dims"]) for i in insts], np.int64)
    inlets = np.array([[i["U"], 0.0, 0.0] for i in insts], np.float32)
    batch = capi.Batch(grids)
    t0 = time.perf_counter()
    if autotune:
        batch.autotune(10)
    if schedule is not None:  # after the autotuner's tile choice: time this schedule
        batch.set_schedule(schedule)
    tune_s = time.perf_counter() - t0
    if warmup:
        batch.run(warmup, inlets)
    ms = _timed(batch.stream, lambda: batch.run(steps, inlets))
    total = int(cells.sum()) * steps
    res = {
        "instances": count, "steps": steps, "seed": seed, "storage": storage,
        "tau_clamp": tau_clamp,
        "cells_total": int(cells.sum()), "ms": ms,
        "mlups": total / (ms * 1e-3) / 1e6,
        "gb_per_s": total * grids[0].bytes_per_update() / (ms * 1e-3) / 1e9,
        "tiles_per_step": batch.tiles_per_step, "schedule": batch.schedule,
        "setup_s": setup_s, "autotune_s": tune_s,
        "per_instance": [],
    }
    for k, (inst, g) in enumerate(zip(insts, grids)):
        res["per_instance"].append({
            "index": index[k], "dims": list(inst["dims"]), "kind": inst["kind"], "op": inst["op"],
            "U": inst["U"], "Re": inst["Re"], "tau": float(g.s.tau),
            "Re_run": inst["U"] * inst["length"] / ((float(g.s.tau) - 0.5) / 3.0),
            "tile": list(batch.tile(k)), "area": areas[k],
            "cd": drag_coefficient(g, inst["U"], areas[k]),
            "guard_resets": g.guard_resets(),
        })
    batch.close()
    if solo:
        sgrids = [build_grid(i, storage, tau_clamp) for i in insts]

        def solo_all():
            for inst, g in zip(insts, sgrids):
                if warmup:
                    g.step(inst["U"], n=warmup)
                g.step(inst["U"], n=steps)

        import torch
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        solo_all()
        torch.cuda.synchronize()
        solo_s = time.perf_counter() - t0
        res["solo_wall_ms"] = solo_s * 1e3
        res["solo_mlups_wall"] = total / solo_s / 1e6 if not warmup else None
        same = 0
        for k, g in enumerate(sgrids):
            cd = drag_coefficient(g, insts[k]["U"], areas[k])
            res["per_instance"][k]["cd_solo"] = cd
            same += cd == res["per_instance"][k]["cd"]
        res["cd_identical"] = same
        for g in sgrids:
            g.close()
    for g in grids:
        g.close()
    return res


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--storage", default="fp32")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--schedule", choices=["fused", "graph"], default=None,
                    help="run this schedule instead of the autotuner's pick")
    ap.add_argument("--no-solo", action="store_true")
    ap.add_argument("--tau-clamp", action="store_true",
                    help="viscosity through the reference driver's rule (tau >= 0.52)")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    indices = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")) % torch.cuda.device_count())
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dims = [i["dims"] for i in geometry.sweep_instances(a.seed, a.count)]
        indices = shard(dims, world, rank)
    res = run_sweep(a.count, a.steps, a.seed, not a.no_autotune, not a.no_solo, a.storage,
                    indices=indices, tau_clamp=a.tau_clamp, schedule=a.schedule)
    if world > 1:
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        dist.destroy_process_group()
        if rank != 0:
            return 0
        res = merge_ranks(gathered)
    summary = {k: v for k, v in res.items() if k != "per_instance"}
    tiles = {}
    for p in res["per_instance"]:
        tiles[f"{p['tile'][0]}x{p['tile'][1]}"] = tiles.get(f"{p['tile'][0]}x{p['tile'][1]}", 0) + 1
    summary["tiles"] = tiles
    summary["instances_with_guard_resets"] = sum(p["guard_resets"] > 0 for p in res["per_instance"])
    summary["re_run_range"] = [min(p["Re_run"] for p in res["per_instance"]),
                               max(p["Re_run"] for p in res["per_instance"])]
    print(json.dumps(summary))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
