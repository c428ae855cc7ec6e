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
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import capi, geometry


def build_grid(inst: dict, storage: str = "fp32") -> capi.Grid:
    """One instance through the reference's API: viscosity from Re with the
    reference's 0.52 tau clamp (simulation/src/main.c:447-460), mesh body,
    periodic y/z, uniform inlet flow."""
    nx, ny, nz = inst["dims"]
    _, nu, _, _ = capi.reynolds_to_tau(inst["U"], inst["length"], inst["Re"])
    g = capi.Grid(nx, ny, nz, nu, storage=storage)
    g.set(useRegularized=1 if inst["op"] == "reg" else 0, periodicYZ=1)
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


def run_sweep(count: int = 64, steps: int = 3000, seed: int = 1, autotune: bool = True,
              solo: bool = True, storage: str = "fp32", warmup: int = 0) -> dict:
    insts = geometry.sweep_instances(seed, count)
    t0 = time.perf_counter()
    grids = [build_grid(i, storage) for i in insts]
    setup_s = time.perf_counter() - t0
    areas = [g.projected_area(0) for g in grids]
    cells = np.array([np.prod(i["dims"]) for i in insts], np.int64)
    inlets = np.array([[i["U"], 0.0, 0.0] for i in insts], np.float32)
    batch = capi.Batch(grids)
    t0 = time.perf_counter()
    if autotune:
        batch.autotune(10)
    tune_s = time.perf_counter() - t0
    if warmup:
        batch.run(warmup, inlets)
    ms = _timed(batch.stream, lambda: batch.run(steps, inlets))
    total = int(cells.sum()) * steps
    res = {
        "instances": count, "steps": steps, "seed": seed, "storage": storage,
        "cells_total": int(cells.sum()), "ms": ms,
        "mlups": total / (ms * 1e-3) / 1e6,
        "gb_per_s": total * grids[0].bytes_per_update() / (ms * 1e-3) / 1e9,
        "tiles_per_step": batch.tiles_per_step, "schedule": batch.schedule,
        "setup_s": setup_s, "autotune_s": tune_s,
        "per_instance": [],
    }
    for k, (inst, g) in enumerate(zip(insts, grids)):
        res["per_instance"].append({
            "index": k, "dims": list(inst["dims"]), "kind": inst["kind"], "op": inst["op"],
            "U": inst["U"], "Re": inst["Re"], "tau": float(g.s.tau),
            "tile": list(batch.tile(k)), "area": areas[k],
            "cd": drag_coefficient(g, inst["U"], areas[k]),
            "guard_resets": g.guard_resets(),
        })
    batch.close()
    if solo:
        sgrids = [build_grid(i, storage) for i in insts]

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
    ap.add_argument("--no-solo", action="store_true")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    res = run_sweep(a.count, a.steps, a.seed, not a.no_autotune, not a.no_solo, a.storage)
    summary = {k: v for k, v in res.items() if k != "per_instance"}
    tiles = {}
    for p in res["per_instance"]:
        tiles[f"{p['tile'][0]}x{p['tile'][1]}"] = tiles.get(f"{p['tile'][0]}x{p['tile'][1]}", 0) + 1
    summary["tiles"] = tiles
    print(json.dumps(summary))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
