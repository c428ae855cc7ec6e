"""Benchmark of the D3Q19 wind-tunnel hot path (MLUPS vs the HBM roofline).

Workload (the headline configuration): the procedural Ahmed-style body
(19,800 triangles, 64 cells long) in a 256x128x128 FP32 lattice, MRT +
Smagorinsky (Cs = 0.1), tau from Re = 5e4 at U = 0.05 set directly
(tau = 0.50019), periodic y/z, Bouzidi links from ray-triangle q.  A
"step" is one LBM_Step over all 4,194,304 cells.  The populations (2 x 319
MB) are larger than the 126 MB L2, so consecutive steps stream from HBM.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  python bench.py --op-table [--storage ...] [--op ...] [--arith ...] [--kernel ...]
  python bench.py --cpu-table

Under torchrun (N > 1) every rank runs an independent replica of the
workload (the hot path is single-grid; multi-GPU is replicas only); value
is the sum of cell updates over ranks divided by the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "ahmed_256x128x128_mrt_smagorinsky_fp32"
NX, NY, NZ = 256, 128, 128
U = 0.05
FLAGS = dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1, periodicYZ=1)


def tau_c2() -> float:
    from lattice_fluid_dynamics_b200 import geometry as G
    return G.reynolds_tau(U, 64.0, 5e4)


def config(n_gpus: int) -> dict:
    return {"workload": WORKLOAD, "grid": [NX, NY, NZ], "cells": NX * NY * NZ,
            "collision": "MRT+Smagorinsky(Cs=0.1)", "tau": round(tau_c2(), 6),
            "body": "Ahmed-style 1.044x0.389x0.288, 25deg slant, 19800 tris, 64 cells",
            "boundaries": "Zou-He inlet/outlet, periodic y/z, Bouzidi links",
            "storage": "fp32", "l2_policy": "working set 638 MB > 126 MB L2 (no flush needed)",
            "parallelism": f"replicas{n_gpus}" if n_gpus > 1 else "single-gpu"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int, path: str | None):
        self.index, self.path, self.proc = index, path, None

    def __enter__(self):
        try:
            self.out = open(self.path, "w") if self.path else subprocess.PIPE
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.out, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.text = ""
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        if self.path:
            self.out.close()
            out = open(self.path).read()
        self.text = out or ""

    def summary(self) -> dict:
        rows = []
        for line in (self.text or "").splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        load = [r for r in rows if r[2] > 250.0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in load for k in range(4)
                          if r[3][k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in load),
                "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(load)}


# ---------------------------------------------------------------------------
# distributed plumbing (replicas)
# ---------------------------------------------------------------------------
def dist_setup(n_gpus: int, backend: str | None = None):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    phys = local
    if world > 1:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        if vis:
            ids = vis.split(",")
            phys = int(ids[local]) if ids[local].isdigit() else local
            os.environ["CUDA_VISIBLE_DEVICES"] = ids[local]
        else:
            os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    else:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        if vis and vis.split(",")[0].isdigit():
            phys = int(vis.split(",")[0])
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend is None:  # one GPU per rank over NCCL; gloo on a host without GPUs
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, phys, pg


def _on_gpu(pg) -> bool:
    return pg.get_backend() == "nccl"


def barrier(pg):
    if pg is not None:
        import torch
        t = torch.zeros(1, device="cuda" if _on_gpu(pg) else "cpu")
        pg.all_reduce(t)
        if _on_gpu(pg):
            torch.cuda.synchronize()


def max_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], device="cuda" if _on_gpu(pg) else "cpu", dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_mlups(world: int, cells: int, steps: int, ms_max: float) -> float:
    """Whole-job MLUPS of `world` replicas that each advanced `cells` by
    `steps` steps, timed by the slowest rank (ms_max)."""
    return world * cells * steps / (ms_max / 1e3) / 1e6


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle port on the host cores
# ---------------------------------------------------------------------------
def cpu_oracle_run(budget_s: float, max_steps: int, warmup: int = 1):
    from lattice_fluid_dynamics_b200 import geometry as G
    from oracle import pyoracle as po
    po.build()
    po.set_threads(0)
    tris, bbox = G.ahmed_body()
    g = po.OracleGrid(NX, NY, NZ, 1e-4)
    g.set(tau=tau_c2(), **FLAGS)
    g.set_solid_mesh(tris, bbox)
    g.initialize_flow(U)
    for _ in range(max(warmup, 0)):
        g.step(U)
    t0 = time.perf_counter()
    g.step(U)
    t1 = time.perf_counter()
    per = t1 - t0
    n = max(1, min(max_steps - 1, int(budget_s / max(per, 1e-6)) - 1))
    t2 = time.perf_counter()
    g.step(U, n=n)
    t3 = time.perf_counter()
    steps = n + 1
    secs = (t3 - t2) + per
    cores = os.cpu_count() or 1
    return NX * NY * NZ * steps / secs / 1e6, steps, secs, cores


def cpu_table(budget_s: float) -> list:
    """The oracle's FP32 BGK and MRT steps on the host cores at config 1
    (128x64x64, sphere of radius 8 cells, tau 0.6, half-way bounce-back) and
    config 2 (the bench workload, and the same with BGK): MLUPS from a
    bounded number of steps after one untimed step."""
    from lattice_fluid_dynamics_b200 import geometry as G
    from oracle import pyoracle as po
    po.build()
    po.set_threads(0)
    tris, bbox = G.ahmed_body()
    c1 = ((32 + 0.5) / 16 - 4, (32 + 0.5) / 16 - 2, (32 + 0.5) / 16 - 2, 0.5)
    cases = [
        ("c1_sphere_128x64x64_bgk", (128, 64, 64), dict(), "sphere"),
        ("c1_sphere_128x64x64_mrt", (128, 64, 64), dict(useMRT=1), "sphere"),
        ("c2_ahmed_256x128x128_bgk", (NX, NY, NZ), dict(periodicYZ=1), "mesh"),
        ("c2_ahmed_256x128x128_mrt_smagorinsky", (NX, NY, NZ), FLAGS, "mesh"),
    ]
    rows = []
    for name, (nx, ny, nz), flags, body in cases:
        if body == "sphere":
            g = po.OracleGrid(nx, ny, nz, (0.6 - 0.5) / 3)
            g.set(tau=0.6, **flags)
            g.set_solid_sphere(*c1, halfway=True)
        else:
            g = po.OracleGrid(nx, ny, nz, 1e-4)
            g.set(tau=tau_c2(), **flags)
            g.set_solid_mesh(tris, bbox)
        g.initialize_flow(U)
        g.step(U)
        t0 = time.perf_counter()
        g.step(U)
        per = time.perf_counter() - t0
        n = max(1, int(budget_s / max(per, 1e-6)) - 1)
        t0 = time.perf_counter()
        g.step(U, n=n)
        secs = time.perf_counter() - t0 + per
        g.close()
        rows.append({"case": name, "cells": nx * ny * nz, "steps": n + 1,
                     "seconds": round(secs, 2),
                     "mlups": round(nx * ny * nz * (n + 1) / secs / 1e6, 2),
                     "threads": os.cpu_count() or 1, "kind": "port"})
    return rows


def reference_arm(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    budget = float(os.environ.get("LBM_REF_BUDGET_S", "60"))
    warm = min(max(args.warmup, 3), 10)  # untimed CPU steps, bounded
    mlups, steps, secs, cores = cpu_oracle_run(budget, max(args.steps, 2), warmup=warm)
    line = {"metric": "MLUPS", "value": round(mlups, 3), "unit": "MLUPS", "impl": "reference",
            "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": round(1e3 * secs / steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(world),
            "cpu_baseline": {"value": round(mlups, 3), "unit": "MLUPS", "cores": cores,
                             "kind": "port",
                             "sample": f"{steps} steps of the full 256x128x128 workload "
                                       f"({secs:.1f} s) on the C oracle (OpenMP, all host threads); "
                                       "the reference's GLSL shaders cannot run (no graphics stack)"},
            "e2e": {"value": round(mlups, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# step-kernel table: every storage format, collision operator, arithmetic
# mode and step kernel on the same Ahmed-body tunnel
# ---------------------------------------------------------------------------
TABLE_OPS = {
    "bgk": dict(),
    "reg": dict(useRegularized=1),
    "mrt": dict(useMRT=1),
    "mrt_smag": dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1),
}


def table_grid(dims, storage: str, op: str, arith: int, staged: bool, tris, bbox):
    from lattice_fluid_dynamics_b200 import capi
    nx, ny, nz = dims
    g = capi.Grid(nx, ny, nz, 1e-4, storage=storage)
    g.set(tau=tau_c2(), periodicYZ=1, arithmetic=arith, **TABLE_OPS[op])
    if g.set_tma_staging(staged) != staged:
        g.close()
        raise RuntimeError(f"TMA staging unavailable for {storage} {dims}")
    g.set_solid_mesh(tris, bbox)
    g.initialize_flow(U)
    return g


def table_timed(g, steps: int) -> float:
    """CUDA-event milliseconds of `steps` graph-replayed steps on the grid's
    stream, after 64 untimed steps."""
    import torch
    g.step(U, n=64)
    stream = torch.cuda.ExternalStream(g.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    g.step(U, n=steps)
    e1.record(stream)
    e1.synchronize()
    g.check()
    return e0.elapsed_time(e1)


def table_readbacks(g, k: int) -> dict:
    """Host microseconds of one drag readback and of one LBM_Step + readback
    (means over k; both are synchronous, so host time is the cost)."""
    g.drag_force_decomposed()
    t0 = time.perf_counter()
    for _ in range(k):
        g.drag_force_decomposed()
    t1 = time.perf_counter()
    for _ in range(k):
        g.step(U)
        g.drag_force_decomposed()
    t2 = time.perf_counter()
    g.check()
    return {"readback_us": round(1e6 * (t1 - t0) / k, 1),
            "step_readback_us": round(1e6 * (t2 - t1) / k, 1)}


def op_table(args) -> int:
    """One JSON line per (storage, operator, arithmetic, kernel): MLUPS and
    GB/s of algorithmic population traffic over --table-steps graph-replayed
    steps.  --loop N instead runs N single LBM_Step launches per case with no
    timing (a short target for a profiler); --readback K adds K synchronous
    drag readbacks per case (timed unless --loop)."""
    from lattice_fluid_dynamics_b200 import geometry as G
    dims = tuple(int(v) for v in args.dims.split("x"))
    tris, bbox = G.ahmed_body()
    cells = dims[0] * dims[1] * dims[2]
    for storage in args.storage:
        for op in args.op:
            for arith in args.arith:
                for kernel in args.kernel:
                    g = table_grid(dims, storage, op, arith, kernel == "staged", tris, bbox)
                    row = dict(storage=storage, op=op, arith=arith, kernel=kernel,
                               dims=list(dims))
                    if args.loop:
                        g.step_loop(U, n=args.loop)
                        for _ in range(args.readback):
                            g.drag_force_decomposed()
                        g.check()
                    else:
                        ms = table_timed(g, args.table_steps)
                        sec = ms * 1e-3
                        row.update(steps=args.table_steps, ms=round(ms, 3),
                                   mlups=round(cells * args.table_steps / sec / 1e6, 1),
                                   gb_per_s=round(cells * args.table_steps * g.bytes_per_update()
                                                  / sec / 1e9, 1))
                        if args.readback:
                            row.update(table_readbacks(g, args.readback))
                    g.close()
                    print(json.dumps(row), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=500)
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--clocks-file", default=None)
    ap.add_argument("--cpu-table", action="store_true",
                    help="time the CPU oracle's BGK and MRT steps at configs 1 and 2, then exit")
    ap.add_argument("--op-table", action="store_true",
                    help="time the step kernel per storage / operator / arithmetic / kernel "
                         "on the Ahmed-body tunnel, then exit")
    ap.add_argument("--dims", default="256x128x128", help="--op-table grid")
    ap.add_argument("--storage", nargs="+", default=["fp32", "fp16", "bf16"],
                    help="--op-table storage formats")
    ap.add_argument("--op", nargs="+", default=["bgk", "reg", "mrt_smag"],
                    choices=sorted(TABLE_OPS), help="--op-table collision operators")
    ap.add_argument("--arith", nargs="+", type=int, default=[0], choices=[0, 1],
                    help="--op-table arithmetic: 0 exact, 1 fast")
    ap.add_argument("--kernel", nargs="+", default=["direct"], choices=["direct", "staged"],
                    help="--op-table step kernel: direct, or TMA-staged")
    ap.add_argument("--table-steps", type=int, default=512, help="--op-table timed steps")
    ap.add_argument("--loop", type=int, default=0, help="--op-table: untimed launches only")
    ap.add_argument("--readback", type=int, default=0, help="--op-table: drag readbacks")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return reference_arm(args)
    if args.cpu_table:
        for row in cpu_table(args.cpu_budget / 4):
            print(json.dumps(row), flush=True)
        return 0
    if args.op_table:
        return op_table(args)

    world, rank, phys, pg = dist_setup(args.gpus)
    import numpy as np
    import torch

    import lattice_fluid_dynamics_b200 as lfd
    from lattice_fluid_dynamics_b200 import geometry as G

    torch.cuda.set_device(0)
    tris, bbox = G.ahmed_body()
    g = lfd.Grid(NX, NY, NZ, 1e-4, storage="fp32")
    g.set(tau=tau_c2(), **FLAGS)
    g.set_solid_mesh(tris, bbox)
    A = g.projected_area(0)
    g.initialize_flow(U)
    stream = torch.cuda.ExternalStream(g.stream_ptr())
    cells = NX * NY * NZ

    # warm-up (fused steps through the CUDA-graph path, as timed)
    g.step(U, n=args.warmup)
    torch.cuda.synchronize()
    barrier(pg)

    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(phys, args.clocks_file) as clk:
        barrier(pg)
        torch.cuda.synchronize()
        e0.record(stream)
        g.step(U, n=args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(pg)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(pg, ms)
    g.check()

    # end-to-end through the C ABI: every step passes the host inlet
    # velocity (3 floats of launch parameters) and reads the drag back to
    # the host (LBM_ComputeDragForceDecomposed, a device->host copy)
    ke = min(args.e2e_steps, args.steps)
    barrier(pg)
    torch.cuda.synchronize()
    h0 = torch.cuda.Event(enable_timing=True)
    h1 = torch.cuda.Event(enable_timing=True)
    h0.record(stream)
    cds = []
    for _ in range(ke):
        g.step(U)
        f = g.drag_force_decomposed()
        cds.append(abs(float(f[0])) / (0.5 * U * U * A))
    h1.record(stream)
    h1.synchronize()
    e2e_ms = max_over_ranks(pg, h0.elapsed_time(h1))

    bpu = g.bytes_per_update()
    per_launch_s = ms_max / 1e3 / args.steps
    achieved = bpu * cells / per_launch_s / 1e9
    peak, peak_kind = peaks()
    mlups = job_mlups(world, cells, args.steps, ms_max)
    e2e_mlups = job_mlups(world, cells, ke, e2e_ms)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        c_mlups, c_steps, c_secs, cores = cpu_oracle_run(args.cpu_budget, 1000)
        cpu = {"value": round(c_mlups, 3), "unit": "MLUPS", "cores": cores, "kind": "port",
               "sample": f"{c_steps} steps of the full 256x128x128 workload ({c_secs:.1f} s) on "
                         "the C oracle, OpenMP over all host threads"}

    if rank == 0:
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "dram_traffic_per_launch.txt")
        if os.path.exists(tpath):
            for line in open(tpath):
                parts = line.split()
                if len(parts) == 2 and parts[0] == WORKLOAD:
                    traffic = int(parts[1])
        line = {
            "metric": "MLUPS", "value": round(mlups, 2), "unit": "MLUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_max / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config(world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind,
                         "bytes_per_update": bpu},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_mlups, 2), "unit": "MLUPS", "steps": ke,
                    "h2d_bytes_per_step": 12, "d2h_bytes_per_step": 14 * 8},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "cd_last": round(cds[-1], 5) if cds else None,
            "guard_resets": g.guard_resets(),
        }
        print(json.dumps(line), flush=True)
    g.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
