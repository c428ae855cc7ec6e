"""Precision study: reduced-precision population storage against FP64.

Workload: the Ahmed-style body (geometry.ahmed_body, 2 world units long =
nx/4 cells) in a large lattice (512x192x192 = 18.9 M cells by default), MRT +
Smagorinsky (Cs = 0.1), tau from Re = 5e4 at U = 0.05 (set directly, below
the reference driver's 0.52 clamp), periodic y/z.  The same run is made with
FP64 storage and arithmetic (the reference of the comparison) and with FP32,
FP16 and BF16 storage (FP16/BF16 store the shifted deviation f_i - w_i and
collide in FP32).  Drag and lift are read as FP64 sums of the momentum
exchange (LBM_ComputeDragForceF64); mass as an FP64 sum.

Per storage type: Cd and Cl every `sample` steps and their deviation from
FP64, the relative L2 error of the velocity field at the end (fluid cells),
mass drift, and the step throughput (MLUPS, GB/s of algorithmic population
traffic) timed with CUDA events on the grid's stream.

    python -m lattice_fluid_dynamics_b200.precision --steps 2000
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

from . import capi, geometry

U = 0.05
FLAGS = dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1, periodicYZ=1)


def run_one(storage: str, dims, tris, bbox, tau: float, steps: int, sample: int,
            timed_steps: int):
    import torch
    nx, ny, nz = dims
    g = capi.Grid(nx, ny, nz, 1e-4, storage=storage)
    g.set(tau=tau, **FLAGS)
    g.set_solid_mesh(tris, bbox)
    area = g.projected_area(0)
    g.initialize_flow(U)
    m0 = g.mass_momentum()[0]
    q = 0.5 * U * U * area
    cd, cl = [], []
    done = 0
    while done < steps:
        n = min(sample, steps - done)
        g.step(U, n=n)
        done += n
        f64, _ = g.drag_force_f64()
        cd.append(abs(float(f64[0])) / q)
        cl.append(float(f64[1]) / q)
    vel = g.velocity()
    solid = g.solid()
    mass = g.mass_momentum()[0]
    # throughput: a separate timed run continuing the same flow
    stream = torch.cuda.ExternalStream(g.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    g.step(U, n=timed_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    cells = nx * ny * nz
    out = {
        "storage": storage, "cd": cd, "cl": cl, "mass_drift": float((mass - m0) / m0),
        "mlups": cells * timed_steps / (ms * 1e-3) / 1e6,
        "gb_per_s": cells * timed_steps * g.bytes_per_update() / (ms * 1e-3) / 1e9,
        "bytes_per_update": g.bytes_per_update(), "guard_resets": g.guard_resets(),
    }
    g.close()
    return out, vel, solid


def run_precision(dims=(512, 192, 192), steps: int = 2000, sample: int = 50,
                  timed_steps: int = 500, storages=("fp64", "fp32", "fp16", "bf16")) -> dict:
    nx = dims[0]
    tris, bbox = geometry.ahmed_body()
    tau = geometry.reynolds_tau(U, nx / 4.0, 5e4)
    results = {"dims": list(dims), "steps": steps, "sample": sample, "tau": tau,
               "collision": "MRT+Smagorinsky(Cs=0.1)", "runs": []}
    ref = None
    for s in storages:
        r, vel, solid = run_one(s, dims, tris, bbox, tau, steps, sample, timed_steps)
        fluid = solid == 0
        u = vel[fluid, :3].astype(np.float64)
        if ref is None:
            ref = (r, u)
            r["vs_fp64"] = None
        else:
            cd0, cl0 = np.array(ref[0]["cd"]), np.array(ref[0]["cl"])
            cd1, cl1 = np.array(r["cd"]), np.array(r["cl"])
            r["vs_fp64"] = {
                "cd_final_rel": float(abs(cd1[-1] - cd0[-1]) / abs(cd0[-1])),
                "cd_max_rel": float(np.max(np.abs(cd1 - cd0) / np.abs(cd0))),
                "cd_mean_rel": float(abs(cd1.mean() - cd0.mean()) / abs(cd0.mean())),
                "cl_final_abs": float(abs(cl1[-1] - cl0[-1])),
                "cl_max_abs": float(np.max(np.abs(cl1 - cl0))),
                "l2_u_rel": float(np.linalg.norm(u - ref[1]) / np.linalg.norm(ref[1])),
            }
        results["runs"].append(r)
    return results


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--grid", default="512x192x192")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--sample", type=int, default=50)
    ap.add_argument("--timed-steps", type=int, default=500)
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    dims = tuple(int(v) for v in a.grid.split("x"))
    res = run_precision(dims, a.steps, a.sample, a.timed_steps)
    runs = []
    for r in res["runs"]:
        d = {k: v for k, v in r.items() if k not in ("cd", "cl")}
        d["cd_final"] = r["cd"][-1]
        d["cl_final"] = r["cl"][-1]
        runs.append(d)
    print(json.dumps({"dims": res["dims"], "steps": res["steps"], "tau": res["tau"],
                      "runs": runs}))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
