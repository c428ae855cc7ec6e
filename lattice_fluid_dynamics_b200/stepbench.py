"""Step-kernel throughput per storage format, collision operator, arithmetic
mode and step kernel (direct or TMA-staged), on the 256x128x128 Ahmed-body
tunnel (periodic y/z, Re 5e4 at U = 0.05).

Each case makes a fresh grid, runs 64 untimed steps, then times `--steps`
steps (LBM_StepN, CUDA graph chunks) with CUDA events on the grid's stream
and prints one JSON line: MLUPS and GB/s of algorithmic population traffic.
`--loop N` instead runs N single LBM_Step launches per case and no timing
(a short target for a profiler).  `--readback K` adds K synchronous drag
readbacks (LBM_ComputeDragForceDecomposed) per case; when timing, it reports
the host time of one readback alone and of one LBM_Step + readback pair, the
end-to-end loop of the reference's driver.

    python -m lattice_fluid_dynamics_b200.stepbench --storage fp16 --op bgk
    python -m lattice_fluid_dynamics_b200.stepbench --loop 3 --storage fp16 --op bgk
"""
from __future__ import annotations

import argparse
import json

from . import capi, geometry

OPS = {
    "bgk": dict(),
    "reg": dict(useRegularized=1),
    "mrt": dict(useMRT=1),
    "mrt_smag": dict(useMRT=1, useSmagorinsky=1, smagorinskyCs=0.1),
}
U = 0.05


def make(dims, storage: str, op: str, arith: int, staged: bool, tris, bbox) -> capi.Grid:
    nx, ny, nz = dims
    g = capi.Grid(nx, ny, nz, 1e-4, storage=storage)
    g.set(tau=geometry.reynolds_tau(U, 64.0, 5e4), periodicYZ=1, arithmetic=arith, **OPS[op])
    if g.set_tma_staging(staged) != staged:
        g.close()
        raise RuntimeError(f"TMA staging unavailable for {storage} {dims}")
    g.set_solid_mesh(tris, bbox)
    g.initialize_flow(U)
    return g


def timed(g: capi.Grid, steps: int) -> float:
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


def readbacks(g: capi.Grid, k: int) -> dict:
    """Host microseconds of one drag readback and of one LBM_Step + readback
    (means over k; both are synchronous, so host time is the cost)."""
    import time
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


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--dims", default="256x128x128")
    ap.add_argument("--storage", nargs="+", default=["fp32", "fp16", "bf16"])
    ap.add_argument("--op", nargs="+", default=["bgk", "reg", "mrt_smag"], choices=sorted(OPS))
    ap.add_argument("--arith", nargs="+", type=int, default=[0], choices=[0, 1])
    ap.add_argument("--kernel", nargs="+", default=["direct", "staged"],
                    choices=["direct", "staged"])
    ap.add_argument("--steps", type=int, default=512)
    ap.add_argument("--loop", type=int, default=0)
    ap.add_argument("--readback", type=int, default=0)
    args = ap.parse_args(argv)
    dims = tuple(int(v) for v in args.dims.split("x"))
    tris, bbox = geometry.ahmed_body()
    cells = dims[0] * dims[1] * dims[2]
    for storage in args.storage:
        for op in args.op:
            for arith in args.arith:
                for kernel in args.kernel:
                    g = make(dims, storage, op, arith, kernel == "staged", tris, bbox)
                    row = dict(storage=storage, op=op, arith=arith, kernel=kernel,
                               dims=list(dims))
                    if args.loop:
                        g.step_loop(U, n=args.loop)
                        for _ in range(args.readback):
                            g.drag_force_decomposed()
                        g.check()
                    else:
                        ms = timed(g, args.steps)
                        s = ms * 1e-3
                        row.update(steps=args.steps, ms=round(ms, 3),
                                   mlups=round(cells * args.steps / s / 1e6, 1),
                                   gb_per_s=round(cells * args.steps * g.bytes_per_update()
                                                  / s / 1e9, 1))
                        if args.readback:
                            row.update(readbacks(g, args.readback))
                    g.close()
                    print(json.dumps(row), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
