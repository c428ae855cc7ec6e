"""Learned warm start: train the warm-start network on solver snapshots and
measure what it gains.

Pipeline (all on the GPU, through this library's C ABI):

1. Shapes: random unions (one or two disjoint closed meshes) of ellipsoids,
   boxes and slanted boxes drawn from a seed, placed around world x = -2 the
   way the reference driver places a model (simulation/src/main.c:341-349),
   with U ~ U[0.04, 0.08] and Re ~ U[20, 100] on the body length.
2. Snapshots: each training shape is solved from uniform flow at half the
   evaluation resolution (regularized collision, periodic y/z, tau from Re
   with the reference driver's 0.52 clamp), all shapes of a chunk advanced
   together by LBM_BatchRun; the developed field is reduced to the network's
   resolution (LBM_WarmNetGridTargets) beside its features
   (LBM_WarmNetGridFeatures).
3. Training: Adam on mean squared error over the snapshots, with the
   network's own forward and backward kernels (LBM_WarmNetTrainStepDevice).
4. Evaluation on held-out shapes at the full resolution: a long cold FP32
   run from uniform flow gives the converged Cd (its mean over the last
   steps); then the steps and wall time for Cd, averaged over a trailing
   window that spans several acoustic periods of the tunnel (the raw Cd
   carries a few per cent of pressure-wave oscillation, which the reference
   driver smooths with an EMA, simulation/src/main.c:1308-1314), to enter
   and stay within 0.5 % of it, for
   (a) plain FP32 from uniform flow and (b) FP16 storage initialised by the
   network (LBM_InitializeFromWarmNet), with fallback to uniform flow when
   the warm-started run trips the stability guard or produces a non-finite
   drag.

    python -m lattice_fluid_dynamics_b200.warmstart --train 2000 --eval 100
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

from . import capi, geometry


# ---------------------------------------------------------------------------
# shapes

def _primitive(rng, kind, center, size):
    if kind == "ellipsoid":
        v, f = geometry.ellipsoid_cells(center, size, 20, 20)
    elif kind == "box":
        v, f = geometry.slanted_box_cells(center, size, 0.0)
    else:
        v, f = geometry.slanted_box_cells(center, size, float(rng.uniform(15, 35)))
    return np.asarray(v, np.float64), f


def random_union(seed: int, index: int) -> dict:
    """One shape in world coordinates: a main primitive and, half of the
    time, a second disjoint one downstream or beside it."""
    rng = np.random.default_rng([seed, index])
    kinds = ("ellipsoid", "box", "slanted_box")
    k1 = kinds[int(rng.integers(0, 3))]
    s1 = np.array([rng.uniform(0.5, 1.3), rng.uniform(0.3, 0.8), rng.uniform(0.3, 0.8)])
    c1 = np.array([-2.0, rng.uniform(-0.15, 0.15), rng.uniform(-0.15, 0.15)])
    parts = [_primitive(rng, k1, c1, s1)]
    if rng.random() < 0.5:
        k2 = kinds[int(rng.integers(0, 3))]
        s2 = np.array([rng.uniform(0.25, 0.6), rng.uniform(0.2, 0.5), rng.uniform(0.2, 0.5)])
        if rng.random() < 0.5:  # downstream, with a gap
            c2 = c1 + [(s1[0] + s2[0]) / 2 + rng.uniform(0.15, 0.5), rng.uniform(-0.2, 0.2), 0]
        else:                   # beside, with a gap
            side = 1 if rng.random() < 0.5 else -1
            c2 = c1 + [rng.uniform(-0.3, 0.3), side * ((s1[1] + s2[1]) / 2 + rng.uniform(0.1, 0.3)),
                       0]
        parts.append(_primitive(rng, k2, c2, s2))
    tris, verts = [], []
    for v, f in parts:
        t = np.zeros((len(f), 12), np.float32)
        fa = np.asarray(f)
        t[:, 0:3], t[:, 4:7], t[:, 8:11] = v[fa[:, 0]], v[fa[:, 1]], v[fa[:, 2]]
        tris.append(t)
        verts.append(v)
    v = np.concatenate(verts)
    lo, hi = v.min(0), v.max(0)
    return dict(index=index, triangles=np.concatenate(tris),
                bbox=tuple(float(x) for x in (*lo, *hi)), length_world=float(hi[0] - lo[0]),
                U=float(rng.uniform(0.04, 0.08)), Re=float(rng.uniform(20, 100)))


def make_grid(shape: dict, dims, storage: str = "fp32") -> capi.Grid:
    """storage: fp32 | fp16 | bf16 | fp64, with "-fast" for LBM_ARITH_FAST."""
    nx, ny, nz = dims
    L_cells = shape["length_world"] * nx / 8.0
    _, nu, _, _ = capi.reynolds_to_tau(shape["U"], L_cells, shape["Re"])
    fast = storage.endswith("-fast")
    g = capi.Grid(nx, ny, nz, nu, storage=storage.replace("-fast", ""))
    g.set(useRegularized=1, periodicYZ=1,
          arithmetic=capi.LBM_ARITH_FAST if fast else capi.LBM_ARITH_EXACT)
    g.set_solid_mesh(shape["triangles"], shape["bbox"])
    return g


# ---------------------------------------------------------------------------
# snapshots

def make_dataset(count: int, seed: int, dims=(128, 64, 64), steps: int = 6000,
                 chunk: int = 64, factor: int = 2):
    """Features [count, vox, 3] and targets [count, vox, 4] as CUDA tensors,
    and each instance's stability-guard reset count (instances with resets
    are left out of training)."""
    import torch
    nx, ny, nz = dims
    vox = (nx // factor) * (ny // factor) * (nz // factor)
    feats = torch.zeros((count, vox, 3), dtype=torch.float32, device="cuda")
    tgts = torch.zeros((count, vox, 4), dtype=torch.float32, device="cuda")
    L = capi.load()
    resets = np.zeros(count, np.int64)
    for c0 in range(0, count, chunk):
        shapes = [random_union(seed, i) for i in range(c0, min(count, c0 + chunk))]
        grids = [make_grid(s, dims) for s in shapes]
        for s, g in zip(shapes, grids):
            g.initialize_flow(s["U"])
        b = capi.Batch(grids)
        b.run(steps, np.array([[s["U"], 0, 0] for s in shapes], np.float32))
        for k, (s, g) in enumerate(zip(shapes, grids)):
            i = c0 + k
            rc1 = L.LBM_WarmNetGridFeatures(g.handle, factor, s["U"], s["Re"],
                                            feats[i].data_ptr())
            rc2 = L.LBM_WarmNetGridTargets(g.handle, factor, s["U"], tgts[i].data_ptr())
            assert rc1 == 0 and rc2 == 0
            resets[i] = g.guard_resets()
        b.close()
        for g in grids:
            g.close()
    return feats, tgts, resets


# ---------------------------------------------------------------------------
# training

def train(net: capi.WarmNet, feats, tgts, epochs: int, batch: int, lr: float, seed: int = 0,
          val=None, warmup: int = 200, clip: float = 1.0):
    """Adam with linear warm-up then cosine decay and global gradient-norm
    clipping; with a validation set, the weights of the best validation loss
    are kept."""
    import torch
    n = feats.shape[0]
    rng = np.random.default_rng(seed)
    steps = epochs * (n // batch)
    net.set_grad_clip(clip)
    best, best_params = math.inf, None
    history, t0, s = [], time.perf_counter(), 0
    fb = torch.empty((batch,) + tuple(feats.shape[1:]), dtype=torch.float32, device="cuda")
    tb = torch.empty((batch,) + tuple(tgts.shape[1:]), dtype=torch.float32, device="cuda")
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).cuda()
        losses = []
        for j in range(n // batch):
            idx = perm[j * batch:(j + 1) * batch]
            torch.index_select(feats, 0, idx, out=fb)
            torch.index_select(tgts, 0, idx, out=tb)
            torch.cuda.synchronize()
            lr_s = lr * min(1.0, (s + 1) / warmup) * 0.5 * (1 + math.cos(math.pi * s / steps))
            losses.append(net.train_step_device(fb.data_ptr(), tb.data_ptr(), batch, lr_s))
            s += 1
        rec = {"epoch": ep, "train_loss": float(np.mean(losses))}
        if val is not None:
            rec["val_loss"] = evaluate_loss(net, *val)
            if rec["val_loss"] < best:
                best, best_params = rec["val_loss"], net.params()
        history.append(rec)
    if best_params is not None:
        net.set_params(best_params)
    return history, time.perf_counter() - t0


def evaluate_loss(net: capi.WarmNet, feats, tgts) -> float:
    out = []
    for i in range(feats.shape[0]):
        loss, _ = net.loss_grad(feats[i].cpu().numpy(), tgts[i].cpu().numpy(), want_grad=False)
        out.append(loss)
    return float(np.mean(out))


# ---------------------------------------------------------------------------
# evaluation

def _run(g: capi.Grid, U: float, area: float, sample: int, steps: int, stop=None):
    """Raw Cd every `sample` steps for `steps` steps (or until stop(cds) is
    true); returns (cd list, host seconds at each sample)."""
    import torch
    cds, times = [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done = 0
    while done < steps:
        g.step(U, n=sample)
        done += sample
        cds.append(float(g.drag_coefficient(U, area)))
        times.append(time.perf_counter() - t0)
        if not math.isfinite(cds[-1]) or (stop is not None and stop(cds)):
            break
    return cds, times


def smoothed(cds, window: int):
    """Trailing mean over `window` samples (shorter at the start)."""
    c = np.cumsum(np.concatenate([[0.0], np.asarray(cds, float)]))
    i = np.arange(1, len(cds) + 1)
    lo = np.maximum(0, i - window)
    return (c[i] - c[lo]) / (i - lo)


def entry_index(avg, ref, band=0.005):
    """First sample after which the smoothed Cd stays within band of ref."""
    ok = np.abs(np.asarray(avg) - ref) <= band * abs(ref)
    bad = np.nonzero(~ok)[0]
    if len(bad) == 0:
        return 0
    i = int(bad[-1]) + 1
    return i if i < len(avg) else None


VARIANTS = {
    "cold_fp32": ("fp32", "cold"),   # the plain path
    "warm_fp16": ("fp16", "warm"),   # learned warm start + FP16 storage
    "warm_fp32": ("fp32", "warm"),
    "warmu_fp16": ("fp16", "warm_velocity"),
    "warmc_fp16": ("fp16", "warm_flux"),
    # FP16 storage with the contracted / approximate-division step kernels:
    # the storage rounding (~1e-3) dominates the arithmetic's
    "warmc_fp16fast": ("fp16-fast", "warm_flux"),
    "warmc_fp32": ("fp32", "warm_flux"),
    "cold_fp16": ("fp16", "cold"),
}


def evaluate(net: capi.WarmNet, shapes, dims=(256, 128, 128), sample: int = 50,
             cold_steps: int = 30000, avg_steps: int = 2000, ref_steps: int = 5000,
             hold_steps: int = 5000, variants=("warm_fp16",), fp16_reference: bool = False):
    """Per shape: the converged Cd (mean of the raw Cd over the last
    ref_steps of a cold FP32 run of cold_steps) and, for the cold FP32 run
    and every variant, the steps and wall time until the Cd averaged over the
    trailing avg_steps enters and stays within 0.5 % of it (a variant's run
    stops once it has stayed in the band for hold_steps).  Warm variants fall
    back to uniform flow when the warm-started run trips the stability guard
    or its drag is not finite.

    With fp16_reference, a cold FP16-storage run of cold_steps gives a second
    converged Cd (its own, `cd_ref16`, row "cold_fp16_ref"), and every
    FP16-storage variant also reports the steps and wall time to the band
    around that value ("steps16", "wall_s16"): warm vs uniform start with
    FP16 storage on, each measured against the FP16 cold start's converged Cd.
    Those variants then run until they have held both bands."""
    import torch
    rows = []
    w = max(1, avg_steps // sample)
    hold = max(1, hold_steps // sample)
    L = capi.load()

    def held(cds, ref):
        e = entry_index(smoothed(cds, w), ref)
        return e is not None and len(cds) - e >= hold

    for s in shapes:
        U = s["U"]
        g = make_grid(s, dims, "fp32")
        area = g.projected_area(0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.initialize_flow(U)
        init_cold = time.perf_counter() - t0
        cd_c, t_c = _run(g, U, area, sample, cold_steps)
        cold_resets = g.guard_resets()
        g.close()
        ref = float(np.mean(cd_c[-max(1, ref_steps // sample):]))
        ic = entry_index(smoothed(cd_c, w), ref)
        row = {"index": s["index"], "U": U, "Re": s["Re"], "cd_ref": ref,
               "cold_fp32": {"steps": None if ic is None else (ic + 1) * sample,
                             "wall_s": None if ic is None else init_cold + t_c[ic],
                             "ms_per_step": 1e3 * t_c[-1] / (len(t_c) * sample),
                             "guard_resets": cold_resets,
                             "series": [round(v, 5) for v in smoothed(cd_c, w)[::10]]}}

        ref16 = None
        if fp16_reference:
            g = make_grid(s, dims, "fp16")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g.initialize_flow(U)
            init16 = time.perf_counter() - t0
            cd_h, t_h = _run(g, U, area, sample, cold_steps)
            resets16 = g.guard_resets()
            g.close()
            ref16 = float(np.mean(cd_h[-max(1, ref_steps // sample):]))
            ih = entry_index(smoothed(cd_h, w), ref16)
            row["cd_ref16"] = ref16
            row["cold_fp16_ref"] = {
                "steps": None if ih is None else (ih + 1) * sample,
                "wall_s": None if ih is None else init16 + t_h[ih],
                "ms_per_step": 1e3 * t_h[-1] / (len(t_h) * sample),
                "guard_resets": resets16,
                "series": [round(v, 5) for v in smoothed(cd_h, w)[::10]]}

        for name in variants:
            storage, init = VARIANTS[name]
            use16 = ref16 is not None and storage.startswith("fp16")

            def stop(cds):
                if len(cds) < w:
                    return False
                return held(cds, ref) and (not use16 or held(cds, ref16))

            g = make_grid(s, dims, storage)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fallback = False
            if init == "cold":
                g.initialize_flow(U)
            else:
                flags = {"warm": 0, "warm_velocity": 1, "warm_flux": 2}[init]
                if L.LBM_InitializeFromWarmNet(g.handle, net.handle, U, s["Re"], flags) != 0:
                    g.initialize_flow(U)
                    fallback = True
            torch.cuda.synchronize()
            t_init = time.perf_counter() - t0
            cd_v, t_v = _run(g, U, area, sample, cold_steps, stop)
            if init != "cold" and not fallback and (
                    g.guard_resets() > 0 or not all(map(math.isfinite, cd_v))):
                g.initialize_flow(U)  # unstable warm start: plain start from uniform flow
                fallback = True
                cd_v, t_v = _run(g, U, area, sample, cold_steps, stop)
            g.close()
            iv = entry_index(smoothed(cd_v, w), ref)
            row[name] = {"steps": None if iv is None else (iv + 1) * sample,
                         "wall_s": None if iv is None else t_init + t_v[iv],
                         "init_s": t_init, "fallback": fallback,
                         "ms_per_step": 1e3 * t_v[-1] / (len(t_v) * sample),
                         "cd_end": float(np.mean(cd_v[-w:])),
                         "series": [round(v, 5) for v in smoothed(cd_v, w)[::10]]}
            if use16:
                i16 = entry_index(smoothed(cd_v, w), ref16)
                row[name]["steps16"] = None if i16 is None else (i16 + 1) * sample
                row[name]["wall_s16"] = None if i16 is None else t_init + t_v[i16]
        rows.append(row)
    return rows


def summarize(rows, variant="warm_fp16"):
    """Medians and totals of steps / wall time to the 0.5 % band, `variant`
    against the plain cold FP32 path, over shapes where both entered it."""
    ok = [r for r in rows if r["cold_fp32"]["steps"] and r.get(variant, {}).get("steps")]
    out = {"variant": variant, "evaluated": len(rows), "both_converged": len(ok),
           "fallbacks": int(sum(r.get(variant, {}).get("fallback", False) for r in rows))}
    if not ok:
        return out
    cs = np.array([r["cold_fp32"]["steps"] for r in ok], float)
    vs = np.array([r[variant]["steps"] for r in ok], float)
    ct = np.array([r["cold_fp32"]["wall_s"] for r in ok], float)
    vt = np.array([r[variant]["wall_s"] for r in ok], float)
    out.update({
        "cold_steps_median": float(np.median(cs)), "steps_median": float(np.median(vs)),
        "cold_wall_s_median": float(np.median(ct)), "wall_s_median": float(np.median(vt)),
        "wall_ratio_median": float(np.median(vt / ct)),
        "wall_ratio_total": float(vt.sum() / ct.sum()),
        "steps_ratio_total": float(vs.sum() / cs.sum()),
        "faster_fraction": float(np.mean(vt < ct)),
    })
    return out


def summarize_fp16(rows, variant="warmc_fp16"):
    """The same medians and totals for an FP16-storage variant against the
    cold FP16 start, both measured by the band around the cold FP16 start's
    own converged Cd (rows made with fp16_reference)."""
    ok = [r for r in rows if r.get("cold_fp16_ref", {}).get("steps")
          and r.get(variant, {}).get("steps16")]
    out = {"variant": variant, "baseline": "cold_fp16_ref", "evaluated": len(rows),
           "both_converged": len(ok)}
    if not ok:
        return out
    cs = np.array([r["cold_fp16_ref"]["steps"] for r in ok], float)
    vs = np.array([r[variant]["steps16"] for r in ok], float)
    ct = np.array([r["cold_fp16_ref"]["wall_s"] for r in ok], float)
    vt = np.array([r[variant]["wall_s16"] for r in ok], float)
    out.update({
        "cold_steps_median": float(np.median(cs)), "steps_median": float(np.median(vs)),
        "cold_wall_s_median": float(np.median(ct)), "wall_s_median": float(np.median(vt)),
        "wall_ratio_median": float(np.median(vt / ct)),
        "wall_ratio_total": float(vt.sum() / ct.sum()),
        "steps_ratio_total": float(vs.sum() / cs.sum()),
        "faster_fraction": float(np.mean(vt < ct)),
    })
    return out


def bench_train(steps: int, batch: int = 8, dims=(64, 32, 32)) -> dict:
    """Time `steps` training steps (forward + backward + Adam) on synthetic
    data at the network resolution `dims` (x, y, z) with CUDA events on the
    network's stream; algorithmic FLOPs = 3 x forward convolution FLOPs."""
    import torch
    nx, ny, nz = dims
    net = capi.WarmNet(nx, ny, nz, max_batch=batch, seed=1)
    rng = np.random.default_rng(0)
    m = batch * nx * ny * nz
    feats = torch.from_numpy(np.stack([(rng.random(m) < 0.1), np.full(m, 0.05),
                                       np.full(m, 300.0)], 1).astype(np.float32)).cuda()
    tgt = torch.from_numpy(rng.normal(size=(m, 4)).astype(np.float32)).cuda()
    for _ in range(3):
        net.train_step_device(feats.data_ptr(), tgt.data_ptr(), batch, 1e-4)
    stream = torch.cuda.ExternalStream(capi.load().LBM_WarmNetGetStream(net.handle))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        net.train_step_device(feats.data_ptr(), tgt.data_ptr(), batch, 1e-4)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    flops = 3 * batch * forward_flops(nx, ny, nz)
    return {"dims": [nx, ny, nz], "batch": batch, "ms_per_step": ms,
            "gflop_per_step": flops / 1e9, "tflops": flops / (ms * 1e-3) / 1e12}


# (cin, cout, dims (nb, nz, ny, nx)) of the convolutions bench_conv times:
# the network's shapes at batch 8 and a 64x32x32 input
CONV_SHAPES = [(16, 16, (8, 32, 32, 64)), (48, 16, (8, 32, 32, 64)), (8, 16, (8, 32, 32, 64)),
               (16, 32, (8, 16, 16, 32)), (96, 32, (8, 16, 16, 32)),
               (192, 64, (8, 8, 8, 16)), (64, 128, (8, 4, 4, 8))]


def bench_conv(reps: int, ops=("fwd", "wgrad"), paths=(0, 1, 2)) -> list:
    """Time LBM_NNConvForward / LBM_NNConvWeightGrad at the network's
    shapes (CONV_SHAPES) through the C ABI with CUDA events, `reps` calls
    after one untimed call, for each kernel path of LBM_NNSetConvPath
    (0: halo / pipelined, 1: synchronous gather, 2: pipelined gather).
    Random BF16 data; one dict per (shape, op, path)."""
    import torch
    L = capi.load()
    out = []

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / reps * 1e3

    try:
        for cin, cout, dims in CONV_SHAPES:
            m = int(np.prod(dims))
            nt = max(16, cout)
            x = torch.randn(m, cin, device="cuda").to(torch.bfloat16)
            w = (torch.randn(nt, L.LBM_NNKPad(cin), device="cuda") * 0.05).to(torch.bfloat16)
            y = torch.zeros(m, nt, device="cuda", dtype=torch.bfloat16)
            g = torch.randn(m, nt, device="cuda").to(torch.bfloat16)
            wsb = L.LBM_NNWgradWorkspaceBytes(cin, nt, *dims, 8)
            ws = torch.zeros(wsb // 4, device="cuda")
            dw = torch.zeros(nt, 27 * cin, device="cuda")
            flops = 2.0 * m * 27 * cin * cout
            calls = {
                "fwd": lambda: L.LBM_NNConvForward(x.data_ptr(), cin, 0, cin, w.data_ptr(), None,
                                                   nt, 1, y.data_ptr(), None, nt, 0, nt, 0,
                                                   *dims, None),
                "wgrad": lambda: L.LBM_NNConvWeightGrad(x.data_ptr(), cin, 0, cin, g.data_ptr(),
                                                        nt, nt, nt, dw.data_ptr(), 0,
                                                        ws.data_ptr(), wsb, 8, *dims, None),
            }
            for path in paths:
                L.LBM_NNSetConvPath(path)
                for op in ops:
                    us = timed(calls[op])
                    out.append({"op": op, "path": path, "cin": cin, "cout": cout,
                                "dims": list(dims), "us": round(us, 1),
                                "tflops": round(flops / us / 1e6, 1)})
    finally:
        L.LBM_NNSetConvPath(0)
    if L.LBM_NNTakeError() != 0:
        raise RuntimeError("a convolution kernel gave up waiting for its tensor-core work")
    return out


# (cin, cout, level) of the 16 convolutions
_LAYERS = [(8, 16, 0), (16, 16, 0), (16, 32, 1), (32, 32, 1), (32, 64, 2), (64, 64, 2),
           (64, 128, 3), (128, 128, 3), (128, 128, 3), (192, 64, 2), (64, 64, 2), (96, 32, 1),
           (32, 32, 1), (48, 16, 0), (16, 16, 0), (16, 4, 0)]


def forward_flops(nx: int, ny: int, nz: int) -> float:
    """Algorithmic FLOPs of one forward pass per sample: 2 per multiply-add
    of every 3x3x3 convolution (real channels)."""
    vox = nx * ny * nz
    return float(sum(2 * 27 * ci * co * (vox >> (3 * lv)) for ci, co, lv in _LAYERS))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--val", type=int, default=64)
    ap.add_argument("--eval", type=int, default=100)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--snapshot-steps", type=int, default=6000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=3e-4)
    ap.add_argument("--grid", default="256x128x128")
    ap.add_argument("--cold-steps", type=int, default=30000)
    ap.add_argument("--sample", type=int, default=50)
    ap.add_argument("--variants", default="warm_fp16",
                    help="comma list of " + ",".join(VARIANTS))
    ap.add_argument("--params", default="", help="trained parameters (.npy): skip training")
    ap.add_argument("--scaling", default="", help="results .json holding the output scaling")
    ap.add_argument("--bench-train", type=int, default=0,
                    help="only time this many training steps on synthetic data")
    ap.add_argument("--bench-conv", type=int, default=0,
                    help="only time the convolution kernels at the network's shapes (calls)")
    ap.add_argument("--conv-op", default="fwd,wgrad", help="--bench-conv: fwd and / or wgrad")
    ap.add_argument("--conv-path", default="0,1,2", help="--bench-conv: kernel paths")
    ap.add_argument("--fp16-reference", action="store_true",
                    help="also measure FP16 variants against a cold FP16 run's converged Cd")
    ap.add_argument("--out", default="")
    a = ap.parse_args(argv)
    if a.bench_train:
        print(json.dumps(bench_train(a.bench_train, a.batch)))
        return 0
    if a.bench_conv:
        for row in bench_conv(a.bench_conv, tuple(a.conv_op.split(",")),
                              tuple(int(v) for v in a.conv_path.split(","))):
            print(json.dumps(row), flush=True)
        return 0
    full = tuple(int(v) for v in a.grid.split("x"))
    half = tuple(v // 2 for v in full)
    res = {"grid": list(full), "snapshot_grid": list(half), "train": a.train, "seed": a.seed}
    net = capi.WarmNet(full[0] // 4, full[1] // 4, full[2] // 4, max_batch=a.batch, seed=a.seed)
    hist = []
    if a.params:
        net.set_params(np.load(a.params))
        if a.scaling:
            sc = json.load(open(a.scaling))["output_scaling"]
            net.set_output_scaling(sc["scale"], sc["shift"])
    else:
        hist = _train_from_snapshots(net, a, half, res)
    # held-out shapes: indices beyond the training and validation ones
    shapes = [random_union(a.seed, 100000 + i) for i in range(a.eval)]
    variants = tuple(a.variants.split(","))
    rows = evaluate(net, shapes, full, a.sample, a.cold_steps, variants=variants,
                    fp16_reference=a.fp16_reference)
    res["rows"] = rows
    if a.out:  # the rows first: they hold everything the summaries are made from
        with open(a.out, "w") as fh:
            json.dump(res, fh)
    res["summary"] = {v: summarize(rows, v) for v in variants}
    if a.fp16_reference:
        res["summary_fp16_reference"] = {
            v: summarize_fp16(rows, v) for v in variants if VARIANTS[v][0].startswith("fp16")}
    print(json.dumps({k: v for k, v in res.items() if k not in ("rows", "history")} |
                     {"final": hist[-1] if hist else None}))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh, indent=1)
        np.save(a.out.replace(".json", "_params.npy"), net.params())
    return 0


def train_from_snapshots(net, count: int, val: int, seed: int, snapshot_dims, snapshot_steps: int,
                         epochs: int, batch: int, lr: float, res: dict | None = None):
    """Solve `count + val` random shapes (seed) from uniform flow at
    snapshot_dims for snapshot_steps, keep those that never tripped the
    stability guard, set the network's output scaling from the targets'
    spread, and train on the first share with the rest as validation.
    Returns the loss history; `res` (if given) receives the bookkeeping."""
    import torch
    res = {} if res is None else res
    t0 = time.perf_counter()
    feats, tgts, resets = make_dataset(count + val, seed, snapshot_dims, snapshot_steps)
    res["dataset_s"] = time.perf_counter() - t0
    res["dataset_unstable"] = int((resets > 0).sum())
    res["dataset_unstable_shapes"] = [
        {k: v for k, v in random_union(seed, int(i)).items() if k in ("index", "U", "Re",
                                                                    "length_world")}
        for i in np.nonzero(resets > 0)[0][:20]]
    keep = np.nonzero(resets == 0)[0]
    kt = torch.from_numpy(keep).cuda()
    feats, tgts = feats.index_select(0, kt), tgts.index_select(0, kt)
    ntr = int(round(len(keep) * count / (count + val)))
    t = tgts.reshape(-1, 4)
    res["target_stats"] = {"mean": t.mean(0).tolist(), "std": t.std(0).tolist(),
                           "min": t.min(0).values.tolist(), "max": t.max(0).values.tolist()}
    # every output channel in units of its spread over the training set
    mean, std = t.mean(0), t.std(0).clamp_min(1e-6)
    tgts = ((tgts - mean) / std).clamp(-8.0, 8.0)  # rare stagnation-point outliers
    net.set_output_scaling(std.cpu().numpy(), mean.cpu().numpy())
    res["output_scaling"] = {"scale": std.tolist(), "shift": mean.tolist()}
    hist, tsec = train(net, feats[:ntr], tgts[:ntr], epochs, batch, lr,
                       val=(feats[ntr:], tgts[ntr:]) if ntr < len(keep) else None)
    res["train_s"] = tsec
    res["history"] = hist
    res["trained_on"] = ntr
    return hist


def _train_from_snapshots(net, a, half, res):
    return train_from_snapshots(net, a.train, a.val, a.seed, half, a.snapshot_steps, a.epochs,
                                a.batch, a.lr, res)


if __name__ == "__main__":
    sys.exit(main())
