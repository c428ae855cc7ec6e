"""Restatement of the reference driver's solver loop on the CPU oracle.

Follows simulation/src/main.c:438-553 (Re -> tau, grid set-up, effective Re,
projected area and blockage) and :893-1391 (ramp, Cd start frame, sampling,
EMA, convergence, auto-stop), drag_metrics.c:8-68 for St, all in float32
scalar arithmetic, and produces the lines the reference prints in the order
it prints them.  Used by the tests as the expected output of the headless
driver (LBM_TunnelRun); the model is ingested through the library's OBJ
loader, which is pinned separately to the reference's loadOBJ.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32


def ramp(frame: int):
    return f32(frame) / f32(300) if frame < 300 else f32(1.0)


def cd_start_frame(size_x: int, U, substeps: int, max_frames: int) -> int:
    flow = int(f32(size_x) / (f32(f32(U) * f32(substeps)) * f32(2)))
    start = 300 + 3 * flow
    if max_frames > 0 and start >= max_frames:
        start = max_frames * 2 // 3
        if start < 300 and max_frames > 300:
            start = 300
    return start


class Monitor:
    def __init__(self):
        self.hist = [f32(0)] * 100
        self.count = 0
        self.converged = False
        self.ema = f32(0)
        self.mean = f32(0)
        self.rel = f32(0)

    def add(self, cd, cd_corr) -> bool:
        if self.count == 0:
            self.ema = f32(cd_corr)
        else:
            a = f32(0.1)
            self.ema = f32(a * f32(cd_corr)) + f32(f32(f32(1.0) - a) * self.ema)
        if not (cd > 0 and cd < 1000):
            return False
        self.hist[self.count % 100] = f32(cd)
        self.count += 1
        if self.count < 100 or self.converged:
            return False
        mean = f32(0)
        for v in self.hist:
            mean = f32(mean + v)
        mean = f32(mean / f32(100))
        var = f32(0)
        for v in self.hist:
            d = f32(v - mean)
            var = f32(var + f32(d * d))
        rel = f32(np.sqrt(f32(var / f32(100))) / f32(mean + f32(1e-10)))
        if rel < f32(0.01):
            self.converged, self.mean, self.rel = True, mean, rel
            return True
        return False


def coefficients(fx, fy, px, U, area, factor):
    dyn = f32(f32(f32(0.5) * f32(1.0)) * f32(U)) * f32(U)
    den = f32(dyn * f32(area))
    ok = den > f32(1e-10)
    cd = f32(abs(f32(fx)) / den) if ok else f32(0)
    cl = f32(f32(fy) / den) if ok else f32(0)
    cdp = f32(abs(f32(px)) / den) if ok else f32(0)
    cdf = f32(cd - cdp)
    if cdf < 0:
        cdf = f32(0)
    return cd, f32(cd * f32(factor)), cl, cdp, cdf


def strouhal(cl, substeps: int, L, U):
    """drag_metrics.c:8-68 in float32 with libm-equivalent cos/sin from numpy
    float32 (compared by value tolerance, not by printed digits)."""
    n_all = len(cl)
    start = n_all * 35 // 100
    sig = np.asarray(cl[start:], np.float64)
    n = len(sig)
    w = 0.5 * (1 - np.cos(2 * np.pi * np.arange(n) / (n - 1)))
    x = (sig - sig.mean()) * w
    fs = 1.0 / (20 * substeps)
    k = np.arange(1, n // 2)
    ang = 2 * np.pi * np.outer(k, np.arange(n)) / n
    pw = (x @ np.cos(ang).T) ** 2 + (x @ np.sin(ang).T) ** 2
    if len(pw) == 0:
        return 0.0, 0.0
    f = k[int(np.argmax(pw))] * fs / n
    return (f * L / U if U > 1e-10 else 0.0), f


def run(po, model, nx, ny, nz, duration, substeps=10, U=0.05, wind=1.0, reynolds=0.0,
        cs=0.1):
    """Returns (lines, info).  `model` is a capi.Model; `po` the oracle module."""
    out = []
    p = out.append
    p(f"Model loaded: {model.vertex_count} vertices, {model.face_count} faces")
    s, off, rot = model.place()
    p("Auto scale: %.6f" % s)
    p("Auto-rotation: %d deg" % int(rot))
    b = model.bounds(s, off, rot)
    p("Model bounds (rotated %.1f deg): min(%.2f, %.2f, %.2f) max(%.2f, %.2f, %.2f)"
      % (rot, *[float(v) for v in b[:6]]))
    tris = model.triangles(s, off, rot)
    p(f"Created {len(tris)} valid triangles")
    U = f32(U)
    charL = f32(f32(b[3] - b[0]) * f32(f32(nx) / f32(8.0)))
    re = f32(reynolds)
    if re <= 0:
        re = f32(f32(200.0) * f32(wind))
        if re < f32(50):
            re = f32(50)
    nu = f32(f32(U * charL) / re)
    tau = f32(f32(f32(3.0) * nu) + f32(0.5))
    if tau < f32(0.52):
        nu = f32(f32(f32(0.52) - f32(0.5)) / f32(3.0))
        tau = f32(0.52)
        actual = f32(f32(U * charL) / nu)
        p("  Re capped at %.0f (tau=%.2f needed for stable Cd, requested Re=%.0f)"
          % (actual, tau, re))
        re = actual
    p("Reynolds number: %.0f" % re)
    p("  Char length: %.1f lattice units" % charL)
    p("  Viscosity: %.6f" % nu)
    p("  tau: %.4f" % tau)
    p("  CFL: %.4f" % U)
    p("Initializing LBM grid...")
    g = po.OracleGrid(nx, ny, nz, float(nu))
    gtau = f32(g.tau)
    p("LBM Grid: %dx%dx%d (%d cells), tau=%.3f" % (nx, ny, nz, nx * ny * nz, gtau))
    g.set_solid_mesh(tris, tuple(float(v) for v in b[:6]))
    p("LBM mesh solid: %d cells marked as solid" % int((g.solid == 1).sum()))
    g.set(periodicYZ=1, useSmagorinsky=1, smagorinskyCs=float(cs), useMRT=1)
    p("Smagorinsky SGS enabled (Cs=%.2f), periodic YZ" % f32(cs))
    p("MRT collision enabled")
    assert g.initialize_flow(float(U), 0.0, 0.0)
    nug = f32(f32(gtau - f32(0.5)) / f32(3.0))
    re_eff = f32(f32(U * charL) / nug) if nug > f32(1e-10) else f32(0)
    p("Effective Re = %.0f (U=%.3f, L=%.1f, nu=%.4f)" % (re_eff, U, charL, nug))
    p("  Sample interval: %d lattice steps" % substeps)
    sY, sZ = f32(f32(ny) / f32(4.0)), f32(f32(nz) / f32(4.0))
    bbox_area = f32(f32(f32(f32(b[4] - b[1]) * sY) * f32(b[5] - b[2])) * sZ)
    area = f32(g.projected_area(0))
    if area < f32(1.0):
        area = bbox_area
    eps = f32(area / f32(f32(ny) * f32(nz)))
    factor = f32(f32(f32(1.0) - eps) * f32(f32(1.0) - eps))
    p("LBM initialized successfully")
    cells = nx * ny * nz
    lbm_bytes = cells * 152 + cells * 16 + cells * 4
    p("  LBM buffers:      %.1f MB (%dx%dx%d grid)" % (lbm_bytes / (1024.0 * 1024.0), nx, ny, nz))
    p("  Triangle mesh:    %.1f MB (%d triangles)" % (len(tris) * 48.0 / (1024.0 * 1024.0),
                                                      len(tris)))
    p("  Total:            %.1f MB" % ((lbm_bytes + len(tris) * 48.0) / (1024.0 * 1024.0)))
    frame, outf, max_frames = 0, 0, duration * 60
    mon = Monitor()
    cl = []
    diag = False
    samples = 0
    while True:
        frame += 1
        g.step(float(f32(U * ramp(frame))), 0.0, 0.0, n=substeps)
        start = cd_start_frame(nx, U, substeps, max_frames)
        skip = frame < start
        if frame >= start and frame % 20 == 0:
            fx, fy, fz, px, py, pz = (f32(v) for v in g.drag_force_decomposed())
            cd, cdc, c_l, cdp, cdf = coefficients(fx, fy, px, U, area, factor)
            if not diag:
                by = f32(f32(b[4] - b[1]) * sY)
                bz = f32(f32(b[5] - b[2]) * sZ)
                p("  Cd calculation breakdown:")
                p("    Re = %.0f, U_lattice = %.4f, rho_0 = %.1f" % (re, U, 1.0))
                p("    Body (lattice): %.1f x %.1f x %.1f cells" % (charL, by, bz))
                p("    Projected area = %.1f cells^2 (bbox = %.1f)" % (area, bbox_area))
                p("    Blockage = %.1f%%, correction = %.3f (Pope & Harper 1966)"
                  % (f32(eps * f32(100.0)), factor))
                if min(by, bz) < 10.0:
                    p("    WARNING: body < 10 cells across -- Cd is unreliable at this resolution")
                if eps > f32(0.05):
                    p("    WARNING: blockage > 5% -- confinement inflates Cd")
                diag = True
            newly = mon.add(cd, cdc)
            steps = frame * substeps
            tstar = f32(f32(f32(steps) * U) / charL) if charL > 0 else f32(0)
            ft = f32(f32(f32(steps) * U) / f32(nx))
            p("  Drag Force: (%.4f, %.4f, %.4f), Cd=%.3f Cd_corr=%.3f Cl=%.3f (avg=%.3f) "
              "t*=%.3f flow-throughs=%.2f" % (fx, fy, fz, cd, cdc, c_l, mon.ema, tstar, ft))
            p("  Cd_pressure=%.3f Cd_friction=%.3f" % (cdp, cdf))
            cl.append(c_l)
            samples += 1
            if newly:
                p("  Cd converged (mean=%.3f, relStd=%.4f)" % (mon.mean, mon.rel))
                if outf + 120 < max_frames:
                    max_frames = outf + 120
        if outf >= max_frames:
            p("Render complete: %d frames" % outf)
            break
        if not skip:
            outf += 1
    st, f = strouhal(cl, substeps, float(charL), float(U)) if len(cl) >= 12 else (0.0, 0.0)
    g.close()
    # the St line itself is printed from the library's pinned Strouhal routine
    # by the caller; `st`/`f` here are an independent float64 evaluation
    return out, {"frames": frame, "samples": samples, "st": st, "f": f, "cl": cl,
                 "charLength": float(charL), "ema": float(mon.ema)}
