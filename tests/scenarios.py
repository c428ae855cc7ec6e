"""Shared scenario builder: applies the same sequence of reference API calls
to the CPU oracle and to the CUDA library so their states can be compared.

A scenario is a dict:
  dims=(nx, ny, nz), visc, tau (optional override), flags (dict of
  LBMGrid public fields), geometry (list of (op, args)), init=(ux, uy, uz),
  inlet=(ux, uy, uz), steps.
"""
from __future__ import annotations

import numpy as np


def apply_geometry(target, geometry):
    for op, args in geometry:
        if op == "aabb":
            target.set_solid_aabb(*args)
        elif op == "sphere":
            target.set_solid_sphere(*args)
        elif op == "sphere_halfway":
            target.set_solid_sphere(*args, halfway=True)
        elif op == "ground":
            target.add_ground_plane(*args)
        elif op == "mesh":
            tris, bbox = args
            target.set_solid_mesh(tris, bbox)
        else:
            raise ValueError(op)


def make_oracle(po, sc, prec=4):
    nx, ny, nz = sc["dims"]
    g = po.OracleGrid(nx, ny, nz, sc.get("visc", 0.1), prec=prec)
    if "tau" in sc:
        g.set(tau=sc["tau"])
    g.set(**sc.get("flags", {}))
    apply_geometry(g, sc.get("geometry", []))
    g.initialize_flow(*sc.get("init", (0.05, 0.0, 0.0)))
    return g


def make_gpu(lfd, sc, storage="fp32"):
    nx, ny, nz = sc["dims"]
    g = lfd.Grid(nx, ny, nz, sc.get("visc", 0.1), storage=storage)
    if "tau" in sc:
        g.set(tau=sc["tau"])
    g.set(**sc.get("flags", {}))
    apply_geometry(g, sc.get("geometry", []))
    g.initialize_flow(*sc.get("init", (0.05, 0.0, 0.0)))
    return g


def rel_err(a: np.ndarray, b: np.ndarray, floor: float = 1e-6) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


# test_lbm.c's box (simulation/test/test_lbm.c:276)
BOX = ("aabb", (-0.3, -0.15, -0.15, 0.3, 0.15, 0.15))


def sphere_c1(halfway=False):
    """Config-1 sphere: r = 8 cells centred on lattice cell (32,32,32) of a
    128x64x64 grid (cell centres map to world as (g + 0.5)/scale - offset)."""
    c = ((32 + 0.5) / 16 - 4, (32 + 0.5) / 16 - 2, (32 + 0.5) / 16 - 2)
    return ("sphere_halfway" if halfway else "sphere", (c[0], c[1], c[2], 0.5))
