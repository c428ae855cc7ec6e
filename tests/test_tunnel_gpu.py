"""The headless driver (LBM_TunnelRun and the lattice_tunnel executable) on
the GPU against the restated reference loop on the CPU oracle: every printed
line must be identical (forces are bit-exact, so Cd, Cl, EMA, t* and the
Strouhal line follow)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from lattice_fluid_dynamics_b200 import build, capi, geometry
from tests import tunnel_oracle as to

CASE = dict(nx=48, ny=24, nz=24, duration=4, substeps=2)


def _expected(oracle, obj, case):
    m = capi.Model(obj)
    lines, info = to.run(oracle, m, case["nx"], case["ny"], case["nz"], case["duration"],
                         substeps=case["substeps"])
    if len(info["cl"]) >= 12:
        st, f = capi.strouhal(np.float32(info["cl"]), case["substeps"], info["charLength"], 0.05)
        lines.append("St=%.4f (f=%.6f, L=%.1f, U=%.3f)" % (st, f, np.float32(info["charLength"]),
                                                           np.float32(0.05)))
        assert st == pytest.approx(info["st"], rel=1e-5, abs=1e-7)
    return lines, info


@pytest.fixture(scope="module")
def body_obj(tmp_path_factory):
    tris, _ = geometry.ahmed_body(length=1.0, center=(0.0, 0.0, 0.0), n_theta=14, n_phi=14)
    path = str(tmp_path_factory.mktemp("tunnel") / "ahmed_small.obj")
    geometry.write_obj(tris, path)
    return path


@pytest.mark.gpu
def test_tunnel_run_matches_restated_loop(solver, oracle, body_obj, tmp_path):
    log = str(tmp_path / "run.log")
    r = capi.tunnel_run(modelPath=body_obj, gridX=CASE["nx"], gridY=CASE["ny"],
                        gridZ=CASE["nz"], renderDuration=CASE["duration"],
                        substeps=CASE["substeps"], logPath=log)
    got = [ln for ln in open(log).read().splitlines() if not ln.startswith("Tunnel:")]
    exp, info = _expected(oracle, body_obj, CASE)
    assert got == exp
    assert r.frames == info["frames"] and r.cdSamples == info["samples"] >= 12
    assert r.latticeSteps == r.frames * CASE["substeps"]


@pytest.mark.gpu
def test_tunnel_executable_stdout(solver, oracle, body_obj, tmp_path):
    """The executable with the reference's options prints the same lines."""
    cmd = [build.TUNNEL, f"--model={body_obj}", "--wind=1", "--viz=1", "--collision=2",
           f"--duration={CASE['duration']}", f"--output={tmp_path}",
           f"--grid={CASE['nx']}x{CASE['ny']}x{CASE['nz']}", f"--substeps={CASE['substeps']}"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    start = lines.index(next(ln for ln in lines if ln.startswith("Model loaded:")))
    got = [ln for ln in lines[start:] if not ln.startswith("Tunnel:")]
    exp, _ = _expected(oracle, body_obj, CASE)
    assert got == exp
    # scraped the way modal_worker.py:505-551 does
    cds = [float(ln.split("Cd=")[1].split()[0]) for ln in lines if "Cd=" in ln]
    assert len(cds) >= 12 and all(np.isfinite(cds))
    assert any(ln.startswith("St=") and "f=" in ln for ln in lines)
    assert any("Effective Re" in ln for ln in lines)


@pytest.mark.gpu
def test_tunnel_aabb_fallback_and_vti(solver, tmp_path):
    """No model: the reference falls back to an AABB of computeModelBounds'
    default box; VTI dumps land every vtkInterval frames."""
    vti = tmp_path / "vti"
    vti.mkdir()
    r = capi.tunnel_run(modelPath="", gridX=32, gridY=16, gridZ=16, renderDuration=1,
                        substeps=1, vtkOutputPath=str(vti), vtkInterval=25,
                        logPath=str(tmp_path / "log"))
    assert r.triangles == 0 and r.solidCells > 0
    files = sorted(os.listdir(vti))
    assert files == [f"field_{k:06d}.vti" for k in range(25, r.frames + 1, 25)]
