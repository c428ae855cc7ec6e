"""Host logic of the headless driver (LBM_Tunnel*, LBM_CdMonitor*) against a
float32 restatement of simulation/src/main.c:893-1391 (tests/tunnel_oracle.py),
and the driver executable's command line (simulation/src/cli.c)."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

import lattice_fluid_dynamics_b200 as lfd
from lattice_fluid_dynamics_b200 import build, capi

from tests import tunnel_oracle as to

f32 = np.float32


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build()
    lfd.load()


def test_ramp_factor():
    L = capi.load()
    for frame in range(0, 420):
        assert f32(L.LBM_TunnelRampFactor(frame)) == to.ramp(frame)


@pytest.mark.parametrize("nx", [32, 48, 128, 256, 512])
@pytest.mark.parametrize("U", [0.02, 0.05, 0.1])
@pytest.mark.parametrize("sub", [1, 2, 10])
def test_cd_start_frame(nx, U, sub):
    L = capi.load()
    for max_frames in [0, 30, 60, 240, 301, 600, 1800, 100000]:
        assert L.LBM_TunnelCdStartFrame(nx, U, sub, max_frames) == \
            to.cd_start_frame(nx, f32(U), sub, max_frames)


def test_coefficients():
    rng = np.random.default_rng(3)
    for _ in range(500):
        fx, fy, px = (f32(v) for v in rng.normal(0, 2, 3))
        U = f32(rng.uniform(0.01, 0.1))
        area = f32(rng.choice([0.0, 1e-9, rng.uniform(1, 500)]))
        fac = f32(rng.uniform(0.8, 1.0))
        c = capi.tunnel_coefficients(fx, fy, px, U, area, fac)
        r = to.coefficients(fx, fy, px, U, area, fac)
        got = tuple(f32(v) for v in (c.cd, c.cdCorr, c.cl, c.cdPressure, c.cdFriction))
        assert got == r


def test_cd_monitor_matches_restatement():
    rng = np.random.default_rng(5)
    # a noisy transient with rejected samples, then a tail that settles
    cd = list(rng.uniform(-1, 3, 40)) + [2000.0, 0.0, -3.0] + \
        list(1.2 + 0.3 * np.exp(-np.arange(300) / 30.0) + 0.002 * rng.standard_normal(300))
    m = capi.CdMonitor()
    r = to.Monitor()
    converged_at = None
    for i, v in enumerate(cd):
        v = f32(v)
        corr = f32(v * f32(0.97))
        a = m.add(v, corr)
        b = r.add(v, corr)
        assert a == b
        assert f32(m.m.ema) == r.ema
        assert m.m.historyCount == r.count
        if a:
            converged_at = i
            assert f32(m.m.convergedMean) == r.mean
            assert f32(m.m.convergedRelStd) == r.rel
    assert converged_at is not None and m.m.converged == 1
    assert list(np.float32(m.m.history)) == [f32(v) for v in r.hist]


def test_cd_monitor_ema_reseeds_until_first_accepted_sample():
    m = capi.CdMonitor()
    m.add(-1.0, 5.0)       # rejected: EMA seeded, history empty
    m.add(0.5, 0.4)        # first accepted: EMA re-seeded
    assert m.m.ema == pytest.approx(0.4) and m.m.historyCount == 1
    m.add(0.5, 1.4)
    assert f32(m.m.ema) == f32(f32(0.1) * f32(1.4)) + f32(f32(0.9) * f32(0.4))


def test_defaults_are_the_references():
    o = capi.tunnel_defaults()
    assert (o.gridX, o.gridY, o.gridZ, o.substeps, o.vtkInterval) == (128, 64, 64, 10, 100)
    assert f32(o.windSpeed) == f32(1.0) and f32(o.smagorinskyCs) == f32(0.1)
    assert f32(o.latticeVelocity) == f32(0.05)


def test_cli_help_and_arguments():
    exe = build.TUNNEL
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "Usage:" in r.stdout and "--grid" in r.stdout
    r = subprocess.run([exe, "--wind=1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "--duration" in r.stderr
    r = subprocess.run([exe, "-d", "1", "--storage=fp8"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 2


def test_run_rejects_bad_options():
    with pytest.raises(RuntimeError):
        capi.tunnel_run(renderDuration=0)
    with pytest.raises(RuntimeError):
        capi.tunnel_run(renderDuration=1, substeps=0)
