"""Time-step selection of the CUDA library against the oracle: calculateDt
(MpmSimulationBase.cpp:766-790) from the device-resident particle speeds and
the colliders, and frame stepping (SimulationBase::advanceOneFrame with
TimeStepping)."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene

pytestmark = pytest.mark.gpu

DX = 1.0 / 64


def scene(lib):
    kw = {"grid_log2": 8} if lib is None else {}
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), lib=lib, cfl=0.6, **kw)
    build_scene(s, kind="fcr", n=6, dx=DX, seed=7, v0=(0.5, -1.5, 0.2))
    c = mpm.AnalyticCollisionObject(mpm.Sphere((0, 0, 0), 0.08), abi.SLIP, friction=0.1)
    c.setTranslation((0.45, 0.35, 0.45), (0.0, 0.5, 0.0))
    c.setAngularVelocity((0.0, 2.0, 0.0))
    s.addCollisionObject(c)
    return s


def test_calculate_dt_matches_oracle(cuda_lib, oracle):
    sims = [scene(None), scene(oracle)]
    for _ in range(3):
        dts = [s.calculateDt(0.01) for s in sims]
        assert abs(dts[0] - dts[1]) <= 1e-14 * dts[1]
        for s in sims:
            assert s.advanceOneTimeStep(dts[1]) == abi.OK
    vg, log, hig = sims[0].maxParticleSpeed()
    vo, loo, hio = sims[1].maxParticleSpeed()
    assert abs(vg - vo) <= 1e-12 * vo
    np.testing.assert_allclose(log, loo, rtol=0, atol=1e-12)
    np.testing.assert_allclose(hig, hio, rtol=0, atol=1e-12)


def test_advance_one_frame_matches_oracle(cuda_lib, oracle):
    sims = [scene(None), scene(oracle)]
    counts = []
    for s in sims:
        step = mpm.TimeStepping(frame_dt=1.0 / 120)
        step.max_dt = 2e-3
        counts.append(s.advanceOneFrame(step))
        assert abs(step.time - 1.0 / 120) < 1e-15
    assert counts[0] == counts[1] >= 5
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert np.abs(pg["X"] - po["X"]).max() <= 1e-9 * np.abs(po["X"]).max()


def test_cfl_violation_asks_for_a_restart(cuda_lib):
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), grid_log2=9, cfl=0.6)
    build_scene(s, kind="fcr", n=4, dx=DX, v0=(0, -30.0, 0), lo=(0.4, 0.5, 0.4), ground=None)
    step = mpm.TimeStepping(frame_dt=1.0 / 24)
    step.min_dt = 1e-3  # the clamp overrides the CFL dt: a particle moves 3 cells
    with pytest.raises(mpm.RestartRequired) as e:
        s.advanceOneFrame(step, frame=3)
    assert e.value.frame == 3 and e.value.max_dt == pytest.approx(step.max_dt / 2)
