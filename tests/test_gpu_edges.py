"""Edge cases of the integrators and entry points built after the implicit
substep: empty scenes, a single particle, restart files of an empty scene."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm

pytestmark = pytest.mark.gpu

DX = 1.0 / 64


@pytest.mark.parametrize("integrator", ["explicit", "mls", "admm"])
def test_empty_scene(cuda_lib, tmp_path, integrator):
    s = mpm.MpmSimulation(DX, precision="fp64", grid_log2=8)
    if integrator == "explicit":
        s.useExplicit()
    elif integrator == "mls":
        s.useExplicit(mls_mpm=True)
    else:
        s.useAdmm(admm_max_iterations=3)
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    assert s.advanceOneTimeStep(1e-3) == abi.OK
    assert s.last_stats["num_particles"] == 0
    assert s.calculateDt(0.01) == 0.01
    s.write(tmp_path / "empty.dat")
    s.read(tmp_path / "empty.dat")
    assert s.count == 0
    s.writePartio(tmp_path / "empty.bgeo")
    assert (tmp_path / "empty.bgeo").stat().st_size == 41 + 2


@pytest.mark.parametrize("integrator", ["newton", "explicit"])
def test_single_particle_with_phase_field_and_sand(cuda_lib, oracle, integrator):
    """One particle: one group, one page; the phase-field CG and the return maps
    run on it, and the library matches the oracle."""
    def one(lib):
        kw = {"grid_log2": 8} if lib is None else {}
        s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), lib=lib, **kw)
        h = s.addParticles(np.array([[0.5, 0.5, 0.5]]), np.array([[0.1, -0.2, 0.05]]), 1000 * DX ** 3 / 8, DX ** 3 / 8)
        h.addFBasedMpmForceWithPhaseField(0.05, 0.5 * DX, mpm.NeoHookeanBorden(1e4, 0.3))
        h.addPlasticity(None, mpm.NonAssociativeCamClay(-0.01, 45.0, 0.3, 3.0, True))
        s.setParticles(F=np.diag([1.2, 1.0, 0.95])[None])
        if integrator == "explicit":
            s.useExplicit()
        return s
    sims = [one(None), one(oracle)]
    for _ in range(3):
        for s in sims:
            assert s.advanceOneTimeStep(5e-4) == abi.OK
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    for k in ("X", "V", "F"):
        np.testing.assert_allclose(pg[k], po[k], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(sims[0].getPhaseField()["c"], sims[1].getPhaseField()["c"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(sims[0].getLogJp(), sims[1].getLogJp(), rtol=0, atol=1e-12)


def test_destroy_releases_device_memory(cuda_lib):
    """zmpm_destroy frees every device array a context allocated: MIXED Newton
    (with MINRES's FP32 Krylov copies), the phase-field solve and ADMM, each
    created, stepped and destroyed repeatedly, leave the device's free memory
    where it was."""
    import torch
    from tests.scenes import build_scene

    def cycle():
        for kind in ("mixed", "phase_field", "admm"):
            s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision="mixed" if kind == "mixed" else "fp64", grid_log2=8)
            h, _ = build_scene(s, kind="nh" if kind == "phase_field" else "hencky", n=16, dx=DX)
            if kind == "phase_field":
                h.addFBasedMpmForceWithPhaseField(0.05, 0.5 * DX)
            if kind == "admm":
                s.useAdmm(admm_max_iterations=2)
            assert s.advanceOneTimeStep(1e-3) == abi.OK, (kind, s.last_stats)
            s.close()

    cycle()  # first use: the library's one-time allocations
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        cycle()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 >= free0 - (4 << 20), (free0 - free1) / 2**20
