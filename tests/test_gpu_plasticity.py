"""Drucker-Prager (sand) and non-associative Cam-Clay return maps of the CUDA
library's G2P against the oracle, in implicit and explicit substeps
(PlasticityApplier.cpp:10-317).  FP64 runs differ by summation order only."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene

pytestmark = pytest.mark.gpu

DX = 1.0 / 64


def scene(lib, kind, precision="fp64", integrator="newton", seed=4):
    kw = {"grid_log2": 8} if lib is None else {}
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, lib=lib, **kw)
    model = "hencky" if kind == "dp" else "nh"
    h, x = build_scene(s, kind=model, n=6, dx=DX, v0=(0.2, -2.0, 0.1), lo=(0.375, 8 * DX, 0.375), ground=7 * DX, seed=seed)
    if kind == "dp":
        # dilated sand reaches the cone tip first, then compresses on the ground
        F = np.tile(np.diag([1.04, 1.0, 1.02]), (len(x), 1, 1))
        s.setParticles(F=F)
        h.addPlasticity(None, mpm.DruckerPragerStvkHencky(30.0, 1.0, 0.0, True))
    else:
        h.addPlasticity(None, mpm.NonAssociativeCamClay(-0.01, 45.0, 0.3, 3.0, True))
    s.newton_tolerance = 1e-9
    s.newton_max_iterations = 8
    s.krylov_max_iterations = 60
    if integrator == "explicit":
        s.useExplicit()
    return s


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("kind", ["dp", "cc"])
@pytest.mark.parametrize("integrator", ["newton", "explicit"])
def test_plasticity_matches_oracle_fp64(cuda_lib, oracle, kind, integrator):
    dt = 1e-3 if integrator == "newton" else 2e-4
    sims = [scene(None, kind, integrator=integrator), scene(oracle, kind, integrator=integrator)]
    for _ in range(8):
        for k, s in enumerate(sims):
            rc = s.advanceOneTimeStep(dt)
            assert rc == abi.OK, (k, rc, s.last_stats)
    lg, lo = sims[0].getLogJp(), sims[1].getLogJp()
    assert np.abs(lo).max() > 1e-4
    np.testing.assert_allclose(lg, lo, rtol=1e-7, atol=1e-10)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-10
    assert rel(pg["V"], po["V"]) < 1e-6
    assert rel(pg["F"], po["F"]) < 1e-8


@pytest.mark.parametrize("kind", ["dp", "cc"])
def test_plasticity_mixed_tracks_fp64_oracle(cuda_lib, oracle, kind):
    sims = [scene(None, kind, precision="mixed"), scene(oracle, kind)]
    for _ in range(8):
        for s in sims:
            assert s.advanceOneTimeStep(1e-3) == abi.OK
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-6
    # the return maps run in FP64 on the FP32-evolved F; Cam-Clay's fake hardening
    # (sinh of xi log Jp) amplifies that F's FP32 rounding
    np.testing.assert_allclose(sims[0].getLogJp(), sims[1].getLogJp(), rtol=0, atol=1e-3)


def test_admm_refuses_clay(cuda_lib):
    """The ADMM F-step handles elastic, von Mises and Drucker-Prager particles
    (AdmmSimulationFoam.h:617-633); Cam-Clay is refused."""
    import ctypes as C
    s = scene(None, "cc")
    s.useAdmm(admm_max_iterations=4)
    assert s.lib.substep(s.ctx, 1e-3, C.byref(s.solver()), None) == abi.UNSUPPORTED


def test_admm_sand_matches_oracle_fp64(cuda_lib, oracle):
    """ADMM substeps of Drucker-Prager sand (StvkWithHencky + DruckerPragerStvkHencky
    F-step with projectSigmaAndDerivative, initOmega with projectSigma)."""
    sims = [scene(None, "dp"), scene(oracle, "dp")]
    for s in sims:
        s.useAdmm(admm_max_iterations=10, rho_scale=0.8, global_tolerance=1e-12)
    for _ in range(4):
        for k, s in enumerate(sims):
            rc = s.advanceOneTimeStep(1e-3)
            assert rc == abi.OK, (k, rc, s.last_stats)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-10
    assert rel(pg["V"], po["V"]) < 1e-6
    assert rel(pg["F"], po["F"]) < 1e-8
    np.testing.assert_allclose(sims[0].getLogJp(), sims[1].getLogJp(), rtol=1e-7, atol=1e-10)
