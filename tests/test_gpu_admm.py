"""ADMM substeps (AdmmSimulation, Projects/admm/AdmmSimulationFoam.h) and the
viscoelastic strain of the CUDA library against the oracle on the same seeded
scenes.  The oracle assembles the reference's 125-entry stencil; the library
applies the same operator matrix-free, so results agree to the solver
tolerances, not bit for bit."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import jittered_box

pytestmark = pytest.mark.gpu

DX = 1.0 / 64


def slab(lib, precision="fp64", visco=False, plastic=None, iters=20, E=2e4, nu=0.4, seed=3, grid_log2=None):
    kw = {"grid_log2": grid_log2} if grid_log2 else {}
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, lib=lib, **kw)
    x = jittered_box((12, 4, 12), DX, (0.3, 0.55, 0.3), 8, seed)
    V0 = DX ** 3 / 8
    h = s.addParticles(x, np.tile([0.0, -1.0, 0.0], (len(x), 1)), 1000 * V0, V0)
    model = mpm.StvkWithHenckyIsotropic(E, nu)
    h.addFBasedMpmForce(model)
    if plastic:
        h.addPlasticity(model, mpm.VonMisesStvkHencky(plastic))
    if visco:
        mu = E / (2 * (1 + nu))
        nv = 2 * mu * 0.05
        h.addFElasticNonequilibratedBasedMpmForce(mpm.StvkWithHencky(E, nu), nv, nv)
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.Sphere((0.5, 0.35, 0.5), 0.2), abi.STICKY))
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    s.useAdmm(admm_max_iterations=iters, rho_scale=0.8, global_tolerance=1e-12)
    return s


def run(sims, steps, dt=2e-3):
    for _ in range(steps):
        for k, s in enumerate(sims):
            rc = s.advanceOneTimeStep(dt)
            assert rc == abi.OK, (k, rc, s.last_stats)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("visco,plastic", [(False, None), (True, None), (False, 150.0)])
def test_admm_matches_oracle_fp64(cuda_lib, oracle, visco, plastic):
    sims = [slab(None, visco=visco, plastic=plastic, grid_log2=8), slab(oracle, visco=visco, plastic=plastic)]
    run(sims, 4)
    sg, so = sims[0].last_stats, sims[1].last_stats
    assert sg["newton_iterations"] == so["newton_iterations"] == 20
    assert sg["num_nodes"] == so["num_nodes"]
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-10
    assert rel(pg["V"], po["V"]) < 1e-6
    assert rel(pg["F"], po["F"]) < 1e-8
    if visco:
        Fg, Fo = sims[0].getViscoelasticStrain(), sims[1].getViscoelasticStrain()
        assert np.abs(Fo - np.eye(3)).max() > 1e-3
        assert rel(Fg, Fo) < 1e-8


def test_admm_mixed_precision_tracks_fp64_oracle(cuda_lib, oracle):
    """MIXED: FP32 operator coefficients and products in the global MINRES,
    FP64 local solves, state and reductions."""
    sims = [slab(None, precision="mixed", visco=True, grid_log2=8), slab(oracle, visco=True)]
    for s in sims:
        s.global_tolerance = 1e-9
    run(sims, 4)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-7
    assert rel(pg["V"], po["V"]) < 1e-3


def test_admm_state_persists_across_particle_reordering(cuda_lib, oracle):
    """y, omega and last_dv are per-particle state that the binning permutation
    must carry: a falling slab reorders particles every substep."""
    sims = [slab(None, grid_log2=8, iters=8), slab(oracle, iters=8)]
    run(sims, 6, dt=4e-3)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-9
    assert rel(pg["V"], po["V"]) < 1e-5


def test_newton_refuses_viscoelastic_particles(cuda_lib):
    s = slab(None, visco=True, grid_log2=8)
    s.integrator = abi.NEWTON
    import ctypes as C
    st = abi.Stats()
    assert s.lib.substep(s.ctx, 2e-3, C.byref(s.solver()), C.byref(st)) == abi.BAD_ARG
