"""Symplectic (explicit) substeps of the CUDA library against the oracle
(MpmSimulationBase::advanceOneTimeStep with symplectic = true,
MpmSimulationBase.cpp:264-281): particle stress, P2G of mass, momentum and
force, the explicit grid update with collisions at t, trial collision against
the colliders at t + dt, G2P.  FP64 runs differ from the oracle only by the
summation order of the scatters."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene

pytestmark = pytest.mark.gpu

DX = 1.0 / 64
GROUND = 7 * DX - 1e-3  # just below a grid plane, so trial collision acts


def scene(lib, kind="fcr", precision="fp64", plastic=None, visco=False, damage=False, trial=True, v0=(0.3, -2.0, 0.2),
          gravity=(0, -9.8, 0), ground=True, sphere=True, seed=5, mls=False):
    kw = {"grid_log2": 8} if lib is None else {}
    s = mpm.MpmSimulation(DX, gravity=gravity, precision=precision, lib=lib, **kw)
    h, x = build_scene(s, kind=kind, n=6, dx=DX, v0=v0, plastic=plastic, ground=GROUND if ground else None,
                       seed=seed, lo=(0.375, 8 * DX, 0.375))
    if damage:
        n = x.shape[0]
        F = np.zeros((n, 3, 3))
        F[:, 0, 0] = 1.0 + 0.2 * (x[:, 0] - x[:, 0].min()) / np.ptp(x[:, 0])
        F[:, 1, 1] = F[:, 2, 2] = 1.0
        s.setParticles(F=F)
        h.addRankineDamage(2000.0, residual_phase=0.01)
    if visco:
        E, nu = 1e4, 0.3
        nv = 2 * E / (2 * (1 + nu)) * 0.05
        h.addFElasticNonequilibratedBasedMpmForce(mpm.StvkWithHencky(E, nu), nv, nv)
    if sphere:
        # a sphere moving into the cube from the side: colliders at t and t + dt differ
        c = mpm.AnalyticCollisionObject(mpm.Sphere((0, 0, 0), 0.06), abi.SLIP, friction=0.2)
        c.setTranslation((0.375 - 0.07, 0.2, 0.42), (1.5, 0.0, 0.0))
        s.addCollisionObject(c)
    s.useExplicit(trial_collision=trial, mls_mpm=mls)
    return s


def run(sims, steps, dt=4e-4):
    for _ in range(steps):
        for k, s in enumerate(sims):
            rc = s.advanceOneTimeStep(dt)
            assert rc == abi.OK, (k, rc, s.last_stats)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("kind,plastic,visco,damage", [
    ("fcr", None, False, False),
    ("nh", None, False, True),
    ("hencky", 150.0, False, False),
    ("hencky", None, True, False),
])
@pytest.mark.parametrize("trial", [True, False])
def test_explicit_matches_oracle_fp64(cuda_lib, oracle, kind, plastic, visco, damage, trial):
    sims = [scene(None, kind, plastic=plastic, visco=visco, damage=damage, trial=trial),
            scene(oracle, kind, plastic=plastic, visco=visco, damage=damage, trial=trial)]
    for _ in range(12):
        run(sims, 1)
        sg, so = sims[0].last_stats, sims[1].last_stats
        assert sg["num_nodes"] == so["num_nodes"] and sg["num_blocks"] == so["num_blocks"]
        assert sg["num_groups"] == so["num_groups"]
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-12
    assert rel(pg["V"], po["V"]) < 1e-9
    assert rel(pg["F"], po["F"]) < 1e-10
    assert rel(pg["C"], po["C"]) < 1e-8
    if plastic:
        yg, _ = sims[0].getPlasticState()
        yo, _ = sims[1].getPlasticState()
        np.testing.assert_allclose(yg, yo, rtol=1e-9)
    if visco:
        Fg, Fo = sims[0].getViscoelasticStrain(), sims[1].getViscoelasticStrain()
        assert np.abs(Fo - np.eye(3)).max() > 1e-4
        assert rel(Fg, Fo) < 1e-10
    if damage:
        cg, co = sims[0].getDamage(), sims[1].getDamage()
        assert (co < 1).sum() > 0
        np.testing.assert_allclose(cg, co, rtol=1e-9, atol=0)


@pytest.mark.parametrize("kind,plastic,visco", [("fcr", None, False), ("hencky", 150.0, False), ("hencky", None, True)])
def test_mls_matches_oracle_fp64(cuda_lib, oracle, kind, plastic, visco):
    """MLS-MPM force weight (S_p (x_i - x_p)) w_ip D^-1 and G2P gradV = C."""
    sims = [scene(None, kind, plastic=plastic, visco=visco, mls=True), scene(oracle, kind, plastic=plastic, visco=visco, mls=True)]
    run(sims, 12)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-12
    assert rel(pg["V"], po["V"]) < 1e-9
    assert rel(pg["F"], po["F"]) < 1e-10
    assert rel(pg["C"], po["C"]) < 1e-8
    if visco:
        assert rel(sims[0].getViscoelasticStrain(), sims[1].getViscoelasticStrain()) < 1e-10


def test_mls_mixed_and_refused_by_newton(cuda_lib, oracle):
    sims = [scene(None, "fcr", precision="mixed", mls=True), scene(oracle, "fcr", mls=True)]
    run(sims, 12)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-7
    assert rel(pg["V"], po["V"]) < 1e-4
    import ctypes as C
    g = sims[0]
    g.integrator = abi.NEWTON
    assert g.lib.substep(g.ctx, 4e-4, C.byref(g.solver()), None) == abi.BAD_ARG


def test_explicit_mixed_tracks_fp64_oracle(cuda_lib, oracle):
    """MIXED: FP32 constitutive stress and transfers; FP64 positions and grid sums."""
    sims = [scene(None, "fcr", precision="mixed"), scene(oracle, "fcr")]
    run(sims, 12)
    pg, po = sims[0].getParticles(), sims[1].getParticles()
    assert rel(pg["X"], po["X"]) < 1e-7
    assert rel(pg["V"], po["V"]) < 1e-4
    assert rel(pg["F"], po["F"]) < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_explicit_free_fall_is_exact(cuda_lib, precision):
    s = scene(None, precision=precision, ground=False, sphere=False)
    v0 = s.getParticles()["V"].copy()
    dt = 1e-3
    run([s], 10, dt)
    p = s.getParticles()
    # FP64: exact up to round-off.  MIXED: the FP32 constitutive step at F = I
    # leaves stress round-off of order mu * 1e-7, and the FP32 transfers round
    # the velocity to FP32 (relative 1e-7 of |v| ~ 0.1 m/s per substep)
    atol = 1e-12 if precision == "fp64" else 1e-5
    np.testing.assert_allclose(p["V"], v0 + 10 * dt * np.array([0, -9.8, 0]), rtol=0, atol=atol)
    np.testing.assert_allclose(p["C"], 0, atol=1e-9 if precision == "fp64" else 1e-3)


def test_explicit_conserves_momentum(cuda_lib):
    s = scene(None, gravity=(0, 0, 0), v0=(0, 0, 0), ground=False, sphere=False)
    V = np.random.default_rng(4).normal(0, 0.2, s.getParticles()["V"].shape)
    s.setParticles(V=V)
    mom0 = V.sum(0)
    run([s], 10, 2e-4)
    p = s.getParticles()
    assert np.abs(p["F"].reshape(-1, 3, 3) - np.eye(3)).max() > 1e-4
    assert np.abs(p["V"].sum(0) - mom0).max() < 1e-12 * np.abs(V).sum()


def test_explicit_cfl_status(cuda_lib, oracle):
    """A particle moving more than a cell per substep is reported by both."""
    sims = [scene(None, v0=(0, -40.0, 0), ground=False, sphere=False), scene(oracle, v0=(0, -40.0, 0), ground=False, sphere=False)]
    rcs = [s.advanceOneTimeStep(1e-3) for s in sims]
    assert rcs[0] == rcs[1] == abi.CFL_VIOLATION
