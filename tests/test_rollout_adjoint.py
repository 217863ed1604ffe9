"""Differentiable rollout (checkpointed reverse sweep of the implicit substep)
on the oracle: gradients of a centre-of-mass loss with respect to per-particle
Young's modulus and initial velocity against central finite differences, the
checkpoint interval does not change them, and the torch.autograd wrapper
reproduces them."""
import numpy as np
import pytest
import torch

from ziran2019_b200 import abi, mpm
from ziran2019_b200.rollout import DifferentiableRollout, Rollout
from tests.scenes import jittered_box

DX = 1.0 / 64
NU = 0.3


def scene(lib, n=3, seed=5, precision="fp64", grid_log2=None):
    kw = {"grid_log2": grid_log2} if grid_log2 else {}
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, lib=lib, **kw)
    x = jittered_box(n, DX, (0.4, 0.11, 0.4), 8, seed)
    V0 = DX ** 3 / 8
    h = s.addParticles(x, np.zeros_like(x), 1000 * V0, V0)
    h.addFBasedMpmForce(mpm.FixedCorotated(1e4, NU))
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    s.switchLinearSolver(abi.CG)
    s.newton_tolerance = 1e-13
    s.newton_max_iterations = 60
    s.krylov_max_iterations = 2000
    s.krylov_tolerance = 1e-30
    rng = np.random.default_rng(seed + 1)
    E = 1e4 * np.exp(0.3 * rng.standard_normal(len(x)) - 0.045)
    v0 = rng.uniform(-0.5, 0.5, x.shape)
    return s, E, v0, np.full(len(x), 1000 * V0)


def com_loss(X, m, target):
    com = (m[:, None] * X).sum(0) / m.sum()
    return float(((com - target) ** 2).sum()), 2 * (com - target)[None, :] * (m / m.sum())[:, None]


def test_rollout_gradients_match_finite_differences(oracle):
    s, E, v0, m = scene(oracle)
    target = np.array([0.5, 0.2, 0.45])
    ro = Rollout(s, NU, 1e-3, 12, checkpoint_every=5)
    X = ro.run(E, v0)
    L, gX = com_loss(X, m, target)
    gE, gv = ro.backward(gX)
    assert len(ro.stats) == 12
    rng = np.random.default_rng(9)
    for which, h in (("E", 10.0), ("v", 1e-5)):
        for _ in range(3):
            d = rng.standard_normal(E.shape if which == "E" else v0.shape)
            Ep, vp = (E + h * d, v0) if which == "E" else (E, v0 + h * d)
            Em, vm = (E - h * d, v0) if which == "E" else (E, v0 - h * d)
            fd = (com_loss(ro.run(Ep, vp), m, target)[0] - com_loss(ro.run(Em, vm), m, target)[0]) / (2 * h)
            an = float(((gE if which == "E" else gv) * d).sum())
            assert abs(fd - an) <= 1e-5 * abs(an) + 1e-14, (which, fd, an)


def test_checkpoint_interval_does_not_change_gradients(oracle):
    out = []
    for every in (1, 4, 12):
        s, E, v0, m = scene(oracle)
        ro = Rollout(s, NU, 1e-3, 12, checkpoint_every=every)
        X = ro.run(E, v0)
        _, gX = com_loss(X, m, np.array([0.5, 0.2, 0.45]))
        out.append(ro.backward(gX))
    for gE, gv in out[1:]:
        np.testing.assert_allclose(gE, out[0][0], rtol=1e-12, atol=0)
        np.testing.assert_allclose(gv, out[0][1], rtol=1e-12, atol=0)


def test_torch_autograd_wrapper(oracle):
    s, E, v0, m = scene(oracle)
    target = torch.tensor([0.5, 0.2, 0.45], dtype=torch.float64)
    ro = Rollout(s, NU, 1e-3, 6, checkpoint_every=3)
    Et = torch.tensor(E, requires_grad=True)
    vt = torch.tensor(v0, requires_grad=True)
    X = DifferentiableRollout.apply(Et, vt, ro)
    mt = torch.tensor(m)
    com = (mt[:, None] * X).sum(0) / mt.sum()
    loss = ((com - target) ** 2).sum()
    loss.backward()
    _, gX = com_loss(X.detach().numpy(), m, target.numpy())
    gE, gv = ro.backward(gX)
    np.testing.assert_allclose(Et.grad.numpy(), gE, rtol=1e-10)
    np.testing.assert_allclose(vt.grad.numpy(), gv, rtol=1e-10)


def test_torch_wrapper_refuses_stale_backward(oracle):
    """Two forward calls before a backward: the first call's backward raises
    (the checkpoints hold the second call's states); the second one's gradient
    keeps the shape of its input (a flat v0 stays flat)."""
    s, E, v0, m = scene(oracle, n=2)
    ro = Rollout(s, NU, 1e-3, 2, checkpoint_every=1)
    Et = torch.tensor(E, requires_grad=True)
    vt = torch.tensor(v0.reshape(-1), requires_grad=True)
    X1 = DifferentiableRollout.apply(Et, vt, ro)
    X2 = DifferentiableRollout.apply(Et, vt, ro)
    with pytest.raises(RuntimeError, match="ran forward again"):
        X1.sum().backward()
    X2.sum().backward()
    assert vt.grad.shape == vt.shape and Et.grad.shape == Et.shape


def plastic_scene(lib, n=3, seed=5, precision="fp64", yield_stress=40.0):
    """A sheared StvkWithHenckyIsotropic block with a low von Mises yield stress
    (xi = 0), so that many particles are projected every substep."""
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, lib=lib)
    x = jittered_box(n, DX, (0.4, 0.11, 0.4), 8, seed)
    V0 = DX ** 3 / 8
    h = s.addParticles(x, np.zeros_like(x), 1000 * V0, V0)
    model = mpm.StvkWithHenckyIsotropic(1e4, NU)
    h.addFBasedMpmForce(model)
    h.addPlasticity(model, mpm.VonMisesStvkHencky(yield_stress, 1e30, 0.0))
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    s.switchLinearSolver(abi.CG)
    s.newton_tolerance = 1e-13
    s.newton_max_iterations = 60
    s.krylov_max_iterations = 2000
    s.krylov_tolerance = 1e-30
    rng = np.random.default_rng(seed + 1)
    E = 1e4 * np.exp(0.3 * rng.standard_normal(len(x)) - 0.045)
    v0 = rng.uniform(-0.8, 0.8, x.shape)
    return s, E, v0, np.full(len(x), 1000 * V0)


def test_rollout_gradients_through_von_mises_match_finite_differences(oracle):
    """The adjoint of the von Mises return map (VonMisesStvkHencky::projectStrain,
    PlasticityApplier.cpp:462-502, xi = 0) in a rollout whose particles yield:
    gradients with respect to E (which also sets the yield radius tau_Y / 2 mu)
    and v0 against central differences.  The map has a kink on the yield
    surface; the steps are small enough that no particle crosses it."""
    s, E, v0, m = plastic_scene(oracle)
    target = np.array([0.5, 0.2, 0.45])
    ro = Rollout(s, NU, 1e-3, 6, checkpoint_every=3)
    X = ro.run(E, v0)
    assert s.getPlasticState()[0].shape[0] == len(E)
    L, gX = com_loss(X, m, target)
    gE, gv = ro.backward(gX)
    rng = np.random.default_rng(21)
    for which, h in (("E", 1.0), ("v", 1e-6)):
        for _ in range(3):
            d = rng.standard_normal(E.shape if which == "E" else v0.shape)
            Ep, vp = (E + h * d, v0) if which == "E" else (E, v0 + h * d)
            Em, vm = (E - h * d, v0) if which == "E" else (E, v0 - h * d)
            fd = (com_loss(ro.run(Ep, vp), m, target)[0] - com_loss(ro.run(Em, vm), m, target)[0]) / (2 * h)
            an = float(((gE if which == "E" else gv) * d).sum())
            assert abs(fd - an) <= 1e-5 * abs(an) + 1e-14, (which, fd, an)


def test_von_mises_rollout_projects_particles(oracle):
    """The plastic scene above does yield: most particles end on the yield
    surface (projected in the last substep), and the same rollout without the
    return map ends elsewhere."""
    s, E, v0, m = plastic_scene(oracle)
    X = Rollout(s, NU, 1e-3, 6, checkpoint_every=3).run(E, v0)
    sv = np.linalg.svd(s.getParticles()["F"], compute_uv=False)
    dev = np.log(sv) - np.log(sv).mean(1, keepdims=True)
    mu = E / (2 * (1 + NU))
    assert (np.linalg.norm(dev, axis=1) >= 40.0 / (2 * mu) * (1 - 1e-9)).sum() > len(E) // 2
    e, _, _, _ = plastic_scene(oracle, yield_stress=1e30)
    Xe = Rollout(e, NU, 1e-3, 6, checkpoint_every=3).run(E, v0)
    assert np.abs(X - Xe).max() > 1e-5
