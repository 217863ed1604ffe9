"""Reverse mode of the implicit substep on the GPU: against the oracle's
adjoint (same math, FP64, CPU) and against central finite differences of the
GPU's own forward substep."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import jittered_box

pytestmark = pytest.mark.gpu

DX = 1.0 / 64


def cube(lib, kind="fcr", precision="fp64", n=5, seed=0, E=1e4, nu=0.3):
    kw = {} if lib is not None and lib is not False else {"grid_log2": 8}
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, lib=lib or None, **kw)
    x = jittered_box(n, DX, (0.4, 0.105, 0.4), 8, seed)
    V0 = DX ** 3 / 8
    rng = np.random.default_rng(seed + 1)
    h = s.addParticles(x, rng.uniform(-0.5, 0.5, x.shape), 1000 * V0, V0)
    model = {"fcr": mpm.FixedCorotated, "nh": mpm.NeoHookeanBorden, "hencky": mpm.StvkWithHenckyIsotropic}[kind](E, nu)
    h.addFBasedMpmForce(model)
    Ep = E * np.exp(0.3 * rng.standard_normal(len(x)))
    s.setYoungsModulus(Ep, nu)
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    s.switchLinearSolver(abi.CG)
    s.newton_tolerance = 1e-13 if precision == "fp64" else 1e-7
    s.newton_max_iterations = 60
    s.krylov_max_iterations = 2000
    s.krylov_tolerance = 1e-30
    for _ in range(3):
        assert s.advanceOneTimeStep(1e-3) == abi.OK
    return s, Ep, nu


def upstream(P, seed=7):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((P, 3)), rng.standard_normal((P, 3)), rng.standard_normal((P, 3, 3)), rng.standard_normal((P, 3, 3))]


def adjoint(s, ups, tol=1e-12):
    g = [u.copy() for u in ups] + [np.zeros(s.count)]
    rc = s.adjointSubstep(1e-3, *g, tolerance=tol)
    assert rc == abi.OK, (rc, s.last_stats)
    return g


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("kind", ["fcr", "nh", "hencky"])
def test_adjoint_substep_matches_oracle(cuda_lib, oracle, kind):
    sg, _, _ = cube(False, kind)
    so, _, _ = cube(oracle, kind)
    ups = upstream(sg.count)
    gg, go = adjoint(sg, ups), adjoint(so, ups)
    for a, b, name in zip(gg, go, ("x", "v", "C", "F", "E")):
        assert rel(a, b) < 1e-7, name
    # the adjoint call also advanced the state like a forward substep
    assert rel(sg.getParticles()["X"], so.getParticles()["X"]) < 1e-11


def test_adjoint_substep_matches_finite_differences(cuda_lib):
    s, Ep, nu = cube(False, "fcr")
    P = s.count
    s.checkpointSave(0)
    st0 = s.getParticles()
    ups = upstream(P)
    g = adjoint(s, ups)

    def loss_from(X, V, C, F, E):
        s.checkpointLoad(0)
        s.setParticles(X=X, V=V, C=C, F=F)
        s.setYoungsModulus(E, nu)
        assert s.advanceOneTimeStep(1e-3) == abi.OK
        p = s.getParticles()
        return sum((u * p[k]).sum() for u, k in zip(ups, ("X", "V", "C", "F")))

    base = dict(X=st0["X"], V=st0["V"], C=st0["C"], F=st0["F"], E=Ep)
    rng = np.random.default_rng(3)
    for key, grad, h in (("X", g[0], 1e-7 * DX), ("V", g[1], 1e-6), ("C", g[2], 1e-5), ("F", g[3], 1e-6), ("E", g[4], 1e-1)):
        d = rng.standard_normal(base[key].shape)
        plus = dict(base, **{key: base[key] + h * d})
        minus = dict(base, **{key: base[key] - h * d})
        fd = (loss_from(**plus) - loss_from(**minus)) / (2 * h)
        an = float((grad * d).sum())
        assert abs(fd - an) <= 1e-5 * abs(an) + 1e-9, (key, fd, an)


def test_mixed_precision_adjoint_tracks_fp64(cuda_lib):
    """FP32 Hessian products inside FP64 adjoint CG vectors: the mixed
    context's gradients agree with the FP64 context's to the FP32 operator's
    accuracy."""
    s64, _, _ = cube(False, "fcr")
    smx, _, _ = cube(False, "fcr", precision="mixed")
    ups = upstream(s64.count)
    g64, gmx = adjoint(s64, ups), adjoint(smx, ups, tol=1e-8)
    for a, b, name in zip(gmx, g64, ("x", "v", "C", "F", "E")):
        assert rel(a, b) < 2e-3, name


def test_checkpoint_round_trip(cuda_lib):
    s, _, _ = cube(False, "fcr", n=3)
    s.checkpointSave(2)
    p0 = s.getParticles()
    t0 = s.time
    for _ in range(2):
        s.advanceOneTimeStep(1e-3)
    s.checkpointLoad(2)
    p1 = s.getParticles()
    assert s.time == t0
    for k in p0:
        np.testing.assert_array_equal(p0[k], p1[k])


def test_gpu_rollout_matches_oracle_rollout(cuda_lib, oracle):
    from ziran2019_b200.rollout import Rollout
    from tests.test_rollout_adjoint import NU, com_loss, scene
    target = np.array([0.5, 0.2, 0.45])
    out = []
    for lib, kw in ((None, {"grid_log2": 8}), (oracle, {})):
        s, E, v0, m = scene(lib, n=4, **kw)
        ro = Rollout(s, NU, 1e-3, 10, checkpoint_every=4)
        X = ro.run(E, v0)
        _, gX = com_loss(X, m, target)
        out.append((X,) + ro.backward(gX))
    assert rel(out[0][0], out[1][0]) < 1e-11
    assert rel(out[0][1], out[1][1]) < 1e-6
    assert rel(out[0][2], out[1][2]) < 1e-6


def test_gpu_rollout_finite_differences(cuda_lib):
    from ziran2019_b200.rollout import Rollout
    from tests.test_rollout_adjoint import NU, com_loss, scene
    s, E, v0, m = scene(None, n=4, grid_log2=8)
    target = np.array([0.5, 0.2, 0.45])
    ro = Rollout(s, NU, 1e-3, 10, checkpoint_every=5)
    _, gX = com_loss(ro.run(E, v0), m, target)
    gE, gv = ro.backward(gX)
    rng = np.random.default_rng(2)
    for which, h in (("E", 10.0), ("v", 1e-5)):
        d = rng.standard_normal(E.shape if which == "E" else v0.shape)
        args_p = (E + h * d, v0) if which == "E" else (E, v0 + h * d)
        args_m = (E - h * d, v0) if which == "E" else (E, v0 - h * d)
        fd = (com_loss(ro.run(*args_p), m, target)[0] - com_loss(ro.run(*args_m), m, target)[0]) / (2 * h)
        an = float(((gE if which == "E" else gv) * d).sum())
        assert abs(fd - an) <= 1e-5 * abs(an) + 1e-14, (which, fd, an)


def test_gpu_plastic_rollout_matches_oracle_and_finite_differences(cuda_lib, oracle):
    """The adjoint through the von Mises return map (xi = 0) on the GPU: a
    rollout whose particles yield, against the oracle's adjoint and against
    central differences of the GPU's own forward rollout."""
    from ziran2019_b200.rollout import Rollout
    from tests.test_rollout_adjoint import NU, com_loss, plastic_scene
    target = np.array([0.5, 0.2, 0.45])
    out = []
    for lib, kw in ((None, {}), (oracle, {})):
        s, E, v0, m = plastic_scene(lib, n=3)
        ro = Rollout(s, NU, 1e-3, 6, checkpoint_every=3)
        X = ro.run(E, v0)
        _, gX = com_loss(X, m, target)
        out.append((X,) + ro.backward(gX) + (ro, s, E, v0, m))
    assert rel(out[0][0], out[1][0]) < 1e-11
    assert rel(out[0][1], out[1][1]) < 1e-6
    assert rel(out[0][2], out[1][2]) < 1e-6
    _, gE, gv, ro, s, E, v0, m = out[0]
    rng = np.random.default_rng(4)
    for which, h in (("E", 1.0), ("v", 1e-6)):
        d = rng.standard_normal(E.shape if which == "E" else v0.shape)
        args_p = (E + h * d, v0) if which == "E" else (E, v0 + h * d)
        args_m = (E - h * d, v0) if which == "E" else (E, v0 - h * d)
        fd = (com_loss(ro.run(*args_p), m, target)[0] - com_loss(ro.run(*args_m), m, target)[0]) / (2 * h)
        an = float(((gE if which == "E" else gv) * d).sum())
        assert abs(fd - an) <= 1e-5 * abs(an) + 1e-14, (which, fd, an)


def test_torch_autograd_wrapper_over_cuda_library(cuda_lib):
    """DifferentiableRollout (the torch.autograd.Function over the C ABI) on
    the CUDA library: a loss written in torch backpropagates to E and v0, and
    the gradients equal the rollout's own reverse sweep and central
    differences of the forward."""
    import torch

    from ziran2019_b200.rollout import DifferentiableRollout, Rollout
    from tests.test_rollout_adjoint import NU, com_loss, scene
    s, E, v0, m = scene(None, n=4, grid_log2=8)
    ro = Rollout(s, NU, 1e-3, 8, checkpoint_every=4)
    dev = "cuda"
    Et = torch.tensor(E, device=dev, requires_grad=True)
    vt = torch.tensor(v0, device=dev, requires_grad=True)
    target = torch.tensor([0.5, 0.2, 0.45], dtype=torch.float64, device=dev)
    X = DifferentiableRollout.apply(Et, vt, ro)
    assert X.device.type == "cuda" and X.shape == (s.count, 3)
    mt = torch.tensor(m, device=dev)
    loss = (((mt[:, None] * X).sum(0) / mt.sum() - target) ** 2).sum()
    loss.backward()
    _, gX = com_loss(X.detach().cpu().numpy(), m, target.cpu().numpy())
    gE, gv = ro.backward(gX)
    np.testing.assert_allclose(Et.grad.cpu().numpy(), gE, rtol=1e-10)
    np.testing.assert_allclose(vt.grad.cpu().numpy(), gv, rtol=1e-10)
    rng = np.random.default_rng(8)
    d = rng.standard_normal(v0.shape)
    h = 1e-5
    fd = (com_loss(ro.run(E, v0 + h * d), m, target.cpu().numpy())[0] - com_loss(ro.run(E, v0 - h * d), m, target.cpu().numpy())[0]) / (2 * h)
    an = float((vt.grad.cpu().numpy() * d).sum())
    assert abs(fd - an) <= 1e-5 * abs(an) + 1e-14, (fd, an)
