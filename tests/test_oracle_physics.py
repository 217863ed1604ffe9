"""Analytic known-answer tests that pin the oracle's physics (the reference ships
no golden vectors for it): finite-difference consistency of psi -> P -> dP,
SVD reconstruction, return-map idempotence, transfer conservation, and the
Newton objective's residual / Hessian consistency (the DiffTest.h pattern)."""
import ctypes as C

import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene, jittered_box

P = lambda a: a.ctypes.data_as(abi.c_double_p)
MODELS = [abi.MODEL_NEOHOOKEAN_BORDEN, abi.MODEL_STVK_HENCKY_ISOTROPIC, abi.MODEL_FIXED_COROTATED]


def model_eval(oracle, kind, F, dF=None, E=1e4, nu=0.3):
    psi = C.c_double()
    Pm = np.zeros(9)
    dP = np.zeros(9)
    dFa = np.zeros(9) if dF is None else np.ascontiguousarray(dF, dtype=np.float64).ravel()
    oracle.dll.zoracle_model_eval(kind, E, nu, P(np.ascontiguousarray(F, dtype=np.float64).ravel()), P(dFa), C.byref(psi), P(Pm), P(dP))
    return psi.value, Pm.reshape(3, 3), dP.reshape(3, 3)


@pytest.mark.parametrize("kind", MODELS)
def test_first_piola_is_energy_gradient(oracle, kind):
    rng = np.random.default_rng(kind)
    for _ in range(30):
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if np.linalg.det(F) < 0.2:
            continue
        dF = rng.standard_normal((3, 3))
        h = 1e-6
        _, Pm, _ = model_eval(oracle, kind, F)
        fd = (model_eval(oracle, kind, F + h * dF)[0] - model_eval(oracle, kind, F - h * dF)[0]) / (2 * h)
        assert abs(fd - (Pm * dF).sum()) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("kind", MODELS)
def test_piola_differential_matches_fd(oracle, kind):
    rng = np.random.default_rng(10 + kind)
    for _ in range(30):
        F = np.eye(3) + 0.3 * rng.standard_normal((3, 3))
        if np.linalg.det(F) < 0.2:
            continue
        dF = rng.standard_normal((3, 3))
        h = 1e-6
        _, _, dP = model_eval(oracle, kind, F, dF)
        fd = (model_eval(oracle, kind, F + h * dF)[1] - model_eval(oracle, kind, F - h * dF)[1]) / (2 * h)
        assert np.abs(fd - dP).max() <= 1e-6 * max(1.0, np.abs(dP).max())


def test_rest_state_is_stress_free(oracle):
    for kind in MODELS:
        psi, Pm, _ = model_eval(oracle, kind, np.eye(3))
        assert abs(psi) < 1e-9 and np.abs(Pm).max() < 1e-9


@pytest.mark.parametrize("fp32", [0, 1])
def test_svd_reconstruction(oracle, fp32):
    rng = np.random.default_rng(3 + fp32)
    tol = 1e-12 if fp32 == 0 else 5e-5
    for t in range(1000):
        F = rng.standard_normal((3, 3))
        if t % 4 == 0:  # near-degenerate and repeated singular values
            F = np.diag(rng.choice([1.0, 1.0, 0.5, 1e-8], 3)) + 1e-10 * rng.standard_normal((3, 3))
        U, s, V = np.zeros(9), np.zeros(3), np.zeros(9)
        oracle.dll.zoracle_svd3(P(np.ascontiguousarray(F.ravel())), P(U), P(s), P(V), fp32)
        U, V = U.reshape(3, 3), V.reshape(3, 3)
        scale = max(1.0, np.abs(F).max())
        assert np.abs(U @ np.diag(s) @ V.T - F).max() <= tol * scale
        assert np.abs(U.T @ U - np.eye(3)).max() <= tol * 10 and np.abs(V.T @ V - np.eye(3)).max() <= tol * 10
        assert abs(np.linalg.det(U) - 1) < 1e-4 and abs(np.linalg.det(V) - 1) < 1e-4
        assert abs(s[0]) + 1e-12 >= abs(s[1]) and abs(s[1]) + 1e-12 >= abs(s[2]) and s[0] >= 0 and s[1] >= 0


def test_von_mises_return_map_is_idempotent(oracle):
    rng = np.random.default_rng(5)
    E, nu, ys = 5e4, 0.35, 150.0
    for _ in range(50):
        F = np.eye(3) + 0.05 * rng.standard_normal((3, 3))
        F1 = np.ascontiguousarray(F.ravel())
        out = C.c_double()
        oracle.dll.zoracle_von_mises(abi.MODEL_STVK_HENCKY_ISOTROPIC, E, nu, ys, 0.0, P(F1), C.byref(out))
        F2 = F1.copy()
        oracle.dll.zoracle_von_mises(abi.MODEL_STVK_HENCKY_ISOTROPIC, E, nu, ys, 0.0, P(F2), C.byref(out))
        np.testing.assert_allclose(F2, F1, atol=1e-12)
        # projected state lies on or inside the yield surface: |dev(log sigma)| <= ys / (2 mu)
        s = np.linalg.svd(F1.reshape(3, 3), compute_uv=False)
        eps = np.log(np.maximum(s, 1e-4))
        mu = E / (2 * (1 + nu))
        assert np.linalg.norm(eps - eps.mean()) <= ys / (2 * mu) * (1 + 1e-9)


def test_p2g_conserves_mass_and_momentum(oracle):
    dx = 1.0 / 64
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), lib=oracle)
    x = jittered_box(6, dx, (0.4, 0.4, 0.4), 8, seed=4)
    rng = np.random.default_rng(4)
    v = rng.standard_normal(x.shape)
    m = rng.uniform(0.5, 1.5, x.shape[0])
    sim.addParticles(x, v, m, 1e-6)
    Cm = 0.1 * rng.standard_normal((x.shape[0], 3, 3))
    sim.setParticles(C=Cm)
    sim.beginImplicit(1e-3)
    gm, gv, coord = sim.getGrid()
    assert abs(gm.sum() - m.sum()) <= 1e-12 * m.sum()
    # APIC P2G conserves linear momentum: sum_i m_i v_i = sum_p m_p v_p
    np.testing.assert_allclose((gm[:, None] * gv).sum(0), (m[:, None] * v).sum(0), rtol=1e-11, atol=1e-11)


@pytest.mark.parametrize("kind", ["fcr", "nh", "hencky"])
def test_newton_objective_diff_test(oracle, kind):
    """Residual differences match the Hessian product (DiffTest.h:19-138)."""
    dx = 1.0 / 64
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), lib=oracle)
    build_scene(sim, kind=kind, n=5, dx=dx, ground=None)
    rng = np.random.default_rng(1)
    F = np.eye(3) + 0.1 * rng.standard_normal((sim.count, 3, 3))
    sim.setParticles(F=F)
    N = sim.beginImplicit(1e-3)
    dv0 = 0.01 * rng.standard_normal((N, 3))
    d = rng.standard_normal((N, 3))
    r0, _ = sim.residual(dv0)
    Hd = sim.multiply(d)
    h = 1e-5
    rp, _ = sim.residual(dv0 + h * d)
    rm, _ = sim.residual(dv0 - h * d)
    fd = -(rp - rm) / (2 * h)  # r = -grad E, so dr = -H d
    assert np.abs(fd - Hd).max() <= 1e-5 * np.abs(Hd).max()


def test_newton_converges_on_colliding_cube(oracle):
    dx = 1.0 / 64
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), lib=oracle)
    build_scene(sim, kind="fcr", n=6, dx=dx)
    sim.newton_tolerance = 1e-8
    sim.newton_max_iterations = 20
    sim.switchLinearSolver(abi.CG)
    sim.krylov_max_iterations = 100
    for _ in range(3):
        rc = sim.advanceOneTimeStep(1e-3)
        assert rc == abi.OK
        assert sim.last_stats["newton_converged"] == 1
        assert sim.last_stats["num_collision_nodes"] > 0


def _nh_uniaxial_cauchy_max(s, E, nu):
    """Largest principal Cauchy stress of NeoHookeanBorden (g = 1) under F = R diag(s, 1, 1):
    tau = mu J^(-2/3) dev(F F^T) + J kappa/2 (J - 1/J) I (NeoHookeanBorden.cpp:67-83)."""
    mu = E / (2 * (1 + nu))
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    kappa = 0.666666 * mu + lam
    J = s
    dev = np.array([s * s, 1.0, 1.0]) - (s * s + 2) / 3
    tau = mu * J ** (-2.0 / 3.0) * dev + J * kappa / 2 * (J - 1 / J)
    return (tau / J).max()


def test_rankine_damage_known_answer(oracle):
    """Naive Rankine damage (FractureSimulation.h:509-554): after P2G each
    NeoHookeanBorden particle takes c = min(c, sigma_F / sigma_max) once its
    largest principal Cauchy stress passes sigma_F, and g = c^2 (1 - k) + k.
    Particles of another model are untouched."""
    E, nu, dx = 1e4, 0.3, 1.0 / 64
    sim = mpm.MpmSimulation(dx, gravity=(0, 0, 0), precision="fp64", lib=oracle)
    x = jittered_box(4, dx, (0.4, 0.4, 0.4), 8, seed=3)
    n = x.shape[0]
    h_nh = sim.addParticles(x[: n // 2], np.zeros((n // 2, 3)), 1e-3, dx ** 3 / 8)
    h_hk = sim.addParticles(x[n // 2:], np.zeros((n - n // 2, 3)), 1e-3, dx ** 3 / 8)
    h_nh.addFBasedMpmForce(mpm.NeoHookeanBorden(E, nu))
    h_hk.addFBasedMpmForce(mpm.StvkWithHenckyIsotropic(E, nu))
    rng = np.random.default_rng(5)
    stretch = rng.uniform(0.9, 1.3, n)
    F = np.empty((n, 3, 3))
    for i in range(n):
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        F[i] = q @ np.diag([stretch[i], 1.0, 1.0]) @ q.T
    sim.setParticles(F=F)
    smax = np.array([_nh_uniaxial_cauchy_max(s, E, nu) for s in stretch])
    sigma_f = float(np.median(smax[: n // 2]))
    h_nh.addRankineDamage(sigma_f, residual_phase=0.001)
    h_hk.addRankineDamage(sigma_f, residual_phase=0.001)
    assert np.all(sim.getDamage() == 1.0)
    assert sim.advanceOneTimeStep(1e-4) == abi.OK
    c = sim.getDamage()
    want = np.where(smax > sigma_f, np.minimum(1.0, sigma_f / smax), 1.0)
    np.testing.assert_allclose(c[: n // 2], want[: n // 2], rtol=1e-12)
    assert (c[: n // 2] < 1).sum() > n // 8
    assert np.all(c[n // 2:] == 1.0)


def _eigen_first(oracle, A):
    import ctypes as C
    f = oracle.dll.zoracle_eigen_first_eigenvalue
    f.restype = C.c_double
    f.argtypes = [C.POINTER(C.c_double)]
    A = np.ascontiguousarray(A, dtype=np.float64)
    return f(A.ctypes.data_as(C.POINTER(C.c_double)))


def test_eigen_first_eigenvalue_known_answers(oracle):
    """The reference's Rankine sigma_max is cauchy.eigenvalues()[0].real() of
    Eigen's general eigensolver (FractureSimulation.h:539-543): the first entry
    of the real Schur form.  Known answers of that order: a diagonal matrix is
    already in Schur form (first = a_00, not the largest); a symmetric 2x2
    block [[a, b], [b, d]] over a decoupled third row deflates at the bottom
    and rotates the block so that each diagonal entry keeps its nearer
    eigenvalue (a < d: the smaller one first); a rotation block gives the real
    part of its complex pair; any symmetric matrix gives one of its
    eigenvalues."""
    assert _eigen_first(oracle, np.diag([1.0, 5.0, 3.0])) == 1.0
    assert _eigen_first(oracle, np.diag([7.0, -2.0, 3.0])) == 7.0
    a, b, d = 1.0, 1.0, 2.0
    lam_minus = 0.5 * (a + d) - np.sqrt(0.25 * (a - d) ** 2 + b * b)
    lam_plus = 0.5 * (a + d) + np.sqrt(0.25 * (a - d) ** 2 + b * b)
    A = np.array([[a, b, 0.0], [b, d, 0.0], [0.0, 0.0, 10.0]])
    assert abs(_eigen_first(oracle, A) - lam_minus) < 1e-14
    A = np.array([[d, b, 0.0], [b, a, 0.0], [0.0, 0.0, 10.0]])
    assert abs(_eigen_first(oracle, A) - lam_plus) < 1e-14
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 2.0]])
    assert abs(_eigen_first(oracle, R)) < 1e-15
    rng = np.random.default_rng(0)
    first_is_max = 0
    for _ in range(2000):
        M = rng.standard_normal((3, 3))
        A = M + M.T
        e = np.linalg.eigvalsh(A)
        v = _eigen_first(oracle, A)
        assert np.min(np.abs(e - v)) < 1e-12 * np.abs(e).max()
        first_is_max += abs(v - e.max()) < 1e-12 * np.abs(e).max()
    # the first eigenvalue is the largest in only part of the cases
    assert 200 < first_is_max < 1800


def test_rankine_reference_order_known_answer(oracle):
    """With the reference's order a stretch along y (diagonal Cauchy stress)
    takes sigma_xx, the first diagonal entry, as sigma_max: the particles damage
    only where sigma_xx passes sigma_F, whereas the largest-eigenvalue rule
    damages where sigma_yy does."""
    E, nu, dx = 1e4, 0.3, 1.0 / 64
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    kappa = 0.666666 * mu + lam
    x = jittered_box(4, dx, (0.4, 0.4, 0.4), 8, seed=3)
    n = x.shape[0]
    stretch = np.random.default_rng(5).uniform(0.8, 1.3, n)
    J = stretch
    sxx = (mu * J ** (-2.0 / 3.0) * (1.0 - (stretch ** 2 + 2) / 3) + J * kappa / 2 * (J - 1 / J)) / J
    syy = (mu * J ** (-2.0 / 3.0) * (stretch ** 2 - (stretch ** 2 + 2) / 3) + J * kappa / 2 * (J - 1 / J)) / J
    sigma_f = float(np.median(np.abs(sxx)))
    out = {}
    for ref in (False, True):
        sim = mpm.MpmSimulation(dx, gravity=(0, 0, 0), precision="fp64", lib=oracle)
        h = sim.addParticles(x, np.zeros_like(x), 1e-3, dx ** 3 / 8)
        h.addFBasedMpmForce(mpm.NeoHookeanBorden(E, nu))
        F = np.zeros((n, 3, 3))
        F[:, 0, 0] = F[:, 2, 2] = 1.0
        F[:, 1, 1] = stretch
        sim.setParticles(F=F)
        h.addRankineDamage(sigma_f, residual_phase=0.001, reference_order=ref)
        assert sim.advanceOneTimeStep(1e-4) == abi.OK
        out[ref] = sim.getDamage()
    smax = np.maximum(syy, sxx)
    np.testing.assert_allclose(out[False], np.where(smax > sigma_f, np.minimum(1.0, sigma_f / smax), 1.0), rtol=1e-12)
    np.testing.assert_allclose(out[True], np.where(sxx > sigma_f, np.minimum(1.0, sigma_f / sxx), 1.0), rtol=1e-12)
    assert (out[True] != out[False]).sum() > n // 8


def _admm_scene(lib, integrator, visco=False, iters=20, precision="fp64", E=2e4, nu=0.4, dx=1.0 / 64, seed=3,
                grid_log2=None):
    """Slab dropped on a sticky sphere over a sticky ground (the ADMM benchmark's
    shape, scaled down)."""
    kw = {} if grid_log2 is None else {"grid_log2": grid_log2}
    s = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, lib=lib, **kw)
    x = jittered_box((12, 4, 12), dx, (0.3, 0.55, 0.3), 8, seed)
    V0 = dx ** 3 / 8
    h = s.addParticles(x, np.tile([0.0, -1.0, 0.0], (len(x), 1)), 1000 * V0, V0)
    h.addFBasedMpmForce(mpm.StvkWithHenckyIsotropic(E, nu))
    if visco:
        mu = E / (2 * (1 + nu))
        nv = 2 * mu * 0.05  # relaxation time 0.05 s: alpha = 2 mu / nu_d = 1 / 0.05
        h.addFElasticNonequilibratedBasedMpmForce(mpm.StvkWithHencky(E, nu), nv, nv)
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.Sphere((0.5, 0.35, 0.5), 0.2), abi.STICKY))
    s.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    if integrator == "admm":
        s.useAdmm(admm_max_iterations=iters, rho_scale=0.8, global_tolerance=1e-8)
    else:
        s.switchLinearSolver(abi.CG)
        s.newton_tolerance = 1e-9
        s.newton_max_iterations = 30
        s.krylov_max_iterations = 500
    return s


def test_admm_converges_to_the_newton_solution(oracle):
    """ADMM (AdmmSimulationFoam.h:766-801) minimises the same backward-Euler
    objective as Newton: with enough iterations both restatements land on the
    same velocities."""
    out = {}
    for integ, iters in (("newton", 0), ("admm", 20), ("admm", 100)):
        s = _admm_scene(oracle, integ, iters=iters)
        for _ in range(3):
            assert s.advanceOneTimeStep(2e-3) == abi.OK
        out[iters] = s.getParticles()["V"]
    scale = np.abs(out[0]).max()
    assert np.abs(out[20] - out[0]).max() / scale < 1e-3
    assert np.abs(out[100] - out[0]).max() / scale < 1e-9


def test_viscous_return_map_known_answer(oracle):
    """FElasticNonequilibratedBasedMpmForceHelper::evolveStrain (h:62-87):
    eps = (eps_trial - dt beta / (1 + dt (alpha + 3 beta)) t) / (1 + dt alpha),
    Fe = U exp(eps) V^T, with alpha = 2 mu / nu_d, beta = 2 (2 mu + 3 lambda) /
    (9 nu_v) - 2 mu / (3 nu_d).  t is `epsilon_trial.trace()` of a 3-vector,
    which Eigen evaluates as its first coefficient."""
    rng = np.random.default_rng(4)
    E, nu, vd, vv, dt = 2e4, 0.4, 700.0, 500.0, 2e-3
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    alpha = 2 * mu / vd
    beta = 2 * (2 * mu + 3 * lam) / (9 * vv) - 2 * mu / (3 * vd)
    for _ in range(20):
        s = np.sort(rng.uniform(0.7, 1.4, 3))[::-1]
        U, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        V, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        U *= np.sign(np.linalg.det(U))
        V *= np.sign(np.linalg.det(V))
        F = U @ np.diag(s) @ V.T
        out = np.ascontiguousarray(F.ravel())
        oracle.dll.zoracle_viscous_return(C.c_double(E), C.c_double(nu), C.c_double(vd), C.c_double(vv), C.c_double(dt), P(out))
        et = np.log(s)
        eps = (et - dt * beta / (1 + dt * (alpha + 3 * beta)) * et[0]) / (1 + dt * alpha)
        np.testing.assert_allclose(out.reshape(3, 3), U @ np.diag(np.exp(eps)) @ V.T, rtol=0, atol=1e-12)
    # infinite viscosities leave Fe unchanged
    out = np.ascontiguousarray(F.ravel())
    oracle.dll.zoracle_viscous_return(C.c_double(E), C.c_double(nu), C.c_double(1e300), C.c_double(1e300), C.c_double(dt), P(out))
    np.testing.assert_allclose(out.reshape(3, 3), F, atol=1e-12)


def test_admm_viscoelastic_substeps(oracle):
    """Viscoelastic slab (config 2 shape): Fe deviates from I under load and the
    substep status is clean; Newton refuses viscoelastic particles like the
    reference's StvkWithHencky, which has no stress differential."""
    s = _admm_scene(oracle, "admm", visco=True)
    for _ in range(3):
        assert s.advanceOneTimeStep(2e-3) == abi.OK
    Fe = s.getViscoelasticStrain()
    assert np.abs(Fe - np.eye(3)).max() > 1e-3
    assert np.all(np.isfinite(Fe))
    s.integrator = abi.NEWTON
    assert s.lib.substep(s.ctx, 2e-3, C.byref(s.solver()), None) == abi.BAD_ARG


def _explicit_cube(lib, gravity=(0, -9.8, 0), kind="fcr", v0=(0.3, -1.0, 0.2), ground=None, seed=1, lo=(0.375, 0.105, 0.375)):
    dx = 1.0 / 64
    s = mpm.MpmSimulation(dx, gravity=gravity, precision="fp64", lib=lib)
    build_scene(s, kind=kind, n=6, dx=dx, v0=v0, ground=ground, seed=seed, lo=lo)
    s.useExplicit()
    return s


def test_explicit_free_fall_is_exact(oracle):
    """Symplectic substeps of an unstressed cube in free fall (F = I, no
    colliders): every particle gains g dt per substep, C stays zero."""
    s = _explicit_cube(oracle)
    v0 = s.getParticles()["V"].copy()
    dt = 1e-3
    for _ in range(10):
        assert s.advanceOneTimeStep(dt) == abi.OK
    p = s.getParticles()
    want = v0 + 10 * dt * np.array([0, -9.8, 0])
    np.testing.assert_allclose(p["V"], want, rtol=0, atol=1e-12)
    np.testing.assert_allclose(p["F"].reshape(-1, 9), np.tile(np.eye(3).ravel(), (len(v0), 1)), rtol=0, atol=1e-12)


def test_explicit_conserves_momentum(oracle):
    """Without gravity and colliders, APIC P2G/G2P with the elastic force
    conserves total linear momentum to round-off while the cube deforms."""
    s = _explicit_cube(oracle, gravity=(0, 0, 0), v0=(0, 0, 0))
    p = s.getParticles()
    rng = np.random.default_rng(4)
    V = rng.normal(0, 0.2, p["V"].shape)
    s.setParticles(V=V)
    m = np.full(len(V), 1000.0 * (1 / 64) ** 3 / 8)
    mom0 = (m[:, None] * V).sum(0)
    for _ in range(10):
        assert s.advanceOneTimeStep(2e-4) == abi.OK
    p = s.getParticles()
    assert np.abs(p["F"].reshape(-1, 3, 3) - np.eye(3)).max() > 1e-4
    mom = (m[:, None] * p["V"]).sum(0)
    assert np.abs(mom - mom0).max() < 1e-12 * np.abs(m[:, None] * V).sum()


def test_explicit_trial_collision_keeps_particles_above_ground(oracle):
    """A cube falling fast onto a sticky ground: the explicit collision at t and
    the trial collision against the ground at t + dt keep particles from
    crossing it; turning trial collision off changes the landing substep.  The
    ground sits just below the grid plane y = 7 dx, where nodes that did not
    collide at t reach it within one substep."""
    dx = 1.0 / 64
    ground = 7 * dx - 1e-3
    runs = []
    for trial in (True, False):
        s = _explicit_cube(oracle, v0=(0, -3.0, 0), ground=ground, lo=(0.375, 8 * dx, 0.375))
        s.useExplicit(trial_collision=trial)
        for _ in range(40):
            assert s.advanceOneTimeStep(5e-4) == abi.OK
        runs.append(s.getParticles())
    assert runs[0]["X"][:, 1].min() > ground - dx
    assert np.abs(runs[0]["V"] - runs[1]["V"]).max() > 1e-6


def test_mls_explicit_free_fall_momentum_and_refusal(oracle):
    """MLS-MPM (mls_mpm, MpmSimulationBase.cpp:527-541, :958-961): free fall is
    exact, total linear momentum is conserved without gravity (sum_i w_ip
    (x_i - x_p) = 0 for the quadratic B-spline), the result differs from the
    APIC gradient, and the implicit integrators refuse it as the reference does
    (MpmSimulationBase.cpp:102-106)."""
    s = _explicit_cube(oracle)
    s.useExplicit(mls_mpm=True)
    v0 = s.getParticles()["V"].copy()
    for _ in range(10):
        assert s.advanceOneTimeStep(1e-3) == abi.OK
    np.testing.assert_allclose(s.getParticles()["V"], v0 + 1e-2 * np.array([0, -9.8, 0]), rtol=0, atol=1e-12)

    runs = []
    for mls in (True, False):
        s = _explicit_cube(oracle, gravity=(0, 0, 0), v0=(0, 0, 0))
        s.useExplicit(mls_mpm=mls)
        V = np.random.default_rng(4).normal(0, 0.2, s.getParticles()["V"].shape)
        s.setParticles(V=V)
        for _ in range(10):
            assert s.advanceOneTimeStep(2e-4) == abi.OK
        p = s.getParticles()
        assert np.abs(p["V"].sum(0) - V.sum(0)).max() < 1e-12 * np.abs(V).sum()
        runs.append(p)
    assert np.abs(runs[0]["F"] - runs[1]["F"]).max() > 1e-6

    s = _explicit_cube(oracle)
    s.useExplicit(mls_mpm=True)
    s.integrator = abi.NEWTON
    assert s.lib.substep(s.ctx, 1e-3, C.byref(s.solver()), None) == abi.BAD_ARG


def _nhb_psi_pos(mu, kappa, F):
    J = np.linalg.det(F)
    JaF = J ** (-1.0 / 3.0) * F
    psi_dev = mu / 2 * (np.trace(JaF.T @ JaF) - 3)
    psi_vol = kappa / 2 * ((J * J - 1) / 2 - np.log(J))
    return psi_vol + psi_dev if J >= 1 else psi_dev


def _pf_cube(lib, stretch=0.3, dx=1.0 / 64, seed=2, **kw):
    s = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", lib=lib, **kw)
    h, x = build_scene(s, kind="nh", n=6, dx=dx, seed=seed)
    n = len(x)
    F = np.zeros((n, 3, 3))
    F[:, 0, 0] = 1 + stretch * (x[:, 0] - x[:, 0].min()) / np.ptp(x[:, 0])
    F[:, 1, 1] = F[:, 2, 2] = 1
    s.setParticles(F=F)
    return s, h, x, F


def test_phase_field_known_answers(oracle):
    """CD-MPM phase field (FractureSimulation::solvePhaseFieldSystem): with
    pf_Fp = 1 the elliptic system's solution is c = 1 exactly (the Laplacian of
    a constant vanishes by the partition of unity), so an unstrained body stays
    undamaged after a first CG step that lands on it; vol = V0 det F; H and
    pf_Fp follow Update_Phase_Field_Fp (PhaseField.h:70-76) from the positive
    NeoHookeanBorden energy (NeoHookeanBorden.cpp:53-66); 1/sigma_c follows
    Get_Sigma_C_Based_On_Max_Deformation (PhaseField.h:58-68)."""
    E, nu, l0, pct, k = 1e4, 0.3, 0.5 / 64, 0.05, 0.001
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    kappa = 0.666666 * mu + lam  # NeoHookeanBorden::setLameParameters (NeoHookeanBorden.cpp:20)
    s, h, x, F = _pf_cube(oracle, stretch=0.0)
    h.addFBasedMpmForceWithPhaseField(pct, l0)
    s.setPhaseFieldSolver(cg_tolerance=1e-30)
    assert s.advanceOneTimeStep(1e-3) == abi.OK
    assert s.last_stats["phase_field_iterations"] <= 1
    pf = s.getPhaseField()
    np.testing.assert_allclose(pf["c"], 1.0, rtol=0, atol=1e-12)

    s, h, x, F = _pf_cube(oracle, stretch=0.3)
    h.addFBasedMpmForceWithPhaseField(pct, l0)
    V0 = (1.0 / 64) ** 3 / 8
    assert s.advanceOneTimeStep(1e-3) == abi.OK
    pf = s.getPhaseField()
    np.testing.assert_allclose(pf["vol"], V0 * np.linalg.det(F), rtol=1e-14)
    # H and pf_Fp come from F after the substep's G2P (phaseG2P runs after P2G on
    # the start-of-substep F; getParticles returns the end-of-substep F)
    f = 1 + pct
    J = f ** 3
    isc = 1.0 / (kappa / 2 * ((J * J - 1) / 2 - np.log(J)) + mu / 2 * (3 * (J ** (-1 / 3) * f) ** 2 - 3))
    H = np.array([_nhb_psi_pos(mu, kappa, Fi) for Fi in F])
    np.testing.assert_allclose(pf["H"], H, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(pf["pf_Fp"], 4 * l0 * (1 - k) * H * isc + 1, rtol=1e-12)
    # the first solve still saw pf_Fp = 1 (it is updated after the solve), so
    # damage shows from the second substep on
    np.testing.assert_allclose(pf["c"], 1.0, rtol=0, atol=1e-12)
    assert s.advanceOneTimeStep(1e-3) == abi.OK
    c = s.getDamage()
    assert c.min() < 0.95 and np.all(c <= 1)


@pytest.mark.parametrize("M,lumping", [(0.0, True), (0.0, False), (1.0, True)])
def test_phase_field_cg_converges_and_degrades(oracle, M, lumping):
    """The CG of the phase-field system reaches a tight tolerance, damage grows
    where the body is stretched, and particles that may not be damaged keep c."""
    s, h, x, F = _pf_cube(oracle, stretch=0.3)
    lo = np.argsort(x[:, 0])[:50]
    h.addFBasedMpmForceWithPhaseField(0.05, 0.5 / 64)
    s.setPhaseFieldSolver(parabolic_M=M, lumping=lumping, cg_tolerance=1e-16)
    for _ in range(3):
        assert s.advanceOneTimeStep(1e-3) == abi.OK
        st = s.last_stats
        assert st["phase_field_residual"] < 1e-12 * 1e3 or st["phase_field_iterations"] > 3
    c = s.getDamage()
    assert np.all((c >= 0) & (c <= 1))
    right = x[:, 0] > np.median(x[:, 0])
    assert c[right].mean() < c[~right].mean()


def test_phase_field_refusals(oracle):
    s, h, x, F = _pf_cube(oracle)
    h.addFBasedMpmForceWithPhaseField(0.05, 0.5 / 64)
    s.useAdmm(admm_max_iterations=4)
    assert s.lib.substep(s.ctx, 1e-3, C.byref(s.solver()), None) == abi.BAD_ARG
    s2 = mpm.MpmSimulation(1.0 / 64, gravity=(0, -9.8, 0), precision="fp64", lib=oracle)
    h2, _ = build_scene(s2, kind="fcr", n=4, dx=1.0 / 64)
    with pytest.raises(abi.ZmpmError):
        h2.addFBasedMpmForceWithPhaseField(0.05, 0.5 / 64)


def _dp_numpy(F, mu, lam, alpha, beta, cohesion, vc, logJp):
    """Drucker-Prager return map restated from Klar et al. 2016 (the reference's
    DruckerPragerStvkHencky::projectStrain) with numpy's SVD; isotropic, so the
    SVD's sign and order conventions do not matter for det F > 0."""
    U, s, Vt = np.linalg.svd(F)
    eps = np.log(np.maximum(np.abs(s), 1e-4)) - cohesion
    tr = eps.sum() + logJp
    hat = eps - tr / 3
    if tr >= 0:
        return np.exp(cohesion) * U @ Vt, (beta * eps.sum() + logJp if vc else logJp)
    hn = np.linalg.norm(hat)
    dg = hn + (3 * lam + 2 * mu) / (2 * mu) * tr * alpha
    H = eps + cohesion if dg <= 0 else eps - dg / hn * hat + cohesion
    return U @ np.diag(np.exp(H)) @ Vt, 0.0


def _camclay_numpy(F, mu, kappa, M, beta, xi, logJp):
    """Cam-Clay projection (the reference's Compare_With_Physbam branch of
    NonAssociativeCamClay::projectStrain) restated with numpy's SVD."""
    U, Se, Vt = np.linalg.svd(F)
    p0 = kappa * (1e-5 + np.sinh(xi * max(-logJp, 0.0)))
    a = (1 + 2 * beta) * 3 / 2
    b, c, M2 = beta * p0, p0, M * M
    Je = np.prod(Se)
    Se2 = Se ** 2
    s = mu * Je ** (-2 / 3) * (Se2 - Se2.mean())
    p_trial = -kappa / 2 * (Je - 1 / Je) * Je
    if p_trial > c or p_trial < -b:
        Je_new = np.sqrt(-2 * c / kappa + 1) if p_trial > c else np.sqrt(2 * b / kappa + 1)
        return Je_new ** (1 / 3) * U @ Vt, logJp + np.log(Je / Je_new)
    k = np.sqrt(-M2 * (p_trial + b) * (p_trial - c) / a)
    sn = np.linalg.norm(s)
    if a * sn ** 2 + M2 * (p_trial + b) * (p_trial - c) < 1e-4:
        return F.copy(), logJp
    pc = (1 - beta) * p0 / 2
    if p0 > 1e-4 and p0 - 1e-4 > p_trial > -beta * p0 + 1e-4:
        aa = M2 * (p_trial - pc) ** 2 / (a * sn ** 2)
        dd, ff, gg = 1 + aa, aa * beta * p0 - aa * p0 - 2 * pc, pc ** 2 - aa * beta * p0 ** 2
        zz = np.sqrt(abs(ff ** 2 - 4 * dd * gg))
        p1, p2 = (-ff + zz) / (2 * dd), (-ff - zz) / (2 * dd)
        p_fake = p1 if (p_trial - pc) * (p1 - pc) > 0 else p2
        Jf = np.sqrt(abs(-2 * p_fake / kappa + 1))
        if Jf > 1e-4:
            logJp += np.log(Je / Jf)
    be = k / mu * Je ** (2 / 3) * s / sn + Se2.sum() / 3
    return U @ np.diag(np.sqrt(be)) @ Vt, logJp


def test_drucker_prager_and_cam_clay_known_answers(oracle):
    """The oracle's Drucker-Prager and Cam-Clay return maps against numpy
    restatements over compressed, sheared and stretched strains (every branch:
    inside, cone / ellipse projection, tips, fake hardening)."""
    d = oracle.dll
    rng = np.random.default_rng(12)
    E, nu = 1e4, 0.3
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    kappa = 0.666666 * mu + lam
    sphi = np.sin(30 / 180 * 3.141592653)
    alpha = np.sqrt(2 / 3) * 2 * sphi / (3 - sphi)
    M = alpha * 3 / np.sqrt(2 / 3)
    seen_dp, seen_cc = set(), set()
    for trial in range(400):
        R1, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        R2, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        R1 *= np.sign(np.linalg.det(R1))
        R2 *= np.sign(np.linalg.det(R2))
        vol = rng.choice([0.9, 0.97, 1.0, 1.03, 1.2])
        s = vol * np.exp(rng.normal(0, 0.08, 3))
        F = R1 @ np.diag(s) @ R2.T
        for cohesion, vc, logJp in ((0.0, 1, 0.0), (0.01, 1, -0.02), (0.0, 0, 0.05)):
            out = F.ravel().copy()
            lj = C.c_double(logJp)
            prm = np.array([alpha, 1.0, cohesion])
            assert d.zoracle_plastic_project(2, mu, lam, kappa, P(prm), vc, C.byref(lj), P(out)) == 0
            want, wl = _dp_numpy(F, mu, lam, alpha, 1.0, cohesion, vc, logJp)
            np.testing.assert_allclose(out.reshape(3, 3), want, rtol=0, atol=1e-12)
            assert abs(lj.value - wl) < 1e-12
            seen_dp.add("tip" if np.allclose(want @ want.T, np.exp(2 * cohesion) * np.eye(3)) else
                        ("in" if np.allclose(want, F) else "cone"))
        for beta, xi, logJp in ((0.5, 2.0, -0.05), (0.2, 5.0, -0.2), (0.0, 1.0, 0.0)):
            out = F.ravel().copy()
            lj = C.c_double(logJp)
            prm = np.array([M, beta, xi])
            assert d.zoracle_plastic_project(3, mu, lam, kappa, P(prm), 1, C.byref(lj), P(out)) == 0
            want, wl = _camclay_numpy(F, mu, kappa, M, beta, xi, logJp)
            np.testing.assert_allclose(out.reshape(3, 3), want, rtol=0, atol=1e-11)
            assert abs(lj.value - wl) < 1e-11
            seen_cc.add("moved" if not np.allclose(want, F) else "in")
    assert seen_dp == {"tip", "in", "cone"} and seen_cc == {"moved", "in"}


@pytest.mark.parametrize("kind", ["dp", "cc"])
def test_sand_and_clay_substeps(oracle, kind):
    """A falling block with Drucker-Prager (sand) or Cam-Clay (clay) plasticity
    lands on the ground: log Jp evolves and every substep is clean.  The sand
    starts dilated (F = 1.05 I), which sends it to the cone tip (the volume
    correction then stores the excess in log Jp)."""
    dx = 1.0 / 64
    s = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", lib=oracle)
    model = "hencky" if kind == "dp" else "nh"
    h, x = build_scene(s, kind=model, n=6, dx=dx, v0=(0, -2.0, 0), lo=(0.375, 8 * dx, 0.375), ground=7 * dx)
    if kind == "dp":
        s.setParticles(F=np.tile(1.05 * np.eye(3), (len(x), 1, 1)))
        h.addPlasticity(None, mpm.DruckerPragerStvkHencky(30.0, 1.0, 0.0, True))
    else:
        h.addPlasticity(None, mpm.NonAssociativeCamClay(-0.01, 45.0, 0.3, 3.0, True))
    for _ in range(8):
        assert s.advanceOneTimeStep(1e-3) == abi.OK
    lj = s.getLogJp()
    assert np.all(np.isfinite(lj)) and np.abs(lj).max() > 0


def _dp_sigma_numpy(mu, lam, alpha, cohesion, s):
    """DruckerPragerStvkHencky::projectSigma restated (no log Jp)."""
    eps = np.log(np.maximum(np.abs(s), 1e-4)) - cohesion
    tr = eps.sum()
    hat = eps - tr / 3
    if tr >= 0:
        return np.exp(cohesion) * np.ones(3)
    hn = np.linalg.norm(hat)
    dg = hn + (3 * lam + 2 * mu) / (2 * mu) * tr * alpha
    return np.exp(eps + cohesion) if dg <= 0 else np.exp(eps - dg / hn * hat + cohesion)


def test_admm_drucker_prager_sigma_maps(oracle):
    """The Drucker-Prager maps of the ADMM local step: projectSigma against a
    numpy restatement, projectSigmaAndDerivative's Jacobian against central
    differences of its own projection inside each branch (cone, inside, tip)."""
    d = oracle.dll
    E, nu = 1e4, 0.3
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    sphi = np.sin(30 / 180 * 3.141592653)
    alpha = np.sqrt(2 / 3) * 2 * sphi / (3 - sphi)
    rng = np.random.default_rng(21)
    seen = set()
    for _ in range(300):
        cohesion = rng.choice([0.0, 0.01])
        s = rng.choice([0.9, 0.97, 1.0, 1.05]) * np.exp(rng.normal(0, 0.08, 3))
        out = np.zeros(3)
        assert d.zoracle_dp_project_sigma(mu, lam, alpha, cohesion, P(s), P(out), None) == 0
        np.testing.assert_allclose(out, _dp_sigma_numpy(mu, lam, alpha, cohesion, s), rtol=1e-13, atol=0)
        D = np.zeros(9)
        o2 = np.zeros(3)
        assert d.zoracle_dp_project_sigma(mu, lam, alpha, cohesion, P(s), P(o2), P(D)) == 0
        h = 1e-6
        J = np.zeros((3, 3))
        for c in range(3):
            sp, sm = s.copy(), s.copy()
            sp[c] += h
            sm[c] -= h
            op, om = np.zeros(3), np.zeros(3)
            d.zoracle_dp_project_sigma(mu, lam, alpha, cohesion, P(sp), P(op), P(np.zeros(9)))
            d.zoracle_dp_project_sigma(mu, lam, alpha, cohesion, P(sm), P(om), P(np.zeros(9)))
            J[:, c] = (op - om) / (2 * h)
        branch = "tip" if not D.any() else ("inside" if np.allclose(D.reshape(3, 3), np.eye(3)) else "cone")
        seen.add(branch)
        np.testing.assert_allclose(D.reshape(3, 3), J, rtol=1e-5, atol=1e-6)
    assert seen == {"tip", "inside", "cone"}


def test_admm_sand_substeps(oracle):
    """ADMM with Drucker-Prager sand (AdmmSimulationFoam's StvkWithHencky +
    DruckerPragerStvkHencky F-step): substeps are clean and log Jp evolves;
    Cam-Clay stays refused under ADMM."""
    dx = 1.0 / 64
    s = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", lib=oracle)
    h, x = build_scene(s, kind="hencky", n=6, dx=dx, v0=(0, -2.0, 0), lo=(0.375, 8 * dx, 0.375), ground=7 * dx)
    s.setParticles(F=np.tile(np.diag([1.04, 1.0, 1.02]), (len(x), 1, 1)))
    h.addPlasticity(None, mpm.DruckerPragerStvkHencky(30.0, 1.0, 0.0, True))
    s.useAdmm(admm_max_iterations=10, rho_scale=0.8, global_tolerance=1e-10)
    for _ in range(4):
        assert s.advanceOneTimeStep(1e-3) == abi.OK
    assert np.all(np.isfinite(s.getParticles()["X"])) and np.abs(s.getLogJp()).max() > 0
    s2 = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", lib=oracle)
    h2, _ = build_scene(s2, kind="nh", n=4, dx=dx)
    h2.addPlasticity(None, mpm.NonAssociativeCamClay(-0.01, 45.0, 0.3, 3.0, True))
    s2.useAdmm(admm_max_iterations=4)
    assert s2.lib.substep(s2.ctx, 1e-3, C.byref(s2.solver()), None) == abi.UNSUPPORTED


def test_calculate_dt_and_time_stepping(oracle):
    """calculateDt (MpmSimulationBase.cpp:766-790) = cfl dx / max speed over
    particles and colliders; TimeStepping hits frame times exactly."""
    dx = 1.0 / 64
    s = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", lib=oracle, cfl=0.5)
    h, x = build_scene(s, kind="fcr", n=4, dx=dx, v0=(0.3, -1.0, 0.2))
    v, lo, hi = s.maxParticleSpeed()
    assert abs(v - np.linalg.norm([0.3, -1.0, 0.2])) < 1e-12
    np.testing.assert_allclose(lo, x.min(0), rtol=0, atol=1e-15)
    np.testing.assert_allclose(hi, x.max(0), rtol=0, atol=1e-15)
    assert abs(s.calculateDt(0.01) - 0.5 * dx / v) < 1e-15
    fast = mpm.AnalyticCollisionObject(mpm.Sphere((0.5, 0.5, 0.5), 0.1), abi.SLIP)
    fast.setTranslation((0.0, 0.0, 0.0), (0.0, 0.0, 5.0))
    s.addCollisionObject(fast)
    assert abs(s.calculateDt(0.01) - 0.5 * dx / 5.0) < 1e-15
    spin = mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.05, 0), (0, 1, 0)), abi.STICKY)
    spin.setAngularVelocity((0, 1.0, 0))
    s.addCollisionObject(spin)
    with pytest.raises(abi.ZmpmError):
        s.calculateDt(0.01)
    step = mpm.TimeStepping(frame_dt=1.0 / 24)
    step.max_dt = 0.01
    dts = []
    while True:
        dt = step.nextDt(0.007)
        dts.append(dt)
        if step.advance(dt) == mpm.TimeStepping.FRAME:
            break
    assert abs(sum(dts) - 1.0 / 24) < 1e-15 and max(dts) <= 0.007 + 1e-15
