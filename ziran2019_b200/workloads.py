"""Seeded synthetic scenes of the benchmark configurations (the benchmark has
no dataset; shapes, sizes and value distributions follow each configuration).

Each `wl_*(precision, lib=None, layout="auto", scale=1)` builds one workload on
the CUDA library (lib=None) or on another library with the same ABI, and
returns (simulation, dt, particles, metadata).  `scale > 1` takes a cut of the
scene (CPU samples and parity tests).  `scene` / `make_sim` build the 1M-particle
elastoplastic workload of four boxes.
"""
import os

import numpy as np

DX = 1.0 / 256
DT = 5e-4
CELLS = (25, 25, 50)
PPC = 8
RHO = 1000.0
E, NU, YIELD = 5e4, 0.35, 150.0


def scene(n_boxes=4, seed_pos=1, seed_vel=2, seed_jit=0, velocity="particle"):
    """Seeded synthetic scene (the benchmark has no dataset; shapes follow the workload).

    velocity="particle": every particle draws its velocity uniformly from [-1,1]^3,
    so the Newton solve works from the first substep.  velocity="box": one rigid
    velocity per box; the boxes then fly undeformed (Newton converges at its first
    residual check, no Hessian products) until they reach a wall."""
    size = np.array(CELLS) * DX
    rng = np.random.default_rng(seed_pos)
    corners = []
    while len(corners) < 4:
        c = rng.uniform(4 * DX, 1 - size - 4 * DX)
        if all(np.any((c + size + 2 * DX <= o) | (o + size + 2 * DX <= c)) for o in corners):
            corners.append(c)
    vel = np.random.default_rng(seed_vel).uniform(-1, 1, size=(4, 3))
    jr = np.random.default_rng(seed_jit)
    grid = np.stack(np.meshgrid(*[np.arange(c) for c in CELLS], indexing="ij"), -1).reshape(-1, 3)
    xs, vs = [], []
    for b in range(n_boxes):
        x = (np.repeat(grid, PPC, 0) + jr.random((grid.shape[0] * PPC, 3))) * DX + corners[b]
        xs.append(x)
        vs.append(np.tile(vel[b], (x.shape[0], 1)))
    x, v = np.concatenate(xs), np.concatenate(vs)
    if velocity == "particle":
        v = np.random.default_rng(seed_vel).uniform(-1, 1, size=x.shape)
    return x, v


def make_sim(x, v, precision, lib=None, model="hencky", layout="auto", plastic="von_mises"):
    from . import abi, mpm

    sim = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, grid_log2=9, layout=layout,
                            device=int(os.environ.get("LOCAL_RANK", "0")) if lib is None else 0, lib=lib)
    V0 = DX ** 3 / PPC
    h = sim.addParticles(x, v, RHO * V0, V0)
    m = mpm.StvkWithHenckyIsotropic(E, NU) if model == "hencky" else mpm.NeoHookeanBorden(E, NU)
    h.addFBasedMpmForce(m)
    if plastic == "von_mises":
        h.addPlasticity(m, mpm.VonMisesStvkHencky(YIELD, 1e30, 0.0))
    elif plastic == "drucker_prager":
        h.addPlasticity(m, mpm.DruckerPragerStvkHencky(30.0, 1.0, 0.0, True))
    mpm.add_all_walls_in_domain(sim, 1.0, 3 * DX, abi.STICKY)
    return sim


# ----------------------------------------------------------------------------
# Secondary workloads (the other benchmark configurations; `--workload`).  Each
# prints its own JSON line; the default workload is the headline above.
def _jitter_box(cells, dx, lo, ppc, seed):
    rng = np.random.default_rng(seed)
    grid = np.stack(np.meshgrid(*[np.arange(c) for c in cells], indexing="ij"), -1).reshape(-1, 3)
    return (np.repeat(grid, ppc, 0) + rng.random((grid.shape[0] * ppc, 3))) * dx + np.asarray(lo, dtype=np.float64)


def wl_cube32k(precision, lib=None, layout="auto", scale=1):
    """Elastic cube: 16^3 cells x 8 ppc = 32,768 particles (seed 0), dx = 1/64,
    min corner (0.375, 0.125, 0.375), fixed corotated E = 1e4, nu = 0.3,
    rho = 1000, gravity, sticky ground y = 0.1, Newton-CG rel. tol 1e-7, dt = 1e-3."""
    from . import abi, mpm
    dx = 1.0 / 64
    x = _jitter_box((16, 16, 16), dx, (0.375, 0.125, 0.375), 8, 0)
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, grid_log2=7, layout=layout, lib=lib)
    V0 = dx ** 3 / 8
    h = sim.addParticles(x, np.zeros_like(x), 1000.0 * V0, V0)
    h.addFBasedMpmForce(mpm.FixedCorotated(1e4, 0.3))
    sim.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    sim.switchLinearSolver(abi.CG)
    sim.newton_tolerance = 1e-7
    sim.newton_max_iterations = 10
    sim.krylov_max_iterations = 100
    return sim, 1e-3, x.shape[0], {"workload": "config0-elastic-cube-32k", "model": "fixed corotated", "solver": "Newton-CG tol 1e-7"}


def wl_admm500k(precision, lib=None, layout="auto", scale=1):
    """Viscoelastic ADMM slab: 0.6 x 0.1 x 0.6 at dx = 1/120, 72 x 12 x 72 cells x 8
    ppc = 497,664 particles (seed 3) over a static sticky sphere of radius 0.2;
    StvkWithHenckyIsotropic E = 2e4, nu = 0.4 plus the non-equilibrated
    StvkWithHencky with nu_d = nu_v = 2 mu tau, tau = 0.05 s; 20 ADMM
    iterations, rho_scale 0.8, dt = 2e-3.  The slab starts touching the sphere
    with the speed of a 0.3 m drop (sqrt(2 g 0.3) = 2.42 m/s) so every timed
    substep deforms it.  scale > 1 takes every scale-th cell column in x and z
    (CPU samples)."""
    from . import abi, mpm
    dx = 1.0 / 120
    nx = 72 // scale
    x = _jitter_box((nx, 12, nx), dx, (0.5 - nx * dx / 2, 0.5 + 2 * dx, 0.5 - nx * dx / 2), 8, 3)
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, grid_log2=8, layout=layout, lib=lib)
    V0 = dx ** 3 / 8
    v = np.tile([0.0, -np.sqrt(2 * 9.8 * 0.3), 0.0], (x.shape[0], 1))
    h = sim.addParticles(x, v, 1000.0 * V0, V0)
    E, nu, tau = 2e4, 0.4, 0.05
    h.addFBasedMpmForce(mpm.StvkWithHenckyIsotropic(E, nu))
    nvis = 2 * E / (2 * (1 + nu)) * tau
    h.addFElasticNonequilibratedBasedMpmForce(mpm.StvkWithHencky(E, nu), nvis, nvis)
    sim.addCollisionObject(mpm.AnalyticCollisionObject(mpm.Sphere((0.5, 0.3, 0.5), 0.2), abi.STICKY))
    sim.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 3 * dx, 0), (0, 1, 0)), abi.STICKY))
    sim.useAdmm(admm_max_iterations=20, rho_scale=0.8, global_tolerance=1e-8, local_tolerance=1e-8)
    return sim, 2e-3, x.shape[0], {"workload": "config2-viscoelastic-admm-500k", "model": "hencky + viscoelastic Fe",
                                   "solver": "ADMM 20 iterations, MINRES abs tol 1e-8"}


def wl_damage2m(precision, lib=None, layout="auto", scale=1, reference_order=True):
    """Notched slab 1.0 x 0.25 x 0.1 with a 0.1-long, one-cell-wide edge notch at
    mid-length, 8 ppc at dx = 1/216 (216 x 54 x 22 cells, about 2.05M
    particles, seed 4); the end faces are held by sticky boxes moving apart at
    +-0.5 m/s; NeoHookeanBorden E = 1e5, nu = 0.3 with Rankine damage sigma_F =
    1e3 Pa, k = 1e-3; dt = 2e-4, no gravity.  reference_order: sigma_max is the
    first eigenvalue of Eigen's general eigensolver, as the reference takes it
    (default), else the largest.  scale > 1 keeps every scale-th cell layer in
    z (CPU samples)."""
    from . import abi, mpm
    dx = 1.0 / 216
    nx, ny, nz = 216, 54, max(1, 22 // scale)
    lo = np.array([0.25, 0.5, 0.5])
    x = _jitter_box((nx, ny, nz), dx, lo, 8, 4)
    rel = (x - lo) / dx
    notch = (np.abs(rel[:, 0] - nx / 2) < 0.5) & (rel[:, 1] < 0.1 / dx)
    x = x[~notch]
    sim = mpm.MpmSimulation(dx, gravity=(0, 0, 0), precision=precision, grid_log2=9, layout=layout, lib=lib)
    V0 = dx ** 3 / 8
    h = sim.addParticles(x, np.zeros_like(x), 1000.0 * V0, V0)
    h.addFBasedMpmForce(mpm.NeoHookeanBorden(1e5, 0.3))
    h.addRankineDamage(1e3, residual_phase=1e-3, reference_order=reference_order)
    hi = lo + np.array([nx, ny, nz]) * dx
    grip = 3 * dx
    for side, vel in ((0, -0.5), (1, 0.5)):
        a = [lo[0] - 4 * dx if side == 0 else hi[0] - grip, lo[1] - 4 * dx, lo[2] - 4 * dx]
        b = [lo[0] + grip if side == 0 else hi[0] + 4 * dx, hi[1] + 4 * dx, hi[2] + 4 * dx]
        box = mpm.AnalyticCollisionObject(mpm.AxisAlignedAnalyticBox(a, b), abi.STICKY)
        box.setTranslation((0.0, 0.0, 0.0), (vel, 0.0, 0.0))
        sim.addCollisionObject(box)
    return sim, 2e-4, x.shape[0], {"workload": "config3-rankine-notched-slab-2m", "model": "neo-Hookean + Rankine damage",
                                   "solver": "MINRES, Newton 3 x Krylov 20 (reference defaults)"}


def wl_explicit1m(precision, lib=None, layout="auto", scale=1):
    """The headline scene (four boxes of 250,000 particles, StvkWithHencky +
    von Mises, sticky walls) advanced by the explicit symplectic substep
    (symplectic = true, trial collision on) at dt = 1e-4 (the p-wave speed is
    about 9.6 m/s at dx = 1/256).  scale > 1 keeps 4 // scale boxes (CPU samples)."""
    x, v = scene(n_boxes=max(1, 4 // scale))
    sim = make_sim(x, v, precision, lib=lib, layout=layout)
    sim.useExplicit()
    return sim, 1e-4, x.shape[0], {"workload": "explicit-elastoplastic-4boxes-1m", "model": "hencky+von Mises",
                                   "solver": "explicit symplectic substep, trial collision"}


def wl_sand1m(precision, lib=None, layout="auto", scale=1):
    """The headline scene with Drucker-Prager sand plasticity (friction angle 30
    degrees, beta 1, no cohesion, volume correction) instead of von Mises;
    implicit substep with the reference solver defaults.  scale > 1 keeps
    4 // scale boxes (CPU samples)."""
    x, v = scene(n_boxes=max(1, 4 // scale))
    sim = make_sim(x, v, precision, lib=lib, layout=layout, plastic="drucker_prager")
    return sim, DT, x.shape[0], {"workload": "sand-drucker-prager-4boxes-1m", "model": "hencky+Drucker-Prager",
                                 "solver": "MINRES, Newton 3 x Krylov 20 (reference defaults)"}


def wl_phasefield2m(precision, lib=None, layout="auto", scale=1):
    """The notched slab of damage2m (about 2.05M particles, ends pulled apart at
    +-0.5 m/s, NeoHookeanBorden E = 1e5, nu = 0.3) with the CD-MPM phase field
    instead of Rankine damage: l0 = dx / 2, sigma_c from 1% volumetric stretch,
    parabolic_M = 1, lumped mass, CG tolerance 1e-6 and cap 100 (the fracture
    project's settings).  scale > 1 keeps every scale-th cell layer in z."""
    from . import abi, mpm
    dx = 1.0 / 216
    nx, ny, nz = 216, 54, max(1, 22 // scale)
    lo = np.array([0.25, 0.5, 0.5])
    x = _jitter_box((nx, ny, nz), dx, lo, 8, 4)
    rel = (x - lo) / dx
    notch = (np.abs(rel[:, 0] - nx / 2) < 0.5) & (rel[:, 1] < 0.1 / dx)
    x = x[~notch]
    sim = mpm.MpmSimulation(dx, gravity=(0, 0, 0), precision=precision, grid_log2=9, layout=layout, lib=lib)
    V0 = dx ** 3 / 8
    h = sim.addParticles(x, np.zeros_like(x), 1000.0 * V0, V0)
    h.addFBasedMpmForceWithPhaseField(0.01, 0.5 * dx, mpm.NeoHookeanBorden(1e5, 0.3))
    sim.setPhaseFieldSolver(parabolic_M=1.0, lumping=True)
    hi = lo + np.array([nx, ny, nz]) * dx
    grip = 3 * dx
    for side, vel in ((0, -0.5), (1, 0.5)):
        a = [lo[0] - 4 * dx if side == 0 else hi[0] - grip, lo[1] - 4 * dx, lo[2] - 4 * dx]
        b = [lo[0] + grip if side == 0 else hi[0] + 4 * dx, hi[1] + 4 * dx, hi[2] + 4 * dx]
        box = mpm.AnalyticCollisionObject(mpm.AxisAlignedAnalyticBox(a, b), abi.STICKY)
        box.setTranslation((0.0, 0.0, 0.0), (vel, 0.0, 0.0))
        sim.addCollisionObject(box)
    return sim, 2e-4, x.shape[0], {"workload": "cdmpm-phase-field-notched-slab-2m", "model": "neo-Hookean + CD-MPM phase field",
                                   "solver": "MINRES, Newton 3 x Krylov 20; phase-field CG 1e-6 x 100"}


def wl_rollout256k(precision, lib=None, layout="auto", scale=1, mixed_tol=1e-12):
    """Differentiable rollout: elastic cube of 32^3 cells x 8 ppc = 262,144
    particles (seed 0) at dx = 1/64 (side 0.5, min corner (0.25, 0.125, 0.25)),
    fixed corotated with per-particle E ~ LogNormal(ln 1e4 - 0.3^2/2, 0.3)
    (seed 5), nu = 0.3, initial velocities uniform in [-0.5, 0.5]^3 (seed 6),
    sticky ground y = 0.1, gravity, Newton-CG, dt = 1e-3; loss = |com(x_100) -
    target|^2 with the target drawn from seed 7.  scale > 1 shrinks the cube's
    edge by that factor (CPU samples)."""
    from . import abi, mpm
    dx = 1.0 / 64
    n = 32 // scale
    x = _jitter_box((n, n, n), dx, (0.25, 0.125, 0.25), 8, 0)
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, grid_log2=7, layout=layout, lib=lib)
    V0 = dx ** 3 / 8
    h = sim.addParticles(x, np.zeros_like(x), 1000.0 * V0, V0)
    h.addFBasedMpmForce(mpm.FixedCorotated(1e4, 0.3))
    sim.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    sim.switchLinearSolver(abi.CG)
    sim.newton_tolerance = 1e-12 if precision == "fp64" else mixed_tol
    sim.newton_max_iterations = 30
    sim.krylov_max_iterations = 500
    sim.krylov_tolerance = 1e-30
    return sim, 1e-3, x.shape[0], {"workload": "config4-differentiable-rollout-256k", "model": "fixed corotated, per-particle E",
                                   "solver": "Newton-CG tol 1e-12, adjoint CG rel tol 1e-10",
                                   "steps": 100, "checkpoint_every": 10}


WORKLOADS = {"cube32k": wl_cube32k, "admm500k": wl_admm500k, "damage2m": wl_damage2m, "rollout256k": wl_rollout256k,
             "explicit1m": wl_explicit1m, "sand1m": wl_sand1m, "phasefield2m": wl_phasefield2m}
