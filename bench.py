#!/usr/bin/env python
"""Benchmark of the implicit APIC MPM substep on the 1M-particle elastoplastic
workload: four jittered boxes of 25x25x50 cells x 8 particles (250,000 each),
dx = 1/256, dt = 5e-4, StvkWithHenckyIsotropic E = 5e4, nu = 0.35 with the
von Mises return map (yield stress 150 Pa), gravity, sticky walls 3 dx inside
the unit cube, reference solver settings (MINRES, 3 Newton x 20 Krylov).

A step is one substep of the whole scene.  `value` is mixed-precision substeps/s
(device time, CUDA events on the library's stream); the FP64 substep is timed on
the same scene for the speed-up and the position error between the two.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU runs are independent replicas (the substep has no data-path
collective); rank 0 prints one JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DX = 1.0 / 256
DT = 5e-4
CELLS = (25, 25, 50)
PPC = 8
RHO = 1000.0
E, NU, YIELD = 5e4, 0.35, 150.0
METRIC = "implicit MPM substeps/sec at 1M particles, mixed vs FP64 GPU, at <=1e-6 rel err"
HVP_WORDS = 22  # compulsory words per particle of one Hessian-vector product: X(3), Fn(9), F(9), V0(1)
# DRAM bytes of one product (k_hvp_stress + k_hvp_scatter) per particle, from an
# ncu capture of this workload at 1M particles (228.7 MB;
# profiles/k_hvp_stress_k_hvp_scatter_1M_mixed.md).
HVP_DRAM_BYTES_PER_PARTICLE = 228.7e6 / 1_000_000


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
    from ziran2019_b200 import abi, mpm

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
    from ziran2019_b200 import abi, mpm
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
    from ziran2019_b200 import abi, mpm
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


def wl_damage2m(precision, lib=None, layout="auto", scale=1):
    """Notched slab 1.0 x 0.25 x 0.1 with a 0.1-long, one-cell-wide edge notch at
    mid-length, 8 ppc at dx = 1/216 (216 x 54 x 22 cells, about 2.05M
    particles, seed 4); the end faces are held by sticky boxes moving apart at
    +-0.5 m/s; NeoHookeanBorden E = 1e5, nu = 0.3 with Rankine damage sigma_F =
    1e3 Pa, k = 1e-3; dt = 2e-4, no gravity.  scale > 1 keeps every scale-th
    cell layer in z (CPU samples)."""
    from ziran2019_b200 import abi, mpm
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
    h.addRankineDamage(1e3, residual_phase=1e-3)
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
    from ziran2019_b200 import abi, mpm
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


MIXED_ROLLOUT_TOL = 1e-12


def wl_rollout256k(precision, lib=None, layout="auto", scale=1):
    """Differentiable rollout: elastic cube of 32^3 cells x 8 ppc = 262,144
    particles (seed 0) at dx = 1/64 (side 0.5, min corner (0.25, 0.125, 0.25)),
    fixed corotated with per-particle E ~ LogNormal(ln 1e4 - 0.3^2/2, 0.3)
    (seed 5), nu = 0.3, initial velocities uniform in [-0.5, 0.5]^3 (seed 6),
    sticky ground y = 0.1, gravity, Newton-CG, dt = 1e-3; loss = |com(x_100) -
    target|^2 with the target drawn from seed 7.  scale > 1 shrinks the cube's
    edge by that factor (CPU samples)."""
    from ziran2019_b200 import abi, mpm
    dx = 1.0 / 64
    n = 32 // scale
    x = _jitter_box((n, n, n), dx, (0.25, 0.125, 0.25), 8, 0)
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, grid_log2=7, layout=layout, lib=lib)
    V0 = dx ** 3 / 8
    h = sim.addParticles(x, np.zeros_like(x), 1000.0 * V0, V0)
    h.addFBasedMpmForce(mpm.FixedCorotated(1e4, 0.3))
    sim.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, 0.1, 0), (0, 1, 0)), abi.STICKY))
    sim.switchLinearSolver(abi.CG)
    sim.newton_tolerance = 1e-12 if precision == "fp64" else MIXED_ROLLOUT_TOL
    sim.newton_max_iterations = 30
    sim.krylov_max_iterations = 500
    sim.krylov_tolerance = 1e-30
    return sim, 1e-3, x.shape[0], {"workload": "config4-differentiable-rollout-256k", "model": "fixed corotated, per-particle E",
                                   "solver": "Newton-CG tol 1e-12, adjoint CG rel tol 1e-10",
                                   "steps": 100, "checkpoint_every": 10}


def run_rollout(args, world, rank):
    """Forward + reverse sweep of the 100-substep rollout (mixed and FP64):
    gradient rollouts per second, mixed-vs-FP64 gradient error, and a central
    finite-difference check of the FP64 gradients in random directions."""
    import torch

    from ziran2019_b200 import build
    from ziran2019_b200.rollout import Rollout
    build.build()
    steps, every, NUR = 100, 10, 0.3
    res = {}
    for p in ("fp64", "mixed"):
        sim, dt, P, meta = wl_rollout256k(p, layout="444")
        rng = np.random.default_rng(5)
        E = np.exp(np.log(1e4) - 0.3 ** 2 / 2 + 0.3 * rng.standard_normal(P))
        v0 = np.random.default_rng(6).uniform(-0.5, 0.5, (P, 3))
        target = np.array([0.5, 0.3, 0.5]) + np.random.default_rng(7).uniform(-0.05, 0.05, 3)
        m = np.full(P, 1000.0 * (1.0 / 64) ** 3 / 8)
        ro = Rollout(sim, NUR, dt, steps, checkpoint_every=every, tolerance=1e-10)

        def loss_and_grad(X):
            com = (m[:, None] * X).sum(0) / m.sum()
            return float(((com - target) ** 2).sum()), 2 * (com - target)[None, :] * (m / m.sum())[:, None]
        X = ro.run(E, v0)  # warm-up (allocations, graphs)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        X = ro.run(E, v0)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        fwd_newton = sim.last_stats["newton_iterations"]
        L, gX = loss_and_grad(X)
        gE, gv = ro.backward(gX)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        res[p] = {"forward_s": t1 - t0, "backward_s": t2 - t1, "loss": L, "gE": gE, "gv": gv,
                  "adjoint_cg_iterations": sum(s["krylov_iterations"] for s in ro.stats),
                  "newton_iterations_last_substep": fwd_newton, "newton_tolerance": sim.newton_tolerance}
        if p == "fp64":
            fd_err = []
            drng = np.random.default_rng(11)
            for k in range(args.fd_directions):
                which = "E" if k % 2 == 0 else "v"
                d = drng.standard_normal(E.shape if which == "E" else v0.shape)
                scale_ = 1e4 if which == "E" else 0.5
                h = 1e-4 * scale_
                Ep, vp = (E + h * d, v0) if which == "E" else (E, v0 + h * d)
                Em, vm = (E - h * d, v0) if which == "E" else (E, v0 - h * d)
                fd = (loss_and_grad(ro.run(Ep, vp))[0] - loss_and_grad(ro.run(Em, vm))[0]) / (2 * h)
                an = float(((gE if which == "E" else gv) * d).sum())
                fd_err.append(abs(fd - an) / max(abs(an), 1e-300))
            res[p]["fd_rel_err"] = fd_err
        sim.close()
    r64, rmx = res["fp64"], res["mixed"]
    relE = float(np.linalg.norm(rmx["gE"] - r64["gE"]) / np.linalg.norm(r64["gE"]))
    relv = float(np.linalg.norm(rmx["gv"] - r64["gv"]) / np.linalg.norm(r64["gv"]))
    if rank == 0:
        tot = rmx["forward_s"] + rmx["backward_s"]
        line = {"metric": "differentiable rollouts/sec (100 implicit substeps forward + reverse), config4-differentiable-rollout-256k",
                "value": 1.0 / tot, "unit": "rollouts/s", "n_gpus": world, "steps": steps, "warmup": 1, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "mixed forward (fp32 HVP) + fp64 adjoint vectors", "data": "synthetic",
                "config": dict(meta, particles=P, dt=1e-3),
                "mixed": {k: rmx[k] for k in ("forward_s", "backward_s", "loss", "adjoint_cg_iterations", "newton_iterations_last_substep", "newton_tolerance")},
                "fp64": {k: r64[k] for k in ("forward_s", "backward_s", "loss", "adjoint_cg_iterations", "newton_iterations_last_substep", "newton_tolerance")},
                "fp64_value": 1.0 / (r64["forward_s"] + r64["backward_s"]),
                "grad_rel_err_mixed_vs_fp64": {"E": relE, "v0": relv},
                "fd_check_fp64": {"directions": args.fd_directions, "h": "1e-4 x (1e4 for E, 0.5 for v0)",
                                  "max_rel_err": max(r64["fd_rel_err"]) if r64.get("fd_rel_err") else None,
                                  "rel_err": r64.get("fd_rel_err")}}
        print(json.dumps(line), flush=True)


WORKLOADS = {"cube32k": wl_cube32k, "admm500k": wl_admm500k, "damage2m": wl_damage2m, "rollout256k": wl_rollout256k,
             "explicit1m": wl_explicit1m, "sand1m": wl_sand1m, "phasefield2m": wl_phasefield2m}


def run_workload(args, world, rank):
    """One secondary workload: mixed and FP64 GPU substeps/s, position error
    of mixed against FP64 after the timed steps, and the oracle on a sample."""
    import torch

    from ziran2019_b200 import build
    build.build()
    fn = WORKLOADS[args.workload]
    sims, meta = {}, None
    for p in ("fp64", "mixed"):
        sims[p], dt, P, meta = fn(p, layout="444", scale=args.scale)
    for p in sims:
        for _ in range(args.warmup):
            rc = sims[p].advanceOneTimeStep(dt)
            assert rc == 0, (p, rc, sims[p].last_stats)
    ms64, st64 = timed_steps(sims["fp64"], args.steps, world, dt=dt)
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    ms_mx, st_mx = timed_steps(sims["mixed"], args.steps, world, dt=dt)
    clk = clocks.stop()
    x64 = sims["fp64"].getParticles()["X"]
    xmx = sims["mixed"].getParticles()["X"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import zoracle
        scale = {"cube32k": 1, "admm500k": 4, "damage2m": 11, "explicit1m": 4, "sand1m": 4, "phasefield2m": 11}[args.workload]
        Pc = fn("fp64", lib=zoracle.lib(), scale=scale)[2]
        n, secs, reps = timed_cpu_window(lambda: fn("fp64", lib=zoracle.lib(), scale=scale)[0], dt, args.warmup, args.steps,
                                         args.cpu_seconds)
        cpu = {"value": n / secs * Pc / P, "unit": "substeps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"the timed window ({args.warmup} warm-up + {args.steps} timed substeps) on a {Pc}-particle cut of the "
                         f"workload, {reps}x, oracle port, {secs:.1f} s timed, scaled by {Pc}/{P}"}
    if rank == 0:
        value = world * args.steps / (ms_mx / 1e3)
        fp64_value = world * args.steps / (ms64 / 1e3)
        kind = "explicit" if args.workload == "explicit1m" else "implicit"
        line = {"metric": f"{kind} MPM substeps/sec, {meta['workload']}", "value": value, "unit": "substeps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mx / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "mixed (fp32 operator, fp64 state)", "data": "synthetic",
                "config": dict(meta, particles=P, dt=dt), "particles_substeps_per_s": value * P,
                "fp64_value": fp64_value, "mixed_over_fp64": value / fp64_value,
                "rel_pos_err_vs_fp64": float(np.linalg.norm(xmx - x64) / np.linalg.norm(x64)),
                "accuracy_steps": args.warmup + args.steps,
                "iterations_per_step": [st_mx[-1]["newton_iterations"], st_mx[-1]["krylov_iterations"]],
                "phase_field_cg_iterations": st_mx[-1].get("phase_field_iterations"),
                "gpu_launches": sum(s["kernel_launches"] for s in st_mx), "cpu_baseline": cpu, "clocks": clk}
        print(json.dumps(line), flush=True)
    for s in sims.values():
        s.close()


class Clocks:
    """nvidia-smi samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, n in enumerate(names):
                if r[5 + k].strip().lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup():
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank


def barrier_max(value, world):
    """Barrier and max over ranks (the slowest replica's time)."""
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def timed_steps(sim, steps, world, profile=False, dt=None):
    """Runs `steps` substeps between CUDA events on the library stream; returns ms and stats."""
    import ctypes

    import torch

    from ziran2019_b200 import abi
    sptr = ctypes.c_void_p()
    sim.lib.check(sim.lib.get_stream(sim.ctx, ctypes.byref(sptr)), "get_stream")
    stream = torch.cuda.ExternalStream(sptr.value or 0)
    sim.lib.set_profiling(sim.ctx, 1 if profile else 0)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier_max(0.0, world)
    torch.cuda.synchronize()
    e0.record(stream)
    stats = []
    for _ in range(steps):
        rc = sim.advanceOneTimeStep(DT if dt is None else dt)
        if rc not in (abi.OK, abi.CFL_VIOLATION):
            raise RuntimeError(f"substep status {rc}")
        stats.append(sim.last_stats)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    sim.lib.set_profiling(sim.ctx, 0)
    return barrier_max(ms, world), stats


def substep_algorithmic_bytes(st, P, hvp_word_bytes):
    """Compulsory DRAM bytes of one implicit substep from its data flow, with
    the Newton and Krylov counts the substep took.  Per particle: binning (X
    read; key, index, offset written: 5.5 words), P2G (X, V, C, m: 16), per
    Newton head the update (X, Fn, V0 read, F written: 22) and the force (X,
    stress: 12), per Hessian product 22 words (X, Fn, F, V0) in the product's
    precision, G2P (33) and the return map (21).  Per active grid node: P2G 4,
    per head 9, per product 27 (operator input / output and the MINRES
    vectors), G2P 3 words.  FP64 words unless stated."""
    heads = st["newton_iterations"] + 1
    nh = st["hvp_count"]
    pw = 5.5 + 16 + heads * (22 + 12) + 33 + 21
    nw = 4 + heads * 9 + nh * 27 + 3
    return (P * pw + st["num_nodes"] * nw) * 8 + P * nh * 22 * hvp_word_bytes


def timed_cpu_window(make, dt, warmup, steps, min_seconds, max_repeats=50):
    """The GPU's timed window on the oracle: a fresh scene from make(), `warmup`
    untimed substeps, then `steps` timed ones; repeated until `min_seconds` of
    timed CPU work (at most max_repeats).  Returns (timed substeps, seconds,
    repeats)."""
    secs, n, reps = 0.0, 0, 0
    while reps < max_repeats and (reps == 0 or secs < min_seconds):
        sim = make()
        for _ in range(warmup):
            sim.advanceOneTimeStep(dt)
        t0 = time.perf_counter()
        for _ in range(steps):
            sim.advanceOneTimeStep(dt)
        secs += time.perf_counter() - t0
        n += steps
        reps += 1
        sim.close()
    return n, secs, reps


def cpu_oracle_rate(steps, warmup, velocity="particle", min_seconds=0.0):
    """The oracle (CPU restatement of the reference substep) on one 250k-particle
    box of the same scene, all host threads, over the GPU's timed window;
    returns 1M-equivalent substeps/s, the sample's particles, seconds, timed
    substeps and repeats of the window."""
    from oracle import zoracle
    x, v = scene(n_boxes=1, velocity=velocity)
    n, dt, reps = timed_cpu_window(lambda: make_sim(x, v, "fp64", lib=zoracle.lib()), DT, warmup, steps, min_seconds)
    P = x.shape[0]
    return n / dt * P / 1_000_000, P, dt, n, reps


def run_reference(args, world, rank):
    if rank != 0:
        return
    cores = os.cpu_count()
    rate, P, secs, _, _ = cpu_oracle_rate(args.steps, args.warmup, args.velocity)
    sample = f"{args.steps} substeps of one {P}-particle box of the workload (oracle port, {cores} threads), scaled by {P}/1e6"
    line = {"metric": METRIC, "value": rate, "unit": "substeps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "config1-elastoplastic-4boxes", "particles": 1_000_000, "sample_particles": P},
            "cpu_baseline": {"value": rate, "unit": "substeps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": "substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="the CPU baseline repeats the timed window on the oracle until this much timed CPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--model", default="hencky", choices=["hencky", "nh"])
    ap.add_argument("--velocity", default="particle", choices=["particle", "box"])
    ap.add_argument("--only", default=None, choices=["fp64", "mixed"], help="time one precision (profiling runs)")
    ap.add_argument("--boxes", type=int, default=4, help="boxes of 250k particles (profiling runs use fewer)")
    ap.add_argument("--fp64-layout", default="444", choices=["444", "auto"],
                    help="page layout of the FP64 substep: 444 = same as the mixed run (only precision differs)")
    ap.add_argument("--scale", type=int, default=1,
                    help="secondary workloads: the cut used for CPU samples, on the GPU too (profiling runs)")
    ap.add_argument("--workload", default="config1", choices=["config1"] + sorted(WORKLOADS),
                    help="config1: the headline 1M-particle workload; others print their own line")
    ap.add_argument("--fd-directions", type=int, default=4, help="finite-difference directions of the rollout gradient check")
    ap.add_argument("--rollout-mixed-tol", type=float, default=None, help="Newton tolerance of the mixed rollout forward")
    args = ap.parse_args()
    if args.rollout_mixed_tol is not None:
        global MIXED_ROLLOUT_TOL
        MIXED_ROLLOUT_TOL = args.rollout_mixed_tol
    if args.warmup < 3:
        args.warmup = 3
    world, rank = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "rollout256k":
        run_rollout(args, world, rank)
        return
    if args.workload != "config1":
        run_workload(args, world, rank)
        return

    import torch

    from ziran2019_b200 import build
    build.build()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    x, v = scene(n_boxes=args.boxes, velocity=args.velocity)
    P = x.shape[0]
    precs = [args.only] if args.only else ["fp64", "mixed"]
    sims = {p: make_sim(x, v, p, model=args.model, layout=args.fp64_layout if p == "fp64" else "auto") for p in precs}
    for p in precs:
        for _ in range(args.warmup):
            sims[p].advanceOneTimeStep(DT)
    if args.only:
        ms, st = timed_steps(sims[args.only], args.steps, world)
        _, stp = timed_steps(sims[args.only], 2, world, profile=True)
        if rank == 0:
            print(json.dumps({"only": args.only, "particles": P, "ms_per_step": ms / args.steps,
                              "hvp_ms": sum(s["ms_hvp"] for s in stp) / max(1, sum(s["hvp_timed"] for s in stp)),
                              "launches_per_step": st[-1]["kernel_launches"], "newton_krylov": [st[-1]["newton_iterations"], st[-1]["krylov_iterations"]]}),
                  flush=True)
        return
    ms64, st64 = timed_steps(sims["fp64"], args.steps, world)
    clocks = Clocks(dev)
    clocks.start()
    ms_mx, st_mx = timed_steps(sims["mixed"], args.steps, world)
    clk = clocks.stop()
    # second timed region with each Hessian-vector product bracketed by CUDA
    # events on the library stream (host-driven solver loop), for the roofline
    nprof = max(2, args.steps // 4)
    _, st_prof = timed_steps(sims["mixed"], nprof, world, profile=True)
    value = world * args.steps / (ms_mx / 1e3)
    fp64_value = world * args.steps / (ms64 / 1e3)

    # position error of the mixed substep against the FP64 substep after
    # `accuracy-steps` substeps from the same initial state
    done = {"fp64": args.warmup + args.steps, "mixed": args.warmup + args.steps + nprof}
    total = max(args.accuracy_steps, max(done.values()))
    for p in ("fp64", "mixed"):
        for _ in range(total - done[p]):
            sims[p].advanceOneTimeStep(DT)
    x64 = sims["fp64"].getParticles()["X"]
    xmx = sims["mixed"].getParticles()["X"]
    rel_err = float(np.linalg.norm(xmx - x64) / np.linalg.norm(x64))
    max_abs_dx = float(np.abs(xmx - x64).max() / DX)

    # dominant kernel: the Hessian-vector product
    hvp_ms = sum(s["ms_hvp"] for s in st_prof)
    hvp_n = sum(s["hvp_timed"] for s in st_prof)
    nodes = st_prof[-1]["num_blocks"] * 64
    hvp_bytes = P * HVP_WORDS * 4 + nodes * 3 * 8 * 2
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = hvp_bytes / (hvp_ms / hvp_n / 1e3) / 1e9 if hvp_n else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": HVP_DRAM_BYTES_PER_PARTICLE * P,
                "traffic_source": "ncu dram__bytes_read+write of both kernels at 1M particles",
                "kernel": "k_hvp (FP32 Hessian-vector product)", "bytes_per_launch": hvp_bytes,
                "avg_launch_ms": hvp_ms / hvp_n if hvp_n else None, "peak_source": "measured" if peaks else "fallback"}

    e2e = None
    if not args.no_e2e:
        sim = sims["mixed"]
        pin = {k: torch.empty(s, dtype=torch.float64, pin_memory=True) for k, s in (("X", (P, 3)), ("V", (P, 3)), ("C", (P, 3, 3)), ("F", (P, 3, 3)))}
        cur = sim.getParticles()
        for k in pin:
            pin[k].numpy()[...] = cur[k]
        import ctypes
        sptr = ctypes.c_void_p()
        sim.lib.get_stream(sim.ctx, ctypes.byref(sptr))
        stream = torch.cuda.ExternalStream(sptr.value or 0)
        arrs = {k: t.numpy() for k, t in pin.items()}
        from ziran2019_b200.abi import ptr

        def e2e_step():
            sim._call("set_particles", ptr(arrs["X"]), ptr(arrs["V"]), ptr(arrs["C"]), ptr(arrs["F"]))
            sim.advanceOneTimeStep(DT)
            sim._call("get_particles", ptr(arrs["X"]), ptr(arrs["V"]), ptr(arrs["C"]), ptr(arrs["F"]))
        for _ in range(args.warmup):
            e2e_step()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier_max(0.0, world)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        e1.synchronize()
        ms_e2e = barrier_max(e0.elapsed_time(e1), world)
        e2e = {"value": world * args.steps / (ms_e2e / 1e3), "unit": "substeps/s", "h2d_bytes_per_step": P * 24 * 8,
               "d2h_bytes_per_step": P * 24 * 8}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, Pc, secs, n, reps = cpu_oracle_rate(args.steps, args.warmup, args.velocity, args.cpu_seconds)
        cpu = {"value": rate, "unit": "substeps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"the timed window ({args.warmup} warm-up + {args.steps} timed substeps) on one {Pc}-particle box of the workload, "
                         f"{reps}x, oracle port, {secs:.1f} s timed, scaled by {Pc}/1e6"}

    launches = sum(s["kernel_launches"] for s in st_mx)
    sub_bytes = sum(substep_algorithmic_bytes(s_, P, 4) for s_ in st_mx) / len(st_mx)
    sub_achieved = sub_bytes / (ms_mx / args.steps / 1e3) / 1e9
    substep_roofline = {"bound": "hbm", "algorithmic_bytes": sub_bytes, "achieved": sub_achieved, "peak": peak, "unit": "GB/s",
                        "frac": sub_achieved / peak, "peak_source": roofline["peak_source"],
                        "model": "compulsory particle and node words of binning, P2G, each Newton head, each Hessian product, G2P "
                                 "and the return map, at the substeps' own Newton / Krylov counts"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "substeps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_mx / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 Hessian products, fp64 state/residual/reductions", "data": "synthetic",
            "config": {"workload": "config1-elastoplastic-4boxes", "particles": P, "dx": DX, "dt": DT,
                       "model": f"{args.model}+von Mises", "velocity": args.velocity, "fp64_layout": args.fp64_layout, "solver": "MINRES, Newton 3 x Krylov 20 (reference defaults)",
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (particle state ~300 MB)"},
            "particles_substeps_per_s": value * P,
            "fp64_value": fp64_value, "mixed_over_fp64": value / fp64_value,
            "rel_pos_err_vs_fp64": rel_err, "max_abs_err_over_dx": max_abs_dx, "accuracy_steps": total,
            "newton_krylov_per_step": [st_mx[-1]["newton_iterations"], st_mx[-1]["krylov_iterations"]],
            "roofline": roofline, "substep_roofline": substep_roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    for s in sims.values():
        s.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
