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

from ziran2019_b200.workloads import CELLS, DT, DX, PPC, RHO, WORKLOADS, make_sim, scene  # noqa: E402,F401
from ziran2019_b200 import workloads  # noqa: E402

METRIC = "implicit MPM substeps/sec at 1M particles, mixed vs FP64 GPU, at <=1e-6 rel err"
HVP_WORDS = 22  # compulsory words per particle of one Hessian-vector product: X(3), Fn(9), F(9), V0(1)
KRYLOV_NODE_WORDS = 27  # compulsory FP64 words per active node of one MINRES iteration's node passes
SOLVE_KERNELS = ("k_mr_persistent",)  # the persistent linear solve (one launch per Newton iteration)
FD_STEPS = (1e-3, 1e-4, 1e-5)  # finite-difference steps of the rollout gradient check, relative to the parameter scale


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
        sim, dt, P, meta = workloads.wl_rollout256k(p, layout="444", mixed_tol=args.rollout_mixed_tol)
        rng = np.random.default_rng(5)
        E = np.exp(np.log(1e4) - 0.3 ** 2 / 2 + 0.3 * rng.standard_normal(P))
        v0 = np.random.default_rng(6).uniform(-0.5, 0.5, (P, 3))
        target = np.array([0.5, 0.3, 0.5]) + np.random.default_rng(7).uniform(-0.05, 0.05, 3)
        m = np.full(P, 1000.0 * (1.0 / 64) ** 3 / 8)
        ro = Rollout(sim, NUR, dt, steps, checkpoint_every=every, tolerance=1e-10)

        def loss_and_grad(X):
            com = (m[:, None] * X).sum(0) / m.sum()
            return float(((com - target) ** 2).sum()), 2 * (com - target)[None, :] * (m / m.sum())[:, None]
        X = ro.run(E, v0)  # warm-up forward and reverse (allocations, graphs, first launches)
        ro.backward(loss_and_grad(X)[1])
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
            # central differences in random directions (alternately of E and of
            # v0) at three step sizes relative to the parameter's scale
            fd_err = {h: [] for h in FD_STEPS}
            drng = np.random.default_rng(11)
            for k in range(args.fd_directions):
                which = "E" if k % 2 == 0 else "v"
                d = drng.standard_normal(E.shape if which == "E" else v0.shape)
                scale_ = 1e4 if which == "E" else 0.5
                an = float(((gE if which == "E" else gv) * d).sum())
                for hrel in FD_STEPS:
                    h = hrel * scale_
                    Ep, vp = (E + h * d, v0) if which == "E" else (E, v0 + h * d)
                    Em, vm = (E - h * d, v0) if which == "E" else (E, v0 - h * d)
                    fd = (loss_and_grad(ro.run(Ep, vp))[0] - loss_and_grad(ro.run(Em, vm))[0]) / (2 * h)
                    fd_err[hrel].append(abs(fd - an) / max(abs(an), 1e-300))
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
                "fd_check_fp64": {"directions": args.fd_directions, "h": f"{list(FD_STEPS)} x (1e4 for E, 0.5 for v0)",
                                  "max_rel_err_per_h": {str(h): max(v) for h, v in r64["fd_rel_err"].items()} if args.fd_directions else None,
                                  "max_rel_err_best_h": max(min(v[k] for v in r64["fd_rel_err"].values()) for k in range(args.fd_directions))
                                  if args.fd_directions else None,
                                  "rel_err": {str(h): v for h, v in r64["fd_rel_err"].items()}}}
        print(json.dumps(line), flush=True)


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
    clocks = Clocks(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    time.sleep(1.0)
    ms64, st64 = timed_steps(sims["fp64"], args.steps, world, dt=dt)
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
                "rankine_first_not_max": st_mx[-1].get("rankine_first_not_max"),
                "svd_fp64_reevaluations": st_mx[-1].get("svd_fp64_reevaluations"),
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


def oracle_lib_native(wait_for=None):
    """The oracle built for this host (-march=native), waiting for its build."""
    from oracle import zoracle
    if wait_for is not None:
        wait_for.wait()
    return zoracle.lib(native=True)


def oracle_run(x, v, steps, warmup, timed, model, lib):
    """The full workload on the oracle (FP64, all host threads): `steps`
    substeps from the initial state (x, v); substeps warmup+1 .. warmup+timed
    are timed (the window of the GPU's timed region).  Returns (final state,
    timed substeps, seconds)."""
    sim = make_sim(x, v, "fp64", lib=lib, model=model)
    timed = min(timed, steps - warmup)
    for _ in range(warmup):
        sim.advanceOneTimeStep(DT)
    t0 = time.perf_counter()
    for _ in range(timed):
        sim.advanceOneTimeStep(DT)
    secs = time.perf_counter() - t0
    for _ in range(steps - warmup - timed):
        sim.advanceOneTimeStep(DT)
    st = sim.getParticles()
    st["yield_active"] = yield_active(st["F"], model)
    sim.close()
    return st, timed, secs


def yield_active(F, model):
    """Particles on the von Mises yield surface: |dev Hencky strain| >= tau_Y / (2 mu)
    up to 1e-9 relative (VonMisesStvkHencky::projectStrain, PlasticityApplier.cpp:
    462-502, projected them in their last substep)."""
    if model != "hencky":
        return None
    s = np.linalg.svd(F, compute_uv=False)
    eps = np.log(np.maximum(np.abs(s), 1e-4))
    dev = eps - eps.mean(1, keepdims=True)
    mu = workloads.E / (2 * (1 + workloads.NU))
    return np.linalg.norm(dev, axis=1) >= (workloads.YIELD / (2 * mu)) * (1 - 1e-9)


def accuracy_vs_oracle(states, ref):
    """Relative L2 errors of positions and velocities against the FP64 oracle,
    the largest position error in cells, and the particles whose von Mises
    branch (projected or not in the last substep) differs from the oracle's."""
    out = {}
    for p, st in states.items():
        row = {"rel_pos_err": float(np.linalg.norm(st["X"] - ref["X"]) / np.linalg.norm(ref["X"])),
               "rel_vel_err": float(np.linalg.norm(st["V"] - ref["V"]) / np.linalg.norm(ref["V"])),
               "max_abs_pos_err_over_dx": float(np.abs(st["X"] - ref["X"]).max() / DX)}
        if ref.get("yield_active") is not None and st.get("yield_active") is not None:
            row["yield_branch_disagreements"] = int(np.count_nonzero(st["yield_active"] != ref["yield_active"]))
            row["yield_active_particles_oracle"] = int(np.count_nonzero(ref["yield_active"]))
        out[p] = row
    return out


def ncu_traffic(path, kernels):
    """DRAM bytes (read + write) of `kernels` summed over every captured launch,
    from an ncu CSV (--metrics dram__bytes_read.sum,dram__bytes_write.sum --csv)."""
    import csv
    per = {}
    with open(path) as f:
        rows = [r for r in csv.reader(f) if len(r) > 5]
    head = rows[0]
    ik, im, iv, iu = head.index("Kernel Name"), head.index("Metric Name"), head.index("Metric Value"), head.index("Metric Unit")
    scale = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9, "B": 1}
    for r in rows[1:]:
        name = r[ik].split("<")[0].split("(")[0].replace("void ", "").strip().split("::")[-1]
        if name in kernels and r[im] in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            per.setdefault(name, []).append(float(r[iv].replace(",", "")) * scale.get(r[iu], 1))
    if not per:
        return None
    return sum(sum(v) for v in per.values())


def run_reference(args, world, rank):
    """The reference's CPU path on the host cores: the oracle (the CPU
    restatement of the reference substep, built for this host) on the full
    1M-particle workload, all threads; `warmup` untimed then `steps` timed
    substeps.  Rank 0 only."""
    if rank != 0:
        return
    cores = os.cpu_count()
    lib = oracle_lib_native(oracle_build_process())
    x, v = scene(n_boxes=args.boxes, velocity=args.velocity)
    P = x.shape[0]
    _, n, secs = oracle_run(x, v, args.warmup + args.steps, args.warmup, args.steps, args.model, lib)
    rate = n / secs
    sample = (f"{args.steps} timed substeps (after {args.warmup} warm-up) of the full {P}-particle workload, oracle port "
              f"({'-march=native' if lib.native else 'portable build'}), {cores} threads")
    line = {"metric": METRIC, "value": rate, "unit": "substeps/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * secs / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "config1-elastoplastic-4boxes", "particles": P, "model": f"{args.model}+von Mises"},
            "cpu_baseline": {"value": rate, "unit": "substeps/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": rate, "unit": "substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def oracle_build_process():
    from oracle import zoracle
    return zoracle.build_native_async()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--accuracy-steps", type=int, default=100)
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="secondary workloads: the CPU baseline repeats the timed window on the oracle until this much timed CPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the FP64 oracle run (accuracy against the oracle and the CPU baseline)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--model", default="hencky", choices=["hencky", "nh"])
    ap.add_argument("--velocity", default="particle", choices=["particle", "box"])
    ap.add_argument("--only", default=None, choices=["fp64", "mixed"], help="time one precision (profiling runs)")
    ap.add_argument("--host-loop", action="store_true",
                    help="with --only: host-driven solver loops (every kernel a plain launch, for ncu launch lists)")
    ap.add_argument("--boxes", type=int, default=4, help="boxes of 250k particles (profiling runs use fewer)")
    ap.add_argument("--fp64-layout", default="444", choices=["444", "auto"],
                    help="page layout of the FP64 substep: 444 = same as the mixed run (only precision differs)")
    ap.add_argument("--scale", type=int, default=1,
                    help="secondary workloads: the cut used for CPU samples, on the GPU too (profiling runs)")
    ap.add_argument("--workload", default="config1", choices=["config1"] + sorted(WORKLOADS),
                    help="config1: the headline 1M-particle workload; others print their own line")
    ap.add_argument("--fd-directions", type=int, default=16, help="finite-difference directions of the rollout gradient check")
    ap.add_argument("--rollout-mixed-tol", type=float, default=1e-12, help="Newton tolerance of the mixed rollout forward")
    ap.add_argument("--ncu-csv", default=None,
                    help="ncu CSV (dram__bytes_read.sum, dram__bytes_write.sum) of every persistent-solve launch of a run of "
                         "this workload: fills roofline.traffic (per Krylov iteration)")
    ap.add_argument("--ncu-iterations", type=int, default=None,
                    help="Krylov iterations the launches in --ncu-csv ran")
    ap.add_argument("--ncu-particles", type=int, default=None,
                    help="particles of the workload that --ncu-csv captured (its traffic is scaled to this run by particle count)")
    args = ap.parse_args()
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
    want_oracle = rank == 0 and world == 1 and not args.no_cpu_baseline and not args.only
    # the oracle's host build (about 20 s of one core) overlaps the scene setup
    # and ends before any timed region
    oracle_build = oracle_build_process() if want_oracle else None
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    x, v = scene(n_boxes=args.boxes, velocity=args.velocity)
    P = x.shape[0]
    precs = [args.only] if args.only else ["fp64", "mixed"]
    sims = {p: make_sim(x, v, p, model=args.model, layout=args.fp64_layout if p == "fp64" else "auto") for p in precs}
    for p in precs:
        for _ in range(args.warmup):
            sims[p].advanceOneTimeStep(DT)
    if oracle_build is not None:
        oracle_build.wait()
    if args.only:
        ms, st = timed_steps(sims[args.only], args.steps, world, profile=args.host_loop)
        _, stp = timed_steps(sims[args.only], 2, world, profile=True)
        if rank == 0:
            print(json.dumps({"only": args.only, "particles": P, "ms_per_step": ms / args.steps, "host_loop": args.host_loop,
                              "iteration_ms": sum(s["ms_hvp"] for s in stp) / max(1, sum(s["hvp_timed"] for s in stp)),
                              "launches_per_step": st[-1]["kernel_launches"], "newton_krylov": [st[-1]["newton_iterations"], st[-1]["krylov_iterations"]],
                              "krylov_iterations_host_loop": sum(x["krylov_iterations"] for x in (st if args.host_loop else []) + stp)}),
                  flush=True)
        return
    # nvidia-smi samples through both timed regions; it starts a second ahead
    # so that its start-up is outside them
    clocks = Clocks(dev)
    clocks.start()
    time.sleep(1.0)
    ms64, st64 = timed_steps(sims["fp64"], args.steps, world)
    ms_mx, st_mx = timed_steps(sims["mixed"], args.steps, world)
    clk = clocks.stop()
    # second timed region with each Hessian-vector product bracketed by CUDA
    # events on the library stream (host-driven solver loop), for the roofline
    nprof = max(2, args.steps // 4)
    _, st_prof = timed_steps(sims["mixed"], nprof, world, profile=True)
    value = world * args.steps / (ms_mx / 1e3)
    fp64_value = world * args.steps / (ms64 / 1e3)

    # dominant kernel: the persistent MINRES solve (one launch per Newton
    # iteration), measured per Krylov iteration: one Hessian-vector product
    # (HVP_WORDS per particle in FP32) and the node passes (KRYLOV_NODE_WORDS
    # FP64 words per active node)
    solve_ms = sum(s["ms_hvp"] for s in st_prof)
    iters = sum(s["hvp_timed"] for s in st_prof)
    nodes = st_prof[-1]["num_nodes"]
    iter_bytes = P * HVP_WORDS * 4 + nodes * KRYLOV_NODE_WORDS * 8
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = iter_bytes / (solve_ms / iters / 1e3) / 1e9 if iters else None
    traffic = None
    if args.ncu_csv and args.ncu_iterations:
        t = ncu_traffic(args.ncu_csv, SOLVE_KERNELS)
        if t is not None:
            traffic = t / args.ncu_iterations * (P / args.ncu_particles if args.ncu_particles else 1.0)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "traffic": traffic,
                "traffic_source": (f"ncu dram__bytes_read+write of every k_mr_persistent launch in {args.ncu_csv}, per Krylov "
                                   f"iteration ({args.ncu_iterations} iterations), scaled by particle count"
                                   if traffic is not None else "no ncu capture in this run"),
                "kernel": "persistent MINRES solve (k_mr_persistent), per Krylov iteration: Hessian-vector product, "
                          "operator pass, Lanczos step",
                "bytes_per_iteration": iter_bytes, "avg_iteration_ms": solve_ms / iters if iters else None,
                "iterations_timed": iters, "peak_source": "measured" if peaks else "fallback"}

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

    # accuracy after `accuracy-steps` substeps from the initial state: both GPU
    # runs against each other and (rank 0, one GPU) against the FP64 oracle
    sims_acc = {p: make_sim(x, v, p, model=args.model, layout=args.fp64_layout if p == "fp64" else "auto") for p in ("fp64", "mixed")}
    states = {}
    for p, s_ in sims_acc.items():
        for _ in range(args.accuracy_steps):
            rc = s_.advanceOneTimeStep(DT)
            if rc not in (0, 1):
                raise RuntimeError(f"accuracy run ({p}): substep status {rc}")
        states[p] = s_.getParticles()
        states[p]["yield_active"] = yield_active(states[p]["F"], args.model)
        s_.close()
    rel_err = float(np.linalg.norm(states["mixed"]["X"] - states["fp64"]["X"]) / np.linalg.norm(states["fp64"]["X"]))
    max_abs_dx = float(np.abs(states["mixed"]["X"] - states["fp64"]["X"]).max() / DX)
    cpu, vs_oracle = None, None
    if want_oracle:
        lib = oracle_lib_native()
        ref, n, secs = oracle_run(x, v, args.accuracy_steps, args.warmup, args.steps, args.model, lib)
        vs_oracle = accuracy_vs_oracle(states, ref)
        cpu = {"value": n / secs, "unit": "substeps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"substeps {args.warmup + 1}..{args.warmup + n} (the GPU's timed window) of the {args.accuracy_steps}-substep "
                         f"accuracy run of the full {P}-particle workload on the oracle "
                         f"({'-march=native' if lib.native else 'portable build'}, {os.cpu_count()} threads), {secs:.1f} s"}

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
            "dtype": "mixed: fp32 particle/grid/Hessian arithmetic, fp64 positions, residual and reductions", "data": "synthetic",
            "config": {"workload": "config1-elastoplastic-4boxes", "particles": P, "dx": DX, "dt": DT,
                       "model": f"{args.model}+von Mises", "velocity": args.velocity, "fp64_layout": args.fp64_layout, "solver": "MINRES, Newton 3 x Krylov 20 (reference defaults)",
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (particle state ~300 MB)"},
            "particles_substeps_per_s": value * P,
            "fp64_value": fp64_value, "mixed_over_fp64": value / fp64_value,
            "ms_per_step_fp64": ms64 / args.steps,
            "rel_pos_err_vs_fp64": rel_err, "max_abs_err_over_dx": max_abs_dx, "accuracy_steps": args.accuracy_steps,
            "vs_oracle": vs_oracle,
            "rel_pos_err_vs_oracle": vs_oracle["mixed"]["rel_pos_err"] if vs_oracle else None,
            "rel_vel_err_vs_oracle": vs_oracle["mixed"]["rel_vel_err"] if vs_oracle else None,
            "newton_krylov_per_step": [st_mx[-1]["newton_iterations"], st_mx[-1]["krylov_iterations"]],
            "newton_krylov_per_step_fp64": [st64[-1]["newton_iterations"], st64[-1]["krylov_iterations"]],
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
