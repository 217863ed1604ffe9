"""The GPU substep against the FP64 oracle at the benchmark configurations:
config 0 in full (32,768 particles, 50 substeps), config 1 as one of its four
250,000-particle boxes (50 substeps), config 2 as a 31,104-particle cut of the
slab (10 ADMM substeps) and config 3 as a 93,144-particle one-cell-thick layer
of the notched slab (20 substeps).  Same seeded scenes, solver settings and
substep counts on both sides; positions and velocities are compared as
relative L2 errors over all particles, for the FP64 and the mixed substep.

FP64 against FP64 differs only in the order of floating-point sums (atomic
scatters and tree reductions on the GPU, the 8-colour schedule and OpenMP
reductions in the oracle): measured 1e-17 to 3e-16 in positions and 1e-15 to
4e-14 in velocities, bounded here at 1e-13 and 1e-11.  The mixed substep
(FP32 particle, grid and Hessian arithmetic) is bounded by the benchmark's
1e-6 relative position error and 1e-4 in velocities."""
import numpy as np
import pytest

from ziran2019_b200 import workloads

pytestmark = pytest.mark.gpu


def l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def advance(sim, dt, steps):
    for n in range(steps):
        rc = sim.advanceOneTimeStep(dt)
        assert rc in (0, 1), (n, rc, sim.last_stats)
    st = sim.getParticles()
    sim.close()
    return st


def compare(build, dt, steps, oracle, tol):
    """build(precision, lib) -> simulation.  tol: {precision: (position, velocity)}."""
    ref = advance(build("fp64", oracle), dt, steps)
    errs = {}
    for p in ("fp64", "mixed"):
        st = advance(build(p, None), dt, steps)
        errs[p] = (l2(st["X"], ref["X"]), l2(st["V"], ref["V"]))
    print("parity", errs)
    for p, (ex, ev) in errs.items():
        assert ex < tol[p][0] and ev < tol[p][1], (p, errs)
    return errs


def test_config0_cube_32k_50_substeps(cuda_lib, oracle):
    def build(p, lib):
        return workloads.wl_cube32k(p, lib=lib, layout="444" if lib is None else "auto")[0]
    compare(build, 1e-3, 50, oracle, {"fp64": (1e-13, 1e-11), "mixed": (1e-6, 1e-4)})


def test_config1_box_250k_50_substeps(cuda_lib, oracle):
    x, v = workloads.scene(n_boxes=1)

    def build(p, lib):
        return workloads.make_sim(x, v, p, lib=lib, layout="444" if lib is None else "auto")
    compare(build, workloads.DT, 50, oracle, {"fp64": (1e-13, 1e-11), "mixed": (1e-6, 1e-4)})


def test_config2_admm_slab_cut_10_substeps(cuda_lib, oracle):
    def build(p, lib):
        return workloads.wl_admm500k(p, lib=lib, layout="444" if lib is None else "auto", scale=4)[0]
    compare(build, 2e-3, 10, oracle, {"fp64": (1e-13, 1e-11), "mixed": (1e-6, 1e-4)})


def test_config3_damage_slab_layer_20_substeps(cuda_lib, oracle):
    def build(p, lib):
        return workloads.wl_damage2m(p, lib=lib, layout="444" if lib is None else "auto", scale=22)[0]
    compare(build, 2e-4, 20, oracle, {"fp64": (1e-13, 1e-11), "mixed": (1e-6, 1e-4)})
