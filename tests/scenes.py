"""Seeded synthetic scenes shared by the tests (shapes of the benchmark configs)."""
import numpy as np

from ziran2019_b200 import abi, mpm


def jittered_box(cells, dx, lo, ppc=8, seed=0):
    """Particles jittered uniformly inside each cell of a box of `cells` cells."""
    rng = np.random.default_rng(seed)
    cells = np.atleast_1d(cells)
    if cells.size == 1:
        cells = np.repeat(cells, 3)
    grid = np.stack(np.meshgrid(*[np.arange(c) for c in cells], indexing="ij"), -1).reshape(-1, 3)
    x = (np.repeat(grid, ppc, 0) + rng.random((grid.shape[0] * ppc, 3))) * dx + np.asarray(lo, dtype=np.float64)
    return x


def build_scene(sim, kind="fcr", n=8, dx=1.0 / 64, ppc=8, seed=0, v0=(0.3, -1.0, 0.2), E=1e4, nu=0.3,
                plastic=None, ground=0.1, walls=False, lo=(0.375, 0.105, 0.375)):
    x = jittered_box(n, dx, lo, ppc, seed)
    V0 = dx ** 3 / ppc
    v = np.tile(np.asarray(v0, dtype=np.float64), (x.shape[0], 1))
    h = sim.addParticles(x, v, 1000.0 * V0, V0)
    model = {"fcr": mpm.FixedCorotated, "nh": mpm.NeoHookeanBorden, "hencky": mpm.StvkWithHenckyIsotropic}[kind](E, nu)
    h.addFBasedMpmForce(model)
    if plastic is not None:
        h.addPlasticity(model, mpm.VonMisesStvkHencky(plastic, 1e30, 0.0))
    if ground is not None:
        sim.addCollisionObject(mpm.AnalyticCollisionObject(mpm.HalfSpace((0, ground, 0), (0, 1, 0)), abi.STICKY))
    if walls:
        mpm.add_all_walls_in_domain(sim, 1.0, 3 * dx, abi.STICKY)
    return h, x


def make_pair(oracle_lib, precision="fp64", dx=1.0 / 64, grid_log2=8, **kw):
    """The same scene in the CUDA library and in the oracle."""
    g = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, grid_log2=grid_log2)
    o = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64" if precision == "fp64" else "mixed", lib=oracle_lib)
    build_scene(g, dx=dx, **kw)
    build_scene(o, dx=dx, **kw)
    return g, o
