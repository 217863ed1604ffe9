"""CUDA binning against the reference's own SPGrid outputs (golden) and the
oracle: keys, order, base offsets, groups and the first-touch page map must be
bit-exact."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import jittered_box

pytestmark = pytest.mark.gpu

FIELDS = ["particle_sorter", "particle_order", "particle_base_offset", "particle_group", "block_offset", "page_offsets"]
GOLD = {"particle_sorter": "_sorter", "particle_order": "_order", "particle_base_offset": "_base",
        "particle_group": "_groups", "block_offset": "_block_offset", "page_offsets": "_blocks"}


def assert_bins_equal(a, b):
    for f in FIELDS:
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)


@pytest.mark.parametrize("scene", ["cube", "clusters", "faces"])
@pytest.mark.parametrize("precision,l2s", [("fp64", 7), ("mixed", 6)])
def test_gpu_binning_matches_reference_golden(cuda_lib, golden, scene, precision, l2s):
    x = golden[f"scene_{scene}_x"]
    dx = float(golden[f"scene_{scene}_dx"])
    sim = mpm.MpmSimulation(dx, precision=precision, grid_log2=9)
    sim.addParticles(x, None, 1.0, 1.0)
    out = sim.binParticles()
    key = f"bin_{scene}_l{l2s}"
    for f in FIELDS:
        np.testing.assert_array_equal(out[f], golden[key + GOLD[f]], err_msg=f)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_binning_large_random_vs_oracle(cuda_lib, oracle, precision):
    rng = np.random.default_rng(11)
    dx = 1.0 / 256
    centers = rng.uniform(0.15, 0.85, size=(12, 3))
    x = np.concatenate([c + rng.normal(scale=0.03, size=(20000, 3)) for c in centers])
    x = np.concatenate([x, jittered_box(20, dx, (0.3, 0.3, 0.3), 8, seed=3)])
    x = x.astype(np.float32).astype(np.float64)
    g = mpm.MpmSimulation(dx, precision=precision, grid_log2=9)
    o = mpm.MpmSimulation(dx, precision=precision, lib=oracle)
    for s in (g, o):
        s.addParticles(x, None, 1.0, 1.0)
    a = g.binParticles()
    assert_bins_equal(a, o.binParticles())
    # binning is deterministic and idempotent on unchanged positions
    assert_bins_equal(a, g.binParticles())


def test_gpu_binning_edge_cases(cuda_lib, oracle):
    dx = 1.0 / 64
    cases = [
        np.array([[0.5, 0.5, 0.5]]),                                 # one particle
        np.tile([[0.25, 0.25, 0.25]], (100, 1)),                      # one cell, equal positions
        np.array([[2.5 * dx, 0.5, 0.5], [0.5, 2.5 * dx, 0.5]]),       # near the low domain edge
    ]
    for x in cases:
        g = mpm.MpmSimulation(dx, precision="fp64", grid_log2=8)
        o = mpm.MpmSimulation(dx, precision="fp64", lib=oracle)
        for s in (g, o):
            s.addParticles(x, None, 1.0, 1.0)
        assert_bins_equal(g.binParticles(), o.binParticles())


def test_gpu_out_of_grid_is_an_error(cuda_lib):
    sim = mpm.MpmSimulation(1.0 / 64, precision="fp64", grid_log2=6)  # 64 nodes per axis
    sim.addParticles(np.array([[0.5, 0.5, 0.5], [0.99, 0.5, 0.5]]), None, 1.0, 1.0)
    with pytest.raises(abi.ZmpmError) as e:
        sim.binParticles()
    assert e.value.status == abi.OUT_OF_GRID
    sim2 = mpm.MpmSimulation(1.0 / 64, precision="fp64", grid_log2=8)
    sim2.addParticles(np.array([[-0.1, 0.5, 0.5]]), None, 1.0, 1.0)
    with pytest.raises(abi.ZmpmError):
        sim2.binParticles()
