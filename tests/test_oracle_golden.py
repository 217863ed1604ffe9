"""The oracle's SPGrid addressing and binning against outputs of the reference's
own SPGrid code (tests/golden/spgrid_golden.npz, made by make_spgrid_golden.py)."""
import ctypes as C

import numpy as np
import pytest

from ziran2019_b200 import abi, mpm


@pytest.mark.parametrize("name,l2s", [("l7", 7), ("l6", 6)])
def test_masks(oracle, golden, name, l2s):
    m = np.zeros(3, dtype=np.uint64)
    oracle.dll.zoracle_masks(l2s, m.ctypes.data_as(abi.c_uint64_p))
    np.testing.assert_array_equal(m, golden[f"masks_{name}"])


@pytest.mark.parametrize("name,l2s", [("l7", 7), ("l6", 6)])
def test_linear_offset(oracle, golden, name, l2s):
    c = golden["coords"]
    got = np.array([oracle.dll.zoracle_linear_offset(l2s, int(a), int(b), int(d)) for a, b, d in c], dtype=np.uint64)
    np.testing.assert_array_equal(got, golden[f"offsets_{name}"])
    np.testing.assert_array_equal(golden[f"roundtrip_{name}"], c)


@pytest.mark.parametrize("name,l2s", [("l7", 7), ("l6", 6)])
def test_packed_add(oracle, golden, name, l2s):
    a, b, want = golden[f"padd_a_{name}"], golden[f"padd_b_{name}"], golden[f"padd_{name}"]
    got = np.array([oracle.dll.zoracle_packed_add(l2s, int(x), int(y)) for x, y in zip(a[:400], b[:400])], dtype=np.uint64)
    np.testing.assert_array_equal(got, want[:400])


@pytest.mark.parametrize("scene", ["cube", "clusters", "faces"])
@pytest.mark.parametrize("precision,l2s", [("fp64", 7), ("mixed", 6)])
def test_binning_matches_reference(oracle, golden, scene, precision, l2s):
    x = golden[f"scene_{scene}_x"]
    dx = float(golden[f"scene_{scene}_dx"])
    sim = mpm.MpmSimulation(dx, precision=precision, lib=oracle)
    sim.addParticles(x, None, 1.0, 1.0)
    out = sim.binParticles()
    key = f"bin_{scene}_l{l2s}"
    np.testing.assert_array_equal(out["particle_sorter"], golden[key + "_sorter"])
    np.testing.assert_array_equal(out["particle_order"], golden[key + "_order"])
    np.testing.assert_array_equal(out["particle_base_offset"], golden[key + "_base"])
    np.testing.assert_array_equal(out["particle_group"], golden[key + "_groups"])
    np.testing.assert_array_equal(out["block_offset"], golden[key + "_block_offset"])
    np.testing.assert_array_equal(out["page_offsets"], golden[key + "_blocks"])
