"""The allocation-free key sort (zmpm_sort_keys_noalloc) against the binning of a
context (zmpm_bin), through the C ABI, on two calls in a row.

The entry point serves callers that cannot call cudaMalloc: the caller owns the
input and output device buffers (allocated here by torch, as such a host would
with its own allocator) and the library works in a fixed scratch array.  The
keys are integers, so the comparison is bit-exact.  This file is collected
last so that a run stopping at the first failure has run every other test."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import jittered_box

pytestmark = pytest.mark.gpu


def context_keys(x, dx, precision):
    sim = mpm.MpmSimulation(dx, precision=precision, grid_log2=9)
    sim.addParticles(x, None, 1.0, 1.0)
    return sim.binParticles()["particle_sorter"]


def noalloc_keys(lib, x, dx, precision):
    import torch
    xd = torch.tensor(np.ascontiguousarray(x, dtype=np.float64), device="cuda")
    kd = torch.empty(x.shape[0], dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream()
    prec = abi.FP64 if precision == "fp64" else abi.MIXED
    rc = lib.sort_keys_noalloc(xd.data_ptr(), x.shape[0], dx, prec, abi.LAYOUT_AUTO, 9, kd.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    assert rc == abi.OK, rc
    return kd.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_sort_matches_context_binning(cuda_lib, precision):
    dx = 1.0 / 256
    rng = np.random.default_rng(42)
    a = np.concatenate([c + rng.normal(scale=0.02, size=(30000, 3)) for c in rng.uniform(0.2, 0.8, size=(5, 3))])
    b = jittered_box((20, 30, 40), dx, (0.3, 0.2, 0.25), 8, seed=5)  # 192,000 particles
    for x in (a, b):  # two calls in a row; the second must not see the first's scratch
        x = x.astype(np.float32).astype(np.float64)
        np.testing.assert_array_equal(noalloc_keys(cuda_lib, x, dx, precision), context_keys(x, dx, precision))


def test_noalloc_rejects_oversize_and_bad_input(cuda_lib):
    import torch
    n = abi.NOALLOC_MAX_PARTICLES + 1
    xd = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    kd = torch.empty(n, dtype=torch.int64, device="cuda")
    rc = cuda_lib.sort_keys_noalloc(xd.data_ptr(), n, 1.0 / 64, abi.FP64, abi.LAYOUT_AUTO, 9, kd.data_ptr(), None)
    assert rc == abi.BAD_ARG
    for bad in ([-0.5, 0.5, 0.5], [0.5, np.nan, 0.5], [np.inf, 0.5, 0.5]):
        x = np.array([[0.5, 0.5, 0.5], bad])
        xd = torch.tensor(x, device="cuda")
        kd = torch.empty(2, dtype=torch.int64, device="cuda")
        rc = cuda_lib.sort_keys_noalloc(xd.data_ptr(), 2, 1.0 / 64, abi.FP64, abi.LAYOUT_AUTO, 9, kd.data_ptr(), None)
        assert rc == abi.OUT_OF_GRID, bad
