"""CUDA P2G, Newton-objective residual and Hessian-vector product against the
oracle on the same seeded scenes (FP64: summation order is the only difference;
MIXED: the HVP runs in FP32)."""
import numpy as np
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene, jittered_box

pytestmark = pytest.mark.gpu

KINDS = ["fcr", "nh", "hencky"]


def pair(oracle, kind, precision="fp64", seed=0):
    dx = 1.0 / 64
    g = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision=precision, grid_log2=8)
    o = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", lib=oracle)
    rng = np.random.default_rng(seed)
    for s in (g, o):
        build_scene(s, kind=kind, n=6, dx=dx, seed=seed)
    P = g.count
    F = np.eye(3) + 0.05 * rng.standard_normal((P, 3, 3))
    Cm = 0.5 * rng.standard_normal((P, 3, 3))
    for s in (g, o):
        s.setParticles(F=F, C=Cm)
    return g, o


def by_coord(sim):
    m, v, c = sim.getGrid()
    key = (c[:, 0].astype(np.int64) << 40) | (c[:, 1].astype(np.int64) << 20) | c[:, 2].astype(np.int64)
    order = np.argsort(key)
    return order, m[order], v[order], c[order]


@pytest.mark.parametrize("kind", KINDS)
def test_p2g_grid_matches_oracle(cuda_lib, oracle, kind):
    g, o = pair(oracle, kind)
    assert g.beginImplicit(1e-3) == o.beginImplicit(1e-3)
    gm, gv, gc = g.getGrid()
    om, ov, oc = o.getGrid()
    np.testing.assert_array_equal(gc, oc)  # same nodes in the same getNumNodes order
    np.testing.assert_allclose(gm, om, rtol=1e-13, atol=0)
    np.testing.assert_allclose(gv, ov, rtol=1e-11, atol=1e-12 * np.abs(ov).max())
    gdv, gcol = g.getInitialDv()
    odv, ocol = o.getInitialDv()
    np.testing.assert_array_equal(gcol, ocol)
    assert gcol.sum() > 0
    np.testing.assert_allclose(gdv, odv, rtol=1e-11, atol=1e-12)


def test_p2g_mixed_matches_fp64_oracle(cuda_lib, oracle):
    """MIXED P2G against the FP64 oracle, nodes matched by coordinate (4x4x4
    against 2x4x4 pages); FP32-level agreement."""
    g, o = pair(oracle, "hencky", precision="mixed", seed=5)
    assert g.beginImplicit(1e-3) == o.beginImplicit(1e-3)
    _, gm, gv, gc = by_coord(g)
    _, om, ov, oc = by_coord(o)
    np.testing.assert_array_equal(gc, oc)
    np.testing.assert_allclose(gm, om, rtol=2e-6, atol=1e-6 * om.max())
    np.testing.assert_allclose(gv, ov, rtol=0, atol=2e-6 * np.abs(ov).max())


@pytest.mark.parametrize("kind", KINDS)
def test_residual_and_hvp_match_oracle_fp64(cuda_lib, oracle, kind):
    g, o = pair(oracle, kind, seed=1)
    N = g.beginImplicit(1e-3)
    assert N == o.beginImplicit(1e-3)
    rng = np.random.default_rng(2)
    dv = 0.01 * rng.standard_normal((N, 3))
    rg, ng = g.residual(dv)
    ro, no = o.residual(dv)
    scale = np.abs(ro).max()
    np.testing.assert_allclose(rg, ro, rtol=0, atol=1e-10 * scale)
    assert abs(ng - no) <= 1e-10 * no
    x = rng.standard_normal((N, 3))
    bg = g.multiply(x)
    bo = o.multiply(x)
    np.testing.assert_allclose(bg, bo, rtol=0, atol=1e-10 * np.abs(bo).max())


@pytest.mark.parametrize("kind", KINDS)
def test_hvp_fp32_mixed_matches_fp64_oracle(cuda_lib, oracle, kind):
    """MIXED contexts use 4x4x4 pages, so nodes are matched by coordinate."""
    g, o = pair(oracle, kind, precision="mixed", seed=3)
    N = g.beginImplicit(1e-3)
    assert N == o.beginImplicit(1e-3)
    og, _, _, cg = by_coord(g)
    oo, _, _, co = by_coord(o)
    np.testing.assert_array_equal(cg, co)
    rng = np.random.default_rng(4)
    dv_sorted = 0.01 * rng.standard_normal((N, 3))
    dv_g = np.empty_like(dv_sorted)
    dv_o = np.empty_like(dv_sorted)
    dv_g[og] = dv_sorted
    dv_o[oo] = dv_sorted
    rg, ng = g.residual(dv_g)
    ro, no = o.residual(dv_o)
    # MIXED: particle stress in FP32 (FP64 for near-degenerate SVDs), force sums and
    # residual assembly in FP64.  The residual is a difference of much larger force
    # sums, so the FP32 stress round-off reaches it amplified: bound 2e-5 of the
    # largest entry, as for the FP32 product below
    np.testing.assert_allclose(rg[og], ro[oo], rtol=0, atol=2e-5 * np.abs(ro).max())
    assert abs(ng - no) <= 2e-5 * no
    x_sorted = rng.standard_normal((N, 3))
    xg = np.empty_like(x_sorted)
    xo = np.empty_like(x_sorted)
    xg[og] = x_sorted
    xo[oo] = x_sorted
    bg = g.multiply(xg, fp32=True)[og]
    bo = o.multiply(xo)[oo]
    # FP32 Hessian-vector product: relative error bound 2e-5 of the largest entry
    np.testing.assert_allclose(bg, bo, rtol=0, atol=2e-5 * np.abs(bo).max())


def test_hvp_is_symmetric(cuda_lib, oracle):
    g, _ = pair(oracle, "hencky", seed=5)
    N = g.beginImplicit(1e-3)
    rng = np.random.default_rng(6)
    g.residual(np.zeros((N, 3)))
    a, b = rng.standard_normal((N, 3)), rng.standard_normal((N, 3))
    ab = (a * g.multiply(b)).sum()
    ba = (b * g.multiply(a)).sum()
    assert abs(ab - ba) <= 1e-10 * max(abs(ab), abs(ba))
