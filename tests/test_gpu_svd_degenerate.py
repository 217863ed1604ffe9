"""Constitutive updates at singular values where FP32 arithmetic is not
enough: inverted F (negative sigma2), near-singular F, a strong stretch
(sigma0 >= 5), and repeated singular values, through the Newton objective's
residual and Hessian-vector product hooks against the FP64 oracle.  The SVD
follows ImplicitQRSVD.h:354-532 (its degenerate bidiagonal branches at
:417-523); the SVD-based models are StvkWithHenckyIsotropic and fixed
corotated.

FP64: the GPU matches the FP64 oracle to round-off.  MIXED: the FP32 update
redoes particles whose FP32 singular values are near inversion (|sigma2| <=
0.2) or strongly stretched (sigma0 >= 5) in FP64 (zmpm_stats reports how many):
on those states the residual and product agree with the FP64 oracle to 1e-6
of their largest entry, at least ten times closer than the oracle's all-FP32
evaluation of the same state (measured 18x to 1900x).  StvkWithHenckyIsotropic
has no Hessian for an inverted element: its divided difference of logarithms
(MathTools.h:247-252) takes log1p of a value below -1 when two singular values
differ in sign, so the reference's product is NaN there, and so is the GPU's."""
import numpy as np
import pytest

from ziran2019_b200 import mpm
from tests.scenes import build_scene

pytestmark = pytest.mark.gpu

DX = 1.0 / 64
TOL = 2e-5  # MIXED: of the largest entry, as the benign-F hook tests

CASES = {
    "benign": (1.05, 0.97, 0.93),
    "inverted": (1.1, 0.9, -0.05),
    "near_singular": (1.0, 0.9, 1e-3),
    "stretched": (8.0, 1.0, 0.5),
    "repeated": (1.2, 1.2, 1.2),
    "two_equal": (1.3, 1.3, 0.9),
}
REEVALUATED = {"inverted", "near_singular", "stretched"}


def rotations(rng, n):
    q, r = np.linalg.qr(rng.standard_normal((n, 3, 3)))
    q = q * np.sign(np.diagonal(r, axis1=1, axis2=2))[:, None, :]
    q[np.linalg.det(q) < 0, :, 0] *= -1
    return q


def state(case, n, seed):
    rng = np.random.default_rng(seed)
    U, V = rotations(rng, n), rotations(rng, n)
    s = np.asarray(CASES[case])
    return np.einsum("nij,j,nkj->nik", U, s, V)


def build(lib, kind, precision, case, seed=7):
    s = mpm.MpmSimulation(DX, gravity=(0, -9.8, 0), precision=precision, lib=lib, **({} if lib else {"grid_log2": 8}))
    build_scene(s, kind=kind, n=4, dx=DX, seed=seed)
    s.setParticles(F=state(case, s.count, seed))
    return s


def by_coord(sim):
    m, v, c = sim.getGrid()
    key = (c[:, 0].astype(np.int64) << 40) | (c[:, 1].astype(np.int64) << 20) | c[:, 2].astype(np.int64)
    return np.argsort(key)


def objective(sim, dv_sorted, x_sorted):
    """Residual and Hessian product at dv, vectors in coordinate order."""
    N = sim.beginImplicit(1e-3)
    o = by_coord(sim)
    dv = np.empty_like(dv_sorted)
    dv[o] = dv_sorted
    r, _ = sim.residual(dv)
    x = np.empty_like(x_sorted)
    x[o] = x_sorted
    b = sim.multiply(x, fp32=sim.precision == "mixed")
    return N, r[o], b[o]


def rel_err(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("kind", ["hencky", "fcr"])
@pytest.mark.parametrize("case", list(CASES))
def test_degenerate_singular_values(cuda_lib, oracle, kind, case):
    rng = np.random.default_rng(3)
    ref = build(oracle, kind, "fp64", case)
    N = ref.beginImplicit(1e-3)
    dv = 0.01 * rng.standard_normal((N, 3))
    x = rng.standard_normal((N, 3))
    _, r64, b64 = objective(ref, dv, x)
    out = {}
    for name, lib, prec in (("gpu_fp64", None, "fp64"), ("gpu_mixed", None, "mixed"), ("oracle_fp32", oracle, "mixed")):
        s = build(lib, kind, prec, case)
        n, r, b = objective(s, dv, x)
        assert n == N
        out[name] = (rel_err(r, r64), rel_err(b, b64))
        if name == "gpu_mixed":
            # a substep of the same state reports the FP64 re-evaluations of its updates
            s.newton_max_iterations = 1
            s.advanceOneTimeStep(1e-6)
            reeval = s.last_stats["svd_fp64_reevaluations"]
    print(kind, case, out, "fp64 re-evaluations", reeval)
    if kind == "hencky" and case == "inverted":
        # no Hessian: NaN in the reference's restatement and on the GPU alike
        assert np.isnan(b64).all() and all(np.isnan(e[1]) for e in out.values()), out
        out = {k: (e[0],) for k, e in out.items()}
    assert max(out["gpu_fp64"]) < 1e-9, out
    assert max(out["gpu_mixed"]) < TOL, out
    if case in REEVALUATED:
        assert reeval > 0
        assert max(out["gpu_mixed"]) < 1e-6, out
        # the all-FP32 evaluation of the same state is at least ten times further off
        assert 10 * max(out["gpu_mixed"]) < max(out["oracle_fp32"]), out
    else:
        assert reeval == 0
