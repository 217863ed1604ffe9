"""The grid-wide barrier of the persistent Krylov kernel is a bounded wait
(CG runs its whole linear solve in one cooperative launch).  With a limit of
one poll the CTAs that reach a barrier first give up: every CTA returns, the
substep reports ZMPM_TIMEOUT, nothing faults, and with the default limit the
same context steps on normally."""
import pytest

from ziran2019_b200 import abi, mpm
from tests.scenes import build_scene

pytestmark = pytest.mark.gpu


def test_grid_barrier_gives_up_and_reports_timeout(cuda_lib):
    dx = 1.0 / 64
    sim = mpm.MpmSimulation(dx, gravity=(0, -9.8, 0), precision="fp64", grid_log2=8)
    build_scene(sim, kind="fcr", n=6, dx=dx, seed=4)
    sim.switchLinearSolver(abi.CG)
    sim.newton_tolerance = 1e-9
    sim.newton_max_iterations = 4
    assert sim.advanceOneTimeStep(1e-3) == abi.OK
    assert sim.last_stats["krylov_iterations"] > 0
    assert sim.lib.set_spin_limit(sim.ctx, 1) == abi.OK
    assert sim.advanceOneTimeStep(1e-3) == abi.TIMEOUT
    assert sim.last_stats["status_flags"] & 2
    assert sim.lib.set_spin_limit(sim.ctx, 0) == abi.OK
    assert sim.advanceOneTimeStep(1e-3) == abi.OK
    assert sim.last_stats["krylov_iterations"] > 0
