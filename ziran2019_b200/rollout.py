"""Differentiable rollouts of the implicit substep over the C ABI.

`Rollout` runs `steps` substeps from an initial state with per-particle Young's
modulus E and initial velocity v0, keeping a device checkpoint every
`checkpoint_every` substeps.  Its reverse sweep walks the segments backwards:
it reloads a segment's checkpoint, replays the segment forward to store every
substep's state in scratch slots, then applies `zmpm_adjoint_substep` (the
hand-written reverse mode of one substep) from the last substep to the first.
Memory is one checkpoint per segment plus one segment of states; work is two
forward sweeps plus one reverse sweep.

`DifferentiableRollout` wraps it as a `torch.autograd.Function` taking (E, v0)
and returning the final positions, so a loss written in torch (for example the
squared distance of the centre of mass to a target) backpropagates to E and v0.
"""
import numpy as np
import torch

from . import abi


class Rollout:
    def __init__(self, sim, nu, dt, steps, checkpoint_every=10, tolerance=1e-12):
        """sim: an MpmSimulation (CUDA library or oracle) with its particles,
        models and colliders added, in the state the rollout starts from
        (its velocities are replaced by v0)."""
        self.sim, self.nu, self.dt, self.steps = sim, float(nu), float(dt), int(steps)
        self.every = max(1, int(checkpoint_every))
        self.tol = float(tolerance)
        self.nseg = (self.steps + self.every - 1) // self.every
        sim.checkpointSave(self._base_slot())
        self.stats = []
        # forward calls so far: the checkpoints belong to the last one only
        self.generation = 0

    # slots: 0 .. nseg-1 segment checkpoints, nseg .. nseg+every-1 segment
    # states, the last one the untouched initial state
    def _base_slot(self):
        return self.nseg + self.every

    def run(self, E, v0):
        sim = self.sim
        self.generation += 1
        sim.checkpointLoad(self._base_slot())
        sim.setYoungsModulus(np.asarray(E, dtype=np.float64), self.nu)
        sim.setParticles(V=np.asarray(v0, dtype=np.float64).reshape(-1, 3))
        for n in range(self.steps):
            if n % self.every == 0:
                sim.checkpointSave(n // self.every)
            rc = sim.advanceOneTimeStep(self.dt)
            if rc not in (abi.OK, abi.CFL_VIOLATION):
                raise RuntimeError(f"substep {n}: status {rc}")
        return sim.getParticles()["X"]

    def backward(self, gX):
        """Gradients of a loss with dL/dX_final = gX: returns (dL/dE, dL/dv0)."""
        sim, P = self.sim, self.sim.count
        gx = np.ascontiguousarray(gX, dtype=np.float64).reshape(P, 3).copy()
        gv = np.zeros((P, 3))
        gC = np.zeros((P, 3, 3))
        gF = np.zeros((P, 3, 3))
        gE = np.zeros(P)
        self.stats = []
        for seg in reversed(range(self.nseg)):
            n0 = seg * self.every
            n1 = min(self.steps, n0 + self.every)
            sim.checkpointLoad(seg)
            for j in range(n1 - n0):
                sim.checkpointSave(self.nseg + j)
                if j < n1 - n0 - 1:
                    rc = sim.advanceOneTimeStep(self.dt)
                    if rc not in (abi.OK, abi.CFL_VIOLATION):
                        raise RuntimeError(f"replay of substep {n0 + j}: status {rc}")
            for j in reversed(range(n1 - n0)):
                sim.checkpointLoad(self.nseg + j)
                rc = sim.adjointSubstep(self.dt, gx, gv, gC, gF, gE, tolerance=self.tol)
                if rc not in (abi.OK, abi.CFL_VIOLATION):
                    raise RuntimeError(f"adjoint of substep {n0 + j}: status {rc}")
                self.stats.append(sim.last_stats)
        return gE, gv


class DifferentiableRollout(torch.autograd.Function):
    """X_final = rollout(E, v0) with the reverse sweep of `Rollout` as backward.

    The rollout's checkpoints hold the state of its latest forward call only, so
    the backward of an earlier forward call (a second forward ran in between)
    raises instead of returning the later call's gradients."""

    @staticmethod
    def forward(ctx, E, v0, rollout):
        X = rollout.run(E.detach().cpu().double().numpy(), v0.detach().cpu().double().numpy())
        ctx.rollout = rollout
        ctx.generation = rollout.generation
        ctx.dev = E.device
        ctx.shapes = (E.shape, v0.shape)
        return torch.from_numpy(np.ascontiguousarray(X)).to(device=E.device, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gX):
        if ctx.rollout.generation != ctx.generation:
            raise RuntimeError("DifferentiableRollout: the rollout ran forward again after this call; "
                               "its checkpoints no longer hold this call's states")
        gE, gv0 = ctx.rollout.backward(gX.detach().cpu().double().numpy())
        sE, sv = ctx.shapes
        return (torch.from_numpy(gE).reshape(sE).to(ctx.dev), torch.from_numpy(gv0).reshape(sv).to(ctx.dev), None)
