"""Host-side mirror of the reference's MPM scene / plugin API over the C ABI.

Names follow the reference so that scene code reads the same:

* `MpmSimulation`      <- MpmSimulationBase<T,3> (Lib/MPM/MpmSimulationBase.h:133-229)
* `MpmParticleHandle`  <- MpmParticleHandleBase<T,3> (Lib/MPM/MpmParticleHandleBase.h:53-107)
* `NeoHookeanBorden`, `StvkWithHenckyIsotropic`, `FixedCorotated`
                        <- constitutive model plugins (Lib/Ziran/Physics/ConstitutiveModel)
* `VonMisesStvkHencky` <- plasticity plugin (Lib/Ziran/Physics/PlasticityApplier.h:187-281)
* `HalfSpace`, `Sphere`, `AxisAlignedAnalyticBox`, `AnalyticCollisionObject`
                        <- collision plugins (Lib/Ziran/Math/Geometry)

Every call goes through the CUDA library (`abi.product_lib()`); a missing
library raises instead of falling back to anything else.
"""
import warnings

import numpy as np

from . import abi
from .abi import ptr


# ------------------------------------------------------------------ models --
class _Model:
    kind = abi.MODEL_NONE

    def __init__(self, E=1.0, nu=0.3):
        self.E = float(E)
        self.nu = float(nu)
        self.lam = self.E * self.nu / ((1 + self.nu) * (1 - 2 * self.nu))
        self.mu = self.E / (2 * (1 + self.nu))


class NeoHookeanBorden(_Model):
    """NeoHookeanBorden(E, nu), NeoHookeanBorden.cpp:10-21."""
    kind = abi.MODEL_NEOHOOKEAN_BORDEN


class StvkWithHenckyIsotropic(_Model):
    """StvkWithHenckyIsotropic(E, nu), StvkWithHenckyIsotropic.h:60-70."""
    kind = abi.MODEL_STVK_HENCKY_ISOTROPIC


class StvkWithHencky(_Model):
    """StvkWithHencky(E, nu), StvkWithHencky.cpp:10-20: the model of the
    non-equilibrated (viscous) strain; same energy as StvkWithHenckyIsotropic."""
    kind = abi.MODEL_STVK_HENCKY_ISOTROPIC


class FixedCorotated(_Model):
    """Fixed corotated elasticity (Stomakhin et al. 2012); no reference counterpart."""
    kind = abi.MODEL_FIXED_COROTATED


class VonMisesStvkHencky:
    """VonMisesStvkHencky(yield_stress, fail_stress, xi), PlasticityApplier.cpp:443-450."""
    kind = abi.PLASTIC_VON_MISES

    def __init__(self, yield_stress, fail_stress=0.0, xi=0.0):
        self.yield_stress = float(yield_stress)
        self.fail_stress = float(fail_stress)
        self.xi = float(xi)


class DruckerPragerStvkHencky:
    """DruckerPragerStvkHencky(friction_angle, beta, cohesion, volume_correction),
    PlasticityApplier.cpp:247-261 (sand; StvkWithHenckyIsotropic particles)."""
    kind = abi.PLASTIC_DRUCKER_PRAGER

    def __init__(self, friction_angle=30.0, beta=1.0, cohesion=0.0, volume_correction=True):
        self.friction_angle = float(friction_angle)
        self.beta = float(beta)
        self.cohesion = float(cohesion)
        self.volume_correction = bool(volume_correction)


class NonAssociativeCamClay:
    """NonAssociativeCamClay(logJp, friction_angle, beta, xi, dim=3, hardeningOn),
    PlasticityApplier.cpp:10-20 (snow / clay; NeoHookeanBorden particles)."""
    kind = abi.PLASTIC_CAM_CLAY

    def __init__(self, logJp=0.0, friction_angle=0.0, beta=0.0, xi=0.0, hardeningOn=True):
        self.logJp = float(logJp)
        self.friction_angle = float(friction_angle)
        self.beta = float(beta)
        self.xi = float(xi)
        self.hardeningOn = bool(hardeningOn)


# -------------------------------------------------------------- colliders --
class HalfSpace:
    """HalfSpace(origin, outward_normal), AnalyticLevelSet.cpp:259-304."""

    def __init__(self, origin, normal):
        self.shape = abi.HALF_SPACE
        self.a = tuple(float(v) for v in origin)
        self.b = tuple(float(v) for v in normal)
        self.radius = 0.0


class Sphere:
    """Sphere(center, radius), AnalyticLevelSet.cpp:388-451."""

    def __init__(self, center, radius):
        self.shape = abi.SPHERE
        self.a = tuple(float(v) for v in center)
        self.b = (0.0, 0.0, 0.0)
        self.radius = float(radius)


class AxisAlignedAnalyticBox:
    """AxisAlignedAnalyticBox(min_corner, max_corner), AnalyticLevelSet.cpp:353-386."""

    def __init__(self, min_corner, max_corner):
        self.shape = abi.BOX
        self.a = tuple(float(v) for v in min_corner)
        self.b = tuple(float(v) for v in max_corner)
        self.radius = 0.0


class AnalyticCollisionObject:
    """AnalyticCollisionObject(level_set, type) with the rigid motion x = R s X + t.

    The reference's `updateState(time, object)` callback is expressed as a
    linear-in-time translation and scale (CollisionObject.h:63-71,146-170).
    """
    STICKY, SLIP, SEPARATE, GHOST = abi.STICKY, abi.SLIP, abi.SEPARATE, abi.GHOST

    def __init__(self, level_set, type_, friction=0.0):
        self.ls = level_set
        self.type = int(type_)
        self.friction = float(friction)
        self.rotation = (1.0, 0.0, 0.0, 0.0)
        self.angular_velocity = (0.0, 0.0, 0.0)
        self.translation = (0.0, 0.0, 0.0)
        self.translation_velocity = (0.0, 0.0, 0.0)
        self.scale = 1.0
        self.scale_velocity = 0.0

    def setFriction(self, f):
        self.friction = float(f)

    def setTranslation(self, b, dbdt=(0.0, 0.0, 0.0)):
        self.translation = tuple(float(v) for v in b)
        self.translation_velocity = tuple(float(v) for v in dbdt)

    def setRotation(self, q):
        self.rotation = tuple(float(v) for v in q)

    def setAngularVelocity(self, w):
        self.angular_velocity = tuple(float(v) for v in w)

    def setScaling(self, s, dsdt=0.0):
        self.scale = float(s)
        self.scale_velocity = float(dsdt)

    def to_struct(self):
        c = abi.Collider()
        c.shape = self.ls.shape
        c.type = self.type
        c.friction = self.friction
        c.a[:] = self.ls.a
        c.b[:] = self.ls.b
        c.radius = self.ls.radius
        c.rotation[:] = self.rotation
        c.angular_velocity[:] = self.angular_velocity
        c.translation[:] = self.translation
        c.translation_velocity[:] = self.translation_velocity
        c.scale = self.scale
        c.scale_velocity = self.scale_velocity
        return c


def add_all_walls_in_domain(sim, max_domain_boundary, offset, type_):
    """MpmInitializationHelper::addAllWallsInDomain (MpmInitializationHelper.h:614-629)."""
    ids = []
    for d in range(3):
        for s in (-1, 1):
            o = [0.0, 0.0, 0.0]
            n = [0.0, 0.0, 0.0]
            o[d] = offset if s == 1 else max_domain_boundary - offset
            n[d] = float(s)
            ids.append(sim.addCollisionObject(AnalyticCollisionObject(HalfSpace(o, n), type_)))
    return ids


# --------------------------------------------------------------- handles --
class MpmParticleHandle:
    """Particle range [lower, upper) of one MpmSimulation (MpmParticleHandleBase)."""

    def __init__(self, sim, lower, upper):
        self.sim = sim
        self.lower = lower
        self.upper = upper

    def addFBasedMpmForce(self, model):
        self.sim._call("add_fbased_force", self.lower, self.upper, model.kind, model.E, model.nu)

    def setLame(self, mu, lam):
        mu = np.ascontiguousarray(mu, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        self.sim._call("set_lame", self.lower, self.upper, ptr(mu), ptr(lam))

    def addRankineDamage(self, sigma_f, residual_phase=0.001, reference_order=False):
        """Phase field + Rankine damage (addFBasedMpmForceWithPhaseField with
        FractureSimulation::useNaiveDamage and sigmaF); needs NeoHookeanBorden.
        reference_order: sigma_max is the first eigenvalue of Eigen's general
        eigensolver, as FractureSimulation.h:539-543 takes it, instead of the
        largest eigenvalue."""
        kind = abi.DAMAGE_RANKINE_REFERENCE if reference_order else abi.DAMAGE_RANKINE
        self.sim._call("add_damage", self.lower, self.upper, kind, float(sigma_f), float(residual_phase))

    def addFBasedMpmForceWithPhaseField(self, percentage, l0, model=None, allow_damage=True, residual_phase=0.001):
        """CD-MPM phase field (MpmParticleHandleBase::addFBasedMpmForceWithPhaseField,
        MpmParticleHandleBase.cpp:92-118) on particles that already carry a
        NeoHookeanBorden model (pass `model` to add it here); the simulation
        then solves the phase-field system after P2G every substep."""
        if model is not None:
            self.addFBasedMpmForce(model)
        self.sim._call("add_phase_field", self.lower, self.upper, float(percentage), float(l0), 1 if allow_damage else 0,
                       float(residual_phase))

    def addFElasticNonequilibratedBasedMpmForce(self, model, viscosity_d, viscosity_v):
        """MpmParticleHandleBase::addFElasticNonequilibratedBasedMpmForce
        (MpmParticleHandleBase.cpp:468-478): Fe starts at I, relaxes by the
        viscous return map; the particles must already use StvkWithHenckyIsotropic."""
        self.sim._call("add_viscoelastic", self.lower, self.upper, model.E, model.nu, float(viscosity_d), float(viscosity_v))

    def addPlasticity(self, model, plasticity):
        del model  # the model is the one attached with addFBasedMpmForce
        if plasticity.kind == abi.PLASTIC_DRUCKER_PRAGER:
            self.sim._call("add_drucker_prager", self.lower, self.upper, plasticity.friction_angle, plasticity.beta,
                           plasticity.cohesion, 1 if plasticity.volume_correction else 0)
        elif plasticity.kind == abi.PLASTIC_CAM_CLAY:
            self.sim._call("add_cam_clay", self.lower, self.upper, plasticity.logJp, plasticity.friction_angle, plasticity.beta,
                           plasticity.xi, 1 if plasticity.hardeningOn else 0)
        else:
            self.sim._call("add_plasticity", self.lower, self.upper, plasticity.kind,
                           plasticity.yield_stress, plasticity.xi, plasticity.fail_stress)


# ----------------------------------------------------------- time stepping --
class TimeStepping:
    """TimeStepping (Lib/Ziran/Sim/TimeStepping.h:8-91): substep sizes that hit
    the frame times exactly.  Set `max_dt` after construction, as the
    reference's scenes do; `nextDt` clamps it to the frame length."""
    FRAME, SUBSTEP = 0, 1

    def __init__(self, frame_dt=1.0 / 24, min_dt=1e-6):
        self.time = 0.0
        self.time_since_last_frame = 0.0
        self.frame_dt = float(frame_dt)
        self.min_dt = float(min_dt)
        self.max_dt = self.frame_dt
        self.max_dt_original = self.frame_dt

    def nextDt(self, dt):
        if not dt > 0:
            raise ValueError("dt must be positive")
        self.max_dt = min(self.max_dt, self.max_dt_original)
        dt = self.min_dt if dt < self.min_dt else (self.max_dt if dt > self.max_dt else dt)
        if self.time_since_last_frame + dt >= self.frame_dt:
            dt = self.frame_dt - self.time_since_last_frame  # final substep of the frame
        elif self.time_since_last_frame + 2 * dt > self.frame_dt:
            dt = (self.frame_dt - self.time_since_last_frame) / 2  # no tiny last substep
        return dt

    def advance(self, dt):
        self.time += dt
        self.time_since_last_frame += dt
        if self.time_since_last_frame >= self.frame_dt:
            self.time_since_last_frame = 0.0
            return self.FRAME
        return self.SUBSTEP

    def reset(self, frame):
        self.time = frame * self.frame_dt
        self.time_since_last_frame = 0.0


class RestartRequired(RuntimeError):
    """A substep moved a particle more than one cell: the reference throws
    RestartException and restarts the frame with half the max dt
    (MpmSimulationBase.cpp:983-1002).  `max_dt` is the suggested new value."""

    def __init__(self, frame, max_dt):
        super().__init__(f"CFL violation in frame {frame}; restart it with max_dt = {max_dt}")
        self.frame = frame
        self.max_dt = max_dt


# ------------------------------------------------------------ simulation --
class MpmSimulation:
    """Implicit APIC MPM on one GPU (MpmSimulationBase<T,3>, symplectic = false).

    precision: "fp64" or "mixed".  `newton_tolerance`, `newton_max_iterations`
    and the Krylov settings mirror `sim.newton` and `sim.objective` of the
    reference (MpmSimulationBase.cpp:51, BackwardEuler.h:51-98).
    """

    def __init__(self, dx, gravity=(0.0, 0.0, 0.0), precision="fp64", layout="auto",
                 grid_log2=10, apic_rpic_ratio=1.0, cfl=0.6, device=0, lib=None):
        self.lib = lib if lib is not None else abi.product_lib()
        cfg = abi.Config()
        cfg.precision = {"fp64": abi.FP64, "mixed": abi.MIXED}[precision]
        cfg.layout = {"auto": abi.LAYOUT_AUTO, "244": abi.LAYOUT_244, "444": abi.LAYOUT_444}[layout]
        cfg.grid_log2 = int(grid_log2)
        cfg.device = int(device)
        cfg.dx = float(dx)
        cfg.gravity[:] = [float(g) for g in gravity]
        cfg.apic_rpic_ratio = float(apic_rpic_ratio)
        cfg.cfl = float(cfl)
        self.cfg = cfg
        self.precision = precision
        h = abi.C.c_void_p()
        self.lib.check(self.lib.create(abi.C.byref(cfg), abi.C.byref(h)), "create")
        self.ctx = h
        self.linear_solver = abi.MINRES
        self.newton_tolerance = 1e-5
        self.newton_max_iterations = 3
        self.krylov_max_iterations = 20
        self.krylov_tolerance = 1.0
        self.linear_solve_tolerance_scale = 1.0
        # ADMM integrator (AdmmSimulation members, AdmmSimulationFoam.h:47-70)
        self.integrator = abi.NEWTON
        self.admm_max_iterations = 100
        self.rho_scale = 0.5
        self.local_tolerance = 1e-8
        self.global_tolerance = 1e-6
        self.global_max_iteration = 10000
        # explicit integrator (MpmSimulationBase::symplectic, useTrialCollision, mls_mpm)
        self.useTrialCollision = True
        self.mls_mpm = False
        self.last_stats = None

    # lifecycle
    def close(self):
        if self.ctx:
            self.lib.destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def _call(self, name, *args):
        return self.lib.check(getattr(self.lib, name)(self.ctx, *args), name, self.ctx)

    # scene
    def addParticles(self, x, v=None, mass=None, volume=None):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        n = x.shape[0]
        v = np.zeros_like(x) if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        mass = np.ascontiguousarray(np.broadcast_to(mass, (n,)), dtype=np.float64)
        volume = np.ascontiguousarray(np.broadcast_to(volume, (n,)), dtype=np.float64)
        lower = abi.C.c_int64()
        self._call("add_particles", n, ptr(x), ptr(v), ptr(mass), ptr(volume), abi.C.byref(lower))
        return MpmParticleHandle(self, lower.value, lower.value + n)

    def addCollisionObject(self, obj):
        cid = abi.C.c_int32()
        s = obj.to_struct()
        self._call("add_collision_object", abi.C.byref(s), abi.C.byref(cid))
        return cid.value

    def setCollisionObject(self, cid, obj):
        s = obj.to_struct()
        self._call("set_collision_object", int(cid), abi.C.byref(s))

    def switchLinearSolver(self, kind):
        """BackwardEulerLagrangianForceObjective::switchLinearSolver (BackwardEuler.h:82-98):
        a fresh solver keeps max 20 iterations and the LinearSolver default
        tolerance 16 eps(T) (LinearSolver.h:24)."""
        self.linear_solver = kind
        self.krylov_max_iterations = 20
        eps = np.finfo(np.float64 if self.precision == "fp64" else np.float32).eps
        self.krylov_tolerance = 16 * float(eps)

    def solver(self):
        s = abi.Solver()
        s.linear_solver = self.linear_solver
        s.newton_max_iterations = self.newton_max_iterations
        s.newton_tolerance = self.newton_tolerance
        s.krylov_max_iterations = self.krylov_max_iterations
        s.krylov_tolerance = self.krylov_tolerance
        s.linear_solve_tolerance_scale = self.linear_solve_tolerance_scale
        s.integrator = self.integrator
        s.admm_iterations = self.admm_max_iterations
        s.admm_rho_scale = self.rho_scale
        s.admm_local_tolerance = self.local_tolerance
        s.admm_global_tolerance = self.global_tolerance
        s.admm_global_max_iterations = self.global_max_iteration
        s.trial_collision = 1 if self.useTrialCollision else 0
        s.mls_mpm = 1 if self.mls_mpm else 0
        return s

    def useExplicit(self, trial_collision=True, mls_mpm=False):
        """Symplectic substeps (MpmSimulationBase::symplectic = true): explicit
        grid update instead of the implicit solve; mls_mpm selects the MLS-MPM
        force and velocity gradient (explicit only, as in the reference)."""
        self.integrator = abi.EXPLICIT
        self.useTrialCollision = bool(trial_collision)
        self.mls_mpm = bool(mls_mpm)

    def useAdmm(self, admm_max_iterations=None, rho_scale=None, local_tolerance=None, global_tolerance=None,
                global_max_iteration=None):
        """Substep with AdmmSimulation::admmStep instead of Newton."""
        self.integrator = abi.ADMM
        for k, v in (("admm_max_iterations", admm_max_iterations), ("rho_scale", rho_scale),
                     ("local_tolerance", local_tolerance), ("global_tolerance", global_tolerance),
                     ("global_max_iteration", global_max_iteration)):
            if v is not None:
                setattr(self, k, v)

    # stepping
    def advanceOneTimeStep(self, dt):
        st = abi.Stats()
        s = self.solver()
        rc = self._call("substep", float(dt), abi.C.byref(s), abi.C.byref(st))
        self.last_stats = st.as_dict()
        self.last_status = rc
        return rc

    # the implicit substep in the phases of MpmSimulationBase's virtuals
    # (MpmSimulationBase.h:133-229), for callers that run their own work between them
    def particlesToGrid(self, dt):
        """reinitialize + particlesToGrid (+ the damage hook and the Newton start)."""
        s = self.solver()
        return self._call("particles_to_grid", float(dt), abi.C.byref(s))

    def backwardEulerStep(self):
        st = abi.Stats()
        rc = self._call("backward_euler_step", abi.C.byref(st))
        self.last_stats = st.as_dict()
        return rc

    def gridToParticles(self, apply_plasticity=True):
        """gridToParticles(dt): G2P, evolveStrain and (by default) applyPlasticity; ends the substep."""
        st = abi.Stats()
        rc = self._call("grid_to_particles", 1 if apply_plasticity else 0, abi.C.byref(st))
        self.last_status = rc
        return rc

    def applyPlasticity(self):
        return self._call("apply_plasticity")

    def calculateDt(self, max_dt):
        """MpmSimulationBase::calculateDt: cfl dx / max(particle, collider speed)."""
        dt = abi.C.c_double()
        self._call("calculate_dt", float(max_dt), abi.C.byref(dt))
        return dt.value

    def maxParticleSpeed(self):
        """evalMaxParticleSpeed: (max |v|, min corner, max corner)."""
        v = abi.C.c_double()
        lo, hi = np.zeros(3), np.zeros(3)
        self._call("max_particle_speed", abi.C.byref(v), ptr(lo), ptr(hi))
        return v.value, lo, hi

    def advanceOneFrame(self, step, frame=0, autorestart=True):
        """SimulationBase::advanceOneFrame (SimulationBase.h:288-321): substeps of
        step.nextDt(calculateDt()) until the frame ends; returns the substep
        count.  A CFL violation raises RestartRequired (autorestart) with half
        the max dt, as the reference's restart does."""
        n = 0
        while True:
            dt = step.nextDt(self.calculateDt(step.max_dt))
            rc = self.advanceOneTimeStep(dt)
            n += 1
            if rc == abi.CFL_VIOLATION and autorestart:
                raise RestartRequired(frame, max(step.max_dt / 2, step.min_dt))
            if rc not in (abi.OK, abi.CFL_VIOLATION):
                raise abi.ZmpmError(rc, "substep")
            if step.advance(dt) == TimeStepping.FRAME:
                return n

    # state
    @property
    def count(self):
        return int(self.lib.num_particles(self.ctx))

    @property
    def time(self):
        return float(self.lib.time(self.ctx))

    def getParticles(self):
        n = self.count
        x = np.empty((n, 3))
        v = np.empty((n, 3))
        Cm = np.empty((n, 3, 3))
        F = np.empty((n, 3, 3))
        self._call("get_particles", ptr(x), ptr(v), ptr(Cm), ptr(F))
        return {"X": x, "V": v, "C": Cm, "F": F}

    def setParticles(self, X=None, V=None, C=None, F=None):
        def p(a, shape):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(shape)
            return a, ptr(a)
        n = self.count
        keep = [p(X, (n, 3)), p(V, (n, 3)), p(C, (n, 3, 3)), p(F, (n, 3, 3))]
        self._call("set_particles", *[k[1] for k in keep])

    def getDamage(self):
        c = np.empty(self.count)
        self._call("get_damage", ptr(c))
        return c

    def setPhaseFieldSolver(self, parabolic_M=0.0, lumping=True, delete_particle_threshold=0.0, cg_max_iterations=100,
                            cg_tolerance=1e-6):
        """FractureSimulation::parabolic_M, lumping, delete_particle_threshold and
        its CG's max iterations and tolerance (FractureSimulation.h:48-63, 444-446)."""
        self._call("set_phase_field_solver", float(parabolic_M), 1 if lumping else 0, float(delete_particle_threshold),
                   int(cg_max_iterations), float(cg_tolerance))

    def getPhaseField(self):
        """Per-particle phase-field state: c, H, pf_Fp and the current volume."""
        out = {k: np.empty(self.count) for k in ("c", "H", "pf_Fp", "vol")}
        self._call("get_phase_field", ptr(out["c"]), ptr(out["H"]), ptr(out["pf_Fp"]), ptr(out["vol"]))
        return out

    def setPhaseFieldSigmaC(self, one_over_sigma_c):
        a = np.ascontiguousarray(one_over_sigma_c, dtype=np.float64)
        self._call("set_phase_field_sigma_c", ptr(a))

    # reverse mode and checkpoints
    def adjointSubstep(self, dt, gx=None, gv=None, gC=None, gF=None, gE=None, tolerance=1e-12):
        """Runs one substep forward from the current state and maps the loss
        gradients with respect to the new state (gx, gv: [P,3]; gC, gF: [P,3,3])
        to gradients with respect to the previous state, in place; gE [P]
        accumulates dL/dE.  Returns the status."""
        n = self.count

        def arr(a, shape):
            if a is None:
                return None
            assert a.dtype == np.float64 and a.flags.c_contiguous and a.shape == shape
            return a
        st = abi.Stats()
        s = self.solver()
        args = [arr(gx, (n, 3)), arr(gv, (n, 3)), arr(gC, (n, 3, 3)), arr(gF, (n, 3, 3)), arr(gE, (n,))]
        rc = self.lib.adjoint_substep(self.ctx, float(dt), abi.C.byref(s), float(tolerance),
                                      *[ptr(a) if a is not None else None for a in args], abi.C.byref(st))
        self.last_stats = st.as_dict()
        return rc

    def checkpointSave(self, slot):
        self._call("checkpoint_save", int(slot))

    def checkpointLoad(self, slot):
        self._call("checkpoint_load", int(slot))

    def setYoungsModulus(self, E, nu, lower=0, upper=None):
        """Per-particle E at Poisson ratio nu (mu and lambda of each particle)."""
        upper = self.count if upper is None else upper
        E = np.ascontiguousarray(np.broadcast_to(E, (upper - lower,)), dtype=np.float64)
        mu = E / (2 * (1 + nu))
        lam = E * nu / ((1 + nu) * (1 - 2 * nu))
        self._call("set_lame", int(lower), int(upper), ptr(np.ascontiguousarray(mu)), ptr(np.ascontiguousarray(lam)))

    def getViscoelasticStrain(self):
        Fe = np.empty((self.count, 3, 3))
        self._call("get_viscoelastic_strain", ptr(Fe))
        return Fe

    def setViscoelasticStrain(self, Fe):
        Fe = np.ascontiguousarray(Fe, dtype=np.float64).reshape(self.count, 3, 3)
        self._call("set_viscoelastic_strain", ptr(Fe))

    # files (SimulationBase::write / read, writePartio)
    def write(self, path):
        """Restart file of the whole scene state (library format)."""
        self._call("write_state", str(path).encode())

    def read(self, path):
        """Replaces the scene with a restart file written by `write`."""
        self._call("read_state", str(path).encode())

    @staticmethod
    def outputFileName(frame, substep=0, name="restart", suffix=".dat"):
        """SimulationBase::outputFileName (SimulationBase.h:192-199)."""
        return f"{name}_{frame}" + (f"_{substep}" if substep > 0 else "") + suffix

    def writeRestart(self, output_dir, frame, substep=0):
        """SimulationBase::write in the reference's restart layout:
        output_dir/restart_<frame>[_<substep>].dat, last_written.txt (the frame)
        and binary_ver.txt (BINARY_VER)."""
        self._call("write_restart", str(output_dir).encode(), int(frame), int(substep))

    def readRestart(self, output_dir, frame, substep=0):
        """SimulationBase::read: fails on restart data of a newer binary version;
        warns, as the reference does, when last_written.txt holds a frame before
        `frame` (stale data).  Returns that last written frame (-1 if missing)."""
        last = abi.C.c_int32(-1)
        self._call("read_restart", str(output_dir).encode(), int(frame), int(substep), abi.C.byref(last))
        if last.value < frame:
            warnings.warn(f"Frame {frame} is after the last written frame {last.value}. Could be reading stale data")
        return last.value

    def writePartio(self, path, velocity=False, phase_field=False):
        """BGEO point file with "position" (+ "v", + "pf" / "sigmaC")."""
        fields = (abi.BGEO_VELOCITY if velocity else 0) | (abi.BGEO_PHASE_FIELD if phase_field else 0)
        self._call("write_bgeo", str(path).encode(), fields)

    def getLogJp(self):
        """log Jp of Drucker-Prager and Cam-Clay particles."""
        out = np.empty(self.count)
        self._call("get_log_jp", ptr(out))
        return out

    def getPlasticState(self):
        n = self.count
        ys = np.empty(n)
        broken = np.empty(n, dtype=np.int32)
        self._call("get_plastic_state", ptr(ys), ptr(broken, abi.C.c_int32))
        return ys, broken

    # hooks on the implicit objective (tests / adjoints)
    def binParticles(self):
        counts = np.zeros(3, dtype=np.int64)
        self._call("bin", ptr(counts, abi.C.c_int64))
        P, G, B = (int(c) for c in counts)
        out = {
            "particle_sorter": np.empty(P, dtype=np.uint64),
            "particle_order": np.empty(P, dtype=np.int32),
            "particle_base_offset": np.empty(P, dtype=np.uint64),
            "particle_group": np.empty((G, 2), dtype=np.int32),
            "block_offset": np.empty(G, dtype=np.uint64),
            "page_offsets": np.empty(B, dtype=np.uint64),
        }
        r = abi.BinResult()
        r.particle_sorter = ptr(out["particle_sorter"], abi.C.c_uint64)
        r.particle_order = ptr(out["particle_order"], abi.C.c_int32)
        r.particle_base_offset = ptr(out["particle_base_offset"], abi.C.c_uint64)
        r.particle_group = ptr(out["particle_group"], abi.C.c_int32)
        r.block_offset = ptr(out["block_offset"], abi.C.c_uint64)
        r.page_offsets = ptr(out["page_offsets"], abi.C.c_uint64)
        self._call("bin_fetch", abi.C.byref(r))
        return out

    def beginImplicit(self, dt):
        n = abi.C.c_int64()
        self._call("begin_implicit", float(dt), abi.C.byref(n))
        self.num_nodes = int(n.value)
        return self.num_nodes

    def getGrid(self):
        n = self.num_nodes
        m = np.empty(n)
        v = np.empty((n, 3))
        coord = np.empty((n, 3), dtype=np.int32)
        self._call("get_grid", ptr(m), ptr(v), ptr(coord, abi.C.c_int32))
        return m, v, coord

    def getInitialDv(self):
        n = self.num_nodes
        dv = np.empty((n, 3))
        col = np.empty(n, dtype=np.int32)
        self._call("get_initial_dv", ptr(dv), ptr(col, abi.C.c_int32))
        return dv, col

    def residual(self, dv):
        dv = np.ascontiguousarray(dv, dtype=np.float64).reshape(-1, 3)
        r = np.empty_like(dv)
        norm = abi.C.c_double()
        self._call("residual", ptr(dv), ptr(r), abi.C.byref(norm))
        return r, norm.value

    def multiply(self, x, fp32=False):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        b = np.empty_like(x)
        self._call("multiply", ptr(x), ptr(b), 1 if fp32 else 0)
        return b
