/* C++ host wrapper over the C ABI of zmpm.h (header only, C++17).
 *
 * GpuMpmSimulation mirrors the entry points of the reference's
 * MpmSimulationBase<T,3> (Lib/MPM/MpmSimulationBase.h:133-229:
 * advanceOneTimeStep, particlesToGrid, backwardEulerStep, gridToParticles,
 * applyPlasticity, calculateDt, addCollisionObject, write / read) and
 * ParticleHandle the registration API of MpmParticleHandleBase
 * (MpmParticleHandleBase.h:53-107: addFBasedMpmForce, addPlasticity,
 * addFElasticNonequilibratedBasedMpmForce, addFBasedMpmForceWithPhaseField).
 * Status codes become exceptions as in the reference: a CFL violation throws
 * CflViolation (the role of RestartException, MpmSimulationBase.cpp:983-1002),
 * any other failing call throws Error (the role of ZIRAN_ASSERT's
 * std::runtime_error, Debug.h:19-38).  A Newton solve that does not converge
 * is reported in lastStats(), as NewtonsMethod::solve only returns false
 * (NewtonsMethod.h:65).  One object owns one context; it is not thread-safe,
 * like the reference simulation. */
#ifndef ZMPM_HPP
#define ZMPM_HPP

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "zmpm.h"

namespace zmpm {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

// A particle moved more than one cell in a substep; the caller restarts the
// frame with a smaller time step.
class CflViolation : public std::runtime_error {
public:
    explicit CflViolation(double time) : std::runtime_error("CFL violation"), time_(time) {}
    double time() const { return time_; }

private:
    double time_;
};

class GpuMpmSimulation;

// The particles [lower, upper) of one addParticles call.
class ParticleHandle {
public:
    int64_t lower() const { return lower_; }
    int64_t upper() const { return upper_; }
    int64_t count() const { return upper_ - lower_; }

    // addFBasedMpmForce(model) with the model's (E, nu)
    ParticleHandle& addFBasedMpmForce(int32_t model, double youngs_modulus, double poisson_ratio);
    // addPlasticity(model, VonMisesStvkHencky(yield_stress, fail_stress, xi))
    ParticleHandle& addVonMises(double yield_stress, double xi = 0.0, double fail_stress = 1e30);
    // addPlasticity(model, DruckerPragerStvkHencky(friction_angle, beta, cohesion, volume_correction))
    ParticleHandle& addDruckerPrager(double friction_angle = 30.0, double beta = 1.0, double cohesion = 0.0, bool volume_correction = true);
    // addPlasticity(model, NonAssociativeCamClay(logJp, friction_angle, beta, xi, 3, hardeningOn))
    ParticleHandle& addCamClay(double log_jp, double friction_angle, double beta, double xi, bool hardening = true);
    // addFElasticNonequilibratedBasedMpmForce(StvkWithHencky(E, nu), nu_d, nu_v)
    ParticleHandle& addFElasticNonequilibratedBasedMpmForce(double youngs_modulus, double poisson_ratio, double viscosity_d, double viscosity_v);
    // addFBasedMpmForceWithPhaseField(percentage, l0, NeoHookeanBorden(E, nu), allow_damage)
    ParticleHandle& addFBasedMpmForceWithPhaseField(double percentage, double l0, double youngs_modulus, double poisson_ratio,
        bool allow_damage = true, double residual_phase = 0.001);
    // FractureSimulation's naive Rankine damage (sigmaF), in the reference's
    // eigenvalue order or with the largest eigenvalue
    ParticleHandle& addRankineDamage(double sigma_f, double residual_phase = 0.001, bool reference_order = true);

private:
    friend class GpuMpmSimulation;
    ParticleHandle(GpuMpmSimulation* sim, int64_t lower, int64_t upper) : sim_(sim), lower_(lower), upper_(upper) {}
    GpuMpmSimulation* sim_;
    int64_t lower_, upper_;
};

class GpuMpmSimulation {
public:
    struct Options {
        double dx = 1.0 / 64;
        std::array<double, 3> gravity{ { 0.0, -9.8, 0.0 } };
        int32_t precision = ZMPM_MIXED;
        int32_t layout = ZMPM_LAYOUT_AUTO;
        int32_t grid_log2 = 10;
        int32_t device = 0;
        double apic_rpic_ratio = 1.0;
        double cfl = 0.6;
    };

    explicit GpuMpmSimulation(const Options& o) : precision_(o.precision)
    {
        zmpm_config cfg{};
        cfg.precision = o.precision;
        cfg.layout = o.layout;
        cfg.grid_log2 = o.grid_log2;
        cfg.device = o.device;
        cfg.dx = o.dx;
        for (int d = 0; d < 3; ++d) cfg.gravity[d] = o.gravity[d];
        cfg.apic_rpic_ratio = o.apic_rpic_ratio;
        cfg.cfl = o.cfl;
        const int rc = zmpm_create(&cfg, &ctx_);
        if (rc < 0) throw Error(rc, std::string("zmpm_create: ") + zmpm_status_string(rc));
        zmpm_default_solver(&solver_, ZMPM_MINRES, o.precision);
    }
    ~GpuMpmSimulation()
    {
        if (ctx_) zmpm_destroy(ctx_);
    }
    GpuMpmSimulation(const GpuMpmSimulation&) = delete;
    GpuMpmSimulation& operator=(const GpuMpmSimulation&) = delete;
    GpuMpmSimulation(GpuMpmSimulation&& o) noexcept : ctx_(std::exchange(o.ctx_, nullptr)), solver_(o.solver_), stats_(o.stats_), precision_(o.precision_) {}

    // ---- solver settings (the reference's members) ----
    zmpm_solver& solver() { return solver_; }
    void switchLinearSolver(int32_t linear_solver)  // ZMPM_MINRES or ZMPM_CG
    {
        const zmpm_solver keep = solver_;
        zmpm_default_solver(&solver_, linear_solver, precision_);
        solver_.newton_tolerance = keep.newton_tolerance;
        solver_.newton_max_iterations = keep.newton_max_iterations;
        solver_.integrator = keep.integrator;
    }

    // ---- scene ----
    ParticleHandle addParticles(const std::vector<double>& x, const std::vector<double>& v, const std::vector<double>& mass,
        const std::vector<double>& volume)
    {
        const int64_t n = (int64_t)mass.size();
        if ((int64_t)x.size() != 3 * n || (int64_t)v.size() != 3 * n || (int64_t)volume.size() != n)
            throw Error(ZMPM_BAD_ARG, "addParticles: x and v need 3 values, mass and volume 1 value per particle");
        int64_t lower = 0;
        check(zmpm_add_particles(ctx_, n, x.data(), v.data(), mass.data(), volume.data(), &lower), "zmpm_add_particles");
        return ParticleHandle(this, lower, lower + n);
    }
    int32_t addCollisionObject(const zmpm_collider& c)
    {
        int32_t id = 0;
        check(zmpm_add_collision_object(ctx_, &c, &id), "zmpm_add_collision_object");
        return id;
    }
    void setCollisionObject(int32_t id, const zmpm_collider& c) { check(zmpm_set_collision_object(ctx_, id, &c), "zmpm_set_collision_object"); }

    // ---- the substep and its phases (MpmSimulationBase virtuals) ----
    void advanceOneTimeStep(double dt)
    {
        const int rc = zmpm_substep(ctx_, dt, &solver_, &stats_);
        if (rc == ZMPM_CFL_VIOLATION) throw CflViolation(zmpm_time(ctx_));
        check(rc, "zmpm_substep");
    }
    void particlesToGrid(double dt) { check(zmpm_particles_to_grid(ctx_, dt, &solver_), "zmpm_particles_to_grid"); }
    void backwardEulerStep() { check(zmpm_backward_euler_step(ctx_, &stats_), "zmpm_backward_euler_step"); }
    // G2P, advection, evolveStrain; the return maps too unless the caller runs
    // applyPlasticity itself
    void gridToParticles(bool with_plasticity = true)
    {
        const int rc = zmpm_grid_to_particles(ctx_, with_plasticity ? 1 : 0, &stats_);
        if (rc == ZMPM_CFL_VIOLATION) throw CflViolation(zmpm_time(ctx_));
        check(rc, "zmpm_grid_to_particles");
    }
    void applyPlasticity() { check(zmpm_apply_plasticity(ctx_), "zmpm_apply_plasticity"); }
    double calculateDt(double max_dt)
    {
        double dt = max_dt;
        check(zmpm_calculate_dt(ctx_, max_dt, &dt), "zmpm_calculate_dt");
        return dt;
    }
    const zmpm_stats& lastStats() const { return stats_; }

    // ---- state ----
    int64_t numParticles() const { return zmpm_num_particles(ctx_); }
    double time() const { return zmpm_time(ctx_); }
    // x, v: [P][3]; C, F: [P][3][3] in particle order; empty vectors are skipped
    void getParticles(std::vector<double>* x, std::vector<double>* v = nullptr, std::vector<double>* C = nullptr,
        std::vector<double>* F = nullptr)
    {
        const size_t n = (size_t)numParticles();
        if (x) x->resize(3 * n);
        if (v) v->resize(3 * n);
        if (C) C->resize(9 * n);
        if (F) F->resize(9 * n);
        check(zmpm_get_particles(ctx_, x ? x->data() : nullptr, v ? v->data() : nullptr, C ? C->data() : nullptr, F ? F->data() : nullptr),
            "zmpm_get_particles");
    }
    void setParticles(const std::vector<double>* x, const std::vector<double>* v = nullptr, const std::vector<double>* C = nullptr,
        const std::vector<double>* F = nullptr)
    {
        check(zmpm_set_particles(ctx_, x ? x->data() : nullptr, v ? v->data() : nullptr, C ? C->data() : nullptr, F ? F->data() : nullptr),
            "zmpm_set_particles");
    }

    // ---- files (SimulationBase::write / read / outputFileName) ----
    void write(const std::string& path) { check(zmpm_write_state(ctx_, path.c_str()), "zmpm_write_state"); }
    void read(const std::string& path) { check(zmpm_read_state(ctx_, path.c_str()), "zmpm_read_state"); }
    void writeRestart(const std::string& output_dir, int32_t frame, int32_t substep = 0)
    {
        check(zmpm_write_restart(ctx_, output_dir.c_str(), frame, substep), "zmpm_write_restart");
    }
    // returns the frame last_written.txt holds (-1 if missing); the reference
    // warns when it is before `frame`
    int32_t readRestart(const std::string& output_dir, int32_t frame, int32_t substep = 0)
    {
        int32_t last = -1;
        check(zmpm_read_restart(ctx_, output_dir.c_str(), frame, substep, &last), "zmpm_read_restart");
        return last;
    }
    void writePartio(const std::string& path, int32_t fields = 0) { check(zmpm_write_bgeo(ctx_, path.c_str(), fields), "zmpm_write_bgeo"); }

    zmpm_ctx* handle() { return ctx_; }
    void* stream()
    {
        void* s = nullptr;
        check(zmpm_get_stream(ctx_, &s), "zmpm_get_stream");
        return s;
    }

    void check(int rc, const char* where)
    {
        if (rc < 0) throw Error(rc, std::string(where) + ": " + zmpm_status_string(rc) + ": " + (ctx_ ? zmpm_last_error(ctx_) : ""));
    }

private:
    zmpm_ctx* ctx_ = nullptr;
    zmpm_solver solver_{};
    zmpm_stats stats_{};
    int32_t precision_;
};

inline ParticleHandle& ParticleHandle::addFBasedMpmForce(int32_t model, double youngs_modulus, double poisson_ratio)
{
    sim_->check(zmpm_add_fbased_force(sim_->handle(), lower_, upper_, model, youngs_modulus, poisson_ratio), "zmpm_add_fbased_force");
    return *this;
}
inline ParticleHandle& ParticleHandle::addVonMises(double yield_stress, double xi, double fail_stress)
{
    sim_->check(zmpm_add_plasticity(sim_->handle(), lower_, upper_, ZMPM_PLASTIC_VON_MISES, yield_stress, xi, fail_stress), "zmpm_add_plasticity");
    return *this;
}
inline ParticleHandle& ParticleHandle::addDruckerPrager(double friction_angle, double beta, double cohesion, bool volume_correction)
{
    sim_->check(zmpm_add_drucker_prager(sim_->handle(), lower_, upper_, friction_angle, beta, cohesion, volume_correction ? 1 : 0),
        "zmpm_add_drucker_prager");
    return *this;
}
inline ParticleHandle& ParticleHandle::addCamClay(double log_jp, double friction_angle, double beta, double xi, bool hardening)
{
    sim_->check(zmpm_add_cam_clay(sim_->handle(), lower_, upper_, log_jp, friction_angle, beta, xi, hardening ? 1 : 0), "zmpm_add_cam_clay");
    return *this;
}
inline ParticleHandle& ParticleHandle::addFElasticNonequilibratedBasedMpmForce(double youngs_modulus, double poisson_ratio, double viscosity_d,
    double viscosity_v)
{
    sim_->check(zmpm_add_viscoelastic(sim_->handle(), lower_, upper_, youngs_modulus, poisson_ratio, viscosity_d, viscosity_v),
        "zmpm_add_viscoelastic");
    return *this;
}
inline ParticleHandle& ParticleHandle::addFBasedMpmForceWithPhaseField(double percentage, double l0, double youngs_modulus,
    double poisson_ratio, bool allow_damage, double residual_phase)
{
    addFBasedMpmForce(ZMPM_MODEL_NEOHOOKEAN_BORDEN, youngs_modulus, poisson_ratio);
    sim_->check(zmpm_add_phase_field(sim_->handle(), lower_, upper_, percentage, l0, allow_damage ? 1 : 0, residual_phase),
        "zmpm_add_phase_field");
    return *this;
}
inline ParticleHandle& ParticleHandle::addRankineDamage(double sigma_f, double residual_phase, bool reference_order)
{
    sim_->check(zmpm_add_damage(sim_->handle(), lower_, upper_, reference_order ? ZMPM_DAMAGE_RANKINE_REFERENCE : ZMPM_DAMAGE_RANKINE,
                    sigma_f, residual_phase),
        "zmpm_add_damage");
    return *this;
}

} // namespace zmpm

#endif /* ZMPM_HPP */
