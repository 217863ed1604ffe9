// A C++ caller of include/zmpm.h, compiled with g++ against the header alone
// and linked with the CUDA library.  It drives the implicit substep the way a
// reference-side adapter does (an MpmSimulationBase subclass that overrides
// advanceOneTimeStep and keeps one phase for itself): particlesToGrid,
// backwardEulerStep, gridToParticles without plasticity, then applyPlasticity
// as the subclass's own step.  The same scene advanced by zmpm_substep is the
// comparison.  Prints one line "max_rel_dx <value> substeps <n>" and exits 0,
// or prints the failing call and exits 1.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "zmpm.h"

#define CHECK(call)                                                                                   \
    do {                                                                                              \
        int rc_ = (call);                                                                             \
        if (rc_ < 0) {                                                                                \
            std::printf("FAILED %s -> %d (%s)\n", #call, rc_, zmpm_status_string(rc_));               \
            std::exit(1);                                                                             \
        }                                                                                             \
    } while (0)

namespace {

struct Scene {
    std::vector<double> x, v, m, vol;
};

// 6 x 6 x 6 cells x 8 jittered particles per cell above a sticky floor.
Scene make_scene(double dx)
{
    Scene s;
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> u(0.0, 1.0), uv(-0.5, 0.5);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
            for (int k = 0; k < 6; ++k)
                for (int p = 0; p < 8; ++p) {
                    const int c[3] = { i, j, k };
                    for (int d = 0; d < 3; ++d) {
                        s.x.push_back(0.4 + (c[d] + u(rng)) * dx);
                        s.v.push_back(uv(rng));
                    }
                    s.vol.push_back(dx * dx * dx / 8);
                    s.m.push_back(1000.0 * dx * dx * dx / 8);
                }
    return s;
}

// The adapter: one context, the reference's registration calls, and a
// substep in phases with plasticity applied as a separate step.
class PhaseAdapter {
public:
    PhaseAdapter(const Scene& sc, double dx, int precision, bool phases) : phases_(phases)
    {
        zmpm_config cfg{};
        cfg.precision = precision;
        cfg.layout = ZMPM_LAYOUT_AUTO;
        cfg.grid_log2 = 7;
        cfg.dx = dx;
        cfg.gravity[1] = -9.8;
        cfg.apic_rpic_ratio = 1;
        cfg.cfl = 0.6;
        CHECK(zmpm_create(&cfg, &ctx_));
        const int64_t n = (int64_t)sc.m.size();
        int64_t lower = 0;
        CHECK(zmpm_add_particles(ctx_, n, sc.x.data(), sc.v.data(), sc.m.data(), sc.vol.data(), &lower));
        CHECK(zmpm_add_fbased_force(ctx_, lower, lower + n, ZMPM_MODEL_STVK_HENCKY_ISOTROPIC, 1e4, 0.3));
        CHECK(zmpm_add_plasticity(ctx_, lower, lower + n, ZMPM_PLASTIC_VON_MISES, 60.0, 0.0, 1e30));
        zmpm_collider floor{};
        floor.shape = ZMPM_HALF_SPACE;
        floor.type = ZMPM_STICKY;
        floor.a[1] = 0.38;
        floor.b[1] = 1.0;
        floor.rotation[0] = 1.0;
        floor.scale = 1.0;
        int32_t id = 0;
        CHECK(zmpm_add_collision_object(ctx_, &floor, &id));
        zmpm_default_solver(&solver_, ZMPM_MINRES, precision);
        solver_.newton_tolerance = 1e-9;
        solver_.newton_max_iterations = 8;
    }
    ~PhaseAdapter() { zmpm_destroy(ctx_); }

    int advanceOneTimeStep(double dt)
    {
        if (!phases_) return zmpm_substep(ctx_, dt, &solver_, nullptr);
        CHECK(zmpm_particles_to_grid(ctx_, dt, &solver_));
        zmpm_stats st;
        CHECK(zmpm_backward_euler_step(ctx_, &st));
        const int rc = zmpm_grid_to_particles(ctx_, 0, nullptr);
        CHECK(rc);
        CHECK(zmpm_apply_plasticity(ctx_));
        return rc;
    }

    std::vector<double> positions()
    {
        std::vector<double> x(3 * zmpm_num_particles(ctx_));
        CHECK(zmpm_get_particles(ctx_, x.data(), nullptr, nullptr, nullptr));
        return x;
    }

private:
    zmpm_ctx* ctx_ = nullptr;
    zmpm_solver solver_;
    bool phases_;
};

} // namespace

int main(int argc, char** argv)
{
    const int precision = (argc > 1 && argv[1][0] == 'm') ? ZMPM_MIXED : ZMPM_FP64;
    const double dx = 1.0 / 64;
    const Scene sc = make_scene(dx);
    PhaseAdapter whole(sc, dx, precision, false), split(sc, dx, precision, true);
    const int steps = 4;
    for (int n = 0; n < steps; ++n) {
        CHECK(whole.advanceOneTimeStep(1e-3));
        CHECK(split.advanceOneTimeStep(1e-3));
    }
    const std::vector<double> a = whole.positions(), b = split.positions();
    double err = 0;
    for (size_t i = 0; i < a.size(); ++i) err = std::fmax(err, std::fabs(a[i] - b[i]) / dx);
    std::printf("max_rel_dx %.3e substeps %d particles %zu\n", err, steps, a.size() / 3);
    return 0;
}
