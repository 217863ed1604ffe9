// A C++ caller of the library through its C++ host wrapper (include/zmpm.hpp
// over include/zmpm.h), compiled with g++ against the headers alone and linked
// with the CUDA library.  It drives the implicit substep the way a
// reference-side adapter does (an MpmSimulationBase subclass that overrides
// advanceOneTimeStep and keeps one phase for itself): particlesToGrid,
// backwardEulerStep, gridToParticles without plasticity, then applyPlasticity
// as the subclass's own step.  The same scene advanced by whole substeps is
// the comparison.  Prints one line "max_rel_dx <value> substeps <n>" and
// exits 0, or prints the failing call and exits 1.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "zmpm.hpp"

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

// The adapter: a GpuMpmSimulation (include/zmpm.hpp) set up through the
// registration calls, and a substep either whole or in phases with
// plasticity applied as a separate step.
class PhaseAdapter {
public:
    PhaseAdapter(const Scene& sc, double dx, int precision, bool phases) : sim_(options(dx, precision)), phases_(phases)
    {
        sim_.addParticles(sc.x, sc.v, sc.m, sc.vol).addFBasedMpmForce(ZMPM_MODEL_STVK_HENCKY_ISOTROPIC, 1e4, 0.3).addVonMises(60.0, 0.0, 1e30);
        zmpm_collider floor{};
        floor.shape = ZMPM_HALF_SPACE;
        floor.type = ZMPM_STICKY;
        floor.a[1] = 0.38;
        floor.b[1] = 1.0;
        floor.rotation[0] = 1.0;
        floor.scale = 1.0;
        sim_.addCollisionObject(floor);
        sim_.solver().newton_tolerance = 1e-9;
        sim_.solver().newton_max_iterations = 8;
    }

    void advanceOneTimeStep(double dt)
    {
        if (!phases_) {
            sim_.advanceOneTimeStep(dt);
            return;
        }
        sim_.particlesToGrid(dt);
        sim_.backwardEulerStep();
        sim_.gridToParticles(false);
        sim_.applyPlasticity();
    }

    std::vector<double> positions()
    {
        std::vector<double> x;
        sim_.getParticles(&x);
        return x;
    }

private:
    static zmpm::GpuMpmSimulation::Options options(double dx, int precision)
    {
        zmpm::GpuMpmSimulation::Options o;
        o.dx = dx;
        o.precision = precision;
        o.grid_log2 = 7;
        return o;
    }
    zmpm::GpuMpmSimulation sim_;
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
    try {
        for (int n = 0; n < steps; ++n) {
            whole.advanceOneTimeStep(1e-3);
            split.advanceOneTimeStep(1e-3);
        }
    }
    catch (const std::exception& e) {
        std::printf("FAILED %s\n", e.what());
        return 1;
    }
    const std::vector<double> a = whole.positions(), b = split.positions();
    double err = 0;
    for (size_t i = 0; i < a.size(); ++i) err = std::fmax(err, std::fabs(a[i] - b[i]) / dx);
    std::printf("max_rel_dx %.3e substeps %d particles %zu\n", err, steps, a.size() / 3);
    return 0;
}
