// Per-particle stress through the CabanaPD API: particles built with
// EnergyStressOutput under the uniform stretch u = s0 x (the linear field of
// the reference's force unit test), the stress computed by Solver::init and
// at output steps. Built on the cabanapd_b200 front end.
// Usage: stress_cube <input.json> <pmb|lps>
//
// Writes stress_init.txt (after init) and stress_final.txt (after the run):
// one line per particle, x y z and the nine components
// xx xy xz yx yy yz zx zy zz.
#include <array>
#include <cstdio>
#include <iostream>
#include <string>

#include <CabanaPD.hpp>

using exec_space = Kokkos::DefaultExecutionSpace;
using memory_space = exec_space::memory_space;

template <class ParticleType>
static void write_stress(const std::string& path, const ParticleType& particles)
{
    auto x = particles.sliceReferencePosition();
    auto sigma = particles.sliceStress();
    FILE* out = std::fopen(path.c_str(), "w");
    for (std::size_t p = 0; p < particles.size(); p++) {
        std::fprintf(out, "%.17g %.17g %.17g", x(p, 0), x(p, 1), x(p, 2));
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) std::fprintf(out, " %.17g", sigma(p, a, b));
        std::fprintf(out, "\n");
    }
    std::fclose(out);
}

template <class Tag, class ModelType>
static void simulate(CabanaPD::Inputs& inputs, Tag tag, ModelType model)
{
    const double rho0 = inputs["density"];
    const double s0 = inputs["stretch"];
    const std::array<double, 3> lo = inputs["low_corner"];
    const std::array<double, 3> hi = inputs["high_corner"];
    const std::array<int, 3> cells = inputs["num_cells"];

    CabanaPD::Particles particles(memory_space{}, tag, CabanaPD::EnergyStressOutput{});
    particles.domain(lo, hi, cells, 0);
    particles.create(exec_space{});
    auto x = particles.sliceReferencePosition();
    auto u = particles.sliceDisplacement();
    auto v = particles.sliceVelocity();
    auto rho = particles.sliceDensity();
    particles.update(exec_space{}, KOKKOS_LAMBDA(const int p) {
        rho(p) = rho0;
        for (int d = 0; d < 3; d++) {
            u(p, d) = s0 * x(p, d);
            v(p, d) = 0.0;
        }
    });

    CabanaPD::Solver solver(inputs, particles, model);
    solver.init();
    write_stress("stress_init.txt", solver.particles);
    solver.run();
    write_stress("stress_final.txt", solver.particles);
}

int main(int argc, char* argv[])
{
    if (argc < 3) {
        std::cerr << "usage: stress_cube <input.json> <pmb|lps>\n";
        return 2;
    }
    Kokkos::initialize(argc, argv);
    {
        CabanaPD::Inputs inputs(argv[1]);
        const double K = inputs["bulk_modulus"];
        const double horizon = inputs["horizon"];
        const std::string which = argv[2];
        if (which == "lps") {
            const double G = inputs["shear_modulus"];
            CabanaPD::ForceModel model(CabanaPD::LPS{}, CabanaPD::NoFracture{}, horizon, K, G, 1);
            simulate(inputs, CabanaPD::LPS{}, model);
        } else {
            CabanaPD::ForceModel model(CabanaPD::PMB{}, CabanaPD::NoFracture{}, horizon, K);
            simulate(inputs, CabanaPD::PMB{}, model);
        }
    }
    Kokkos::finalize();
    return 0;
}
