// Spherical elastic wave in a unit cube with the linearised LPS model,
// written against the CabanaPD API (the program shape of CabanaPD's
// examples/mechanics/elastic_wave.cpp), built on the cabanapd_b200 front end.
// Usage: elastic_wave <input.json>
//
// A Gaussian radial displacement pulse (amplitude 1e-3, centred on the
// sphere |x| = 0.25, width 0.07) is released from rest; the x displacement
// along the x axis is appended to displacement_profile.txt at the end.
#include <array>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <string>

#include <CabanaPD.hpp>

static void run(const std::string& deck)
{
    using exec_space = Kokkos::DefaultExecutionSpace;
    using memory_space = exec_space::memory_space;

    CabanaPD::Inputs inputs(deck);
    const double rho0 = inputs["density"];
    const double K = inputs["bulk_modulus"];
    const double G = inputs["shear_modulus"];
    const double horizon = static_cast<double>(inputs["horizon"]) + 1e-10;

    const std::array<double, 3> lo = inputs["low_corner"];
    const std::array<double, 3> hi = inputs["high_corner"];
    const std::array<int, 3> cells = inputs["num_cells"];
    const int halo = static_cast<int>(std::floor(horizon / ((hi[0] - lo[0]) / cells[0]))) + 1;

    CabanaPD::ForceModel model(CabanaPD::LinearLPS{}, CabanaPD::NoFracture{}, horizon, K, G);

    CabanaPD::Particles particles(memory_space{}, CabanaPD::LinearLPS{});
    particles.domain(lo, hi, cells, halo);
    particles.create(exec_space{});

    auto x = particles.sliceReferencePosition();
    auto u = particles.sliceDisplacement();
    auto v = particles.sliceVelocity();
    auto rho = particles.sliceDensity();
    particles.update(exec_space{}, KOKKOS_LAMBDA(const int p) {
        const double amplitude = 0.001, r0 = 0.25, width = 0.07;
        rho(p) = rho0;
        const double r = std::sqrt(x(p, 0) * x(p, 0) + x(p, 1) * x(p, 1) + x(p, 2) * x(p, 2));
        const double d = r - r0;
        const double arg = d * d / width / width;
        for (int c = 0; c < 3; c++) {
            const double direction = r > 0.0 ? x(p, c) / r : 0.0;
            u(p, c) = amplitude * std::exp(-arg) * direction;
            v(p, c) = 0.0;
        }
    });

    CabanaPD::Solver solver(inputs, particles, model);
    solver.init();
    solver.run();
    CabanaPD::createDisplacementProfile("displacement_profile.txt", solver.particles, 0);
    std::cout << std::setprecision(17) << "strain energy: " << solver.totalStrainEnergy()
              << std::endl;
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        std::cerr << "usage: elastic_wave <input.json>\n";
        return 2;
    }
    Kokkos::initialize(argc, argv);
    run(argv[1]);
    Kokkos::finalize();
    return 0;
}
