// LPS brittle fracture of a thin plate with 20 randomly placed pre-notches
// under a traction on its y faces, written against the CabanaPD API (the
// program shape of CabanaPD's examples/mechanics/random_cracks.cpp), built on
// the cabanapd_b200 front end. Usage: random_cracks <input.json>
//
// The traction is a custom boundary functor f_y += +-sigma0/dy on slabs
// within dy of the y faces; it runs as a device kernel every step. Particles
// within one horizon of the y faces cannot break bonds.
#include <array>
#include <cmath>
#include <iomanip>
#include <iostream>
#include <random>
#include <string>

#include <CabanaPD.hpp>

static void run(const std::string& deck)
{
    using exec_space = Kokkos::DefaultExecutionSpace;
    using memory_space = exec_space::memory_space;
    constexpr std::size_t num_notches = 20;

    CabanaPD::Inputs inputs(deck);
    const double rho0 = inputs["density"];
    const double K = inputs["bulk_modulus"];
    const double G = inputs["shear_modulus"];
    const double G0 = inputs["fracture_energy"];
    const double horizon = inputs["horizon"];
    const double sigma0 = inputs["traction"];
    const double min_len = inputs["minimum_prenotch_length"];
    const double max_len = inputs["maximum_prenotch_length"];
    const int seed = inputs.contains("seed") ? static_cast<int>(inputs["seed"]) : 44758454;

    const std::array<double, 3> lo = inputs["low_corner"];
    const std::array<double, 3> hi = inputs["high_corner"];
    const double thickness = hi[2] - lo[2];

    // Notch corner uniform in the plate shrunk by the longest notch; length
    // U(min, max) at angle pi * U in the xy plane; the second edge tilted in
    // yz by up to 45 degrees.
    std::mt19937 gen(seed);
    std::uniform_real_distribution<> unif(0.0, 1.0);
    Kokkos::Array<Kokkos::Array<double, 3>, num_notches> corner, edge1, edge2;
    for (std::size_t k = 0; k < num_notches; k++) {
        const double rx = unif(gen);
        const double ry = unif(gen);
        corner[k] = {(lo[0] + max_len) + ((hi[0] - max_len) - (lo[0] + max_len)) * rx,
                     (lo[1] + max_len) + ((hi[1] - max_len) - (lo[1] + max_len)) * ry, lo[2]};
        const double len = min_len + (max_len - min_len) * unif(gen);
        const double angle = CabanaPD::pi * unif(gen);
        edge1[k] = {len * std::cos(angle), len * std::sin(angle), 0.0};
        const double tilt = unif(gen);
        edge2[k] = {0.0, (-1.0 + 2.0 * tilt) * thickness, thickness};
    }
    CabanaPD::Prenotch<num_notches> notches(edge1, edge2, corner);

    CabanaPD::ForceModel model(CabanaPD::LPS{}, horizon, K, G, G0);

    CabanaPD::Particles particles(memory_space{}, CabanaPD::LPS{});
    particles.domain(inputs);
    particles.create(exec_space{});

    const double dy = particles.dx[1];
    CabanaPD::Region<CabanaPD::RectangularPrism> bottom(lo[0], hi[0], lo[1] - dy, lo[1] + dy,
                                                        lo[2], hi[2]);
    CabanaPD::Region<CabanaPD::RectangularPrism> top(lo[0], hi[0], hi[1] - dy, hi[1] + dy, lo[2],
                                                     hi[2]);

    auto x = particles.sliceReferencePosition();
    auto rho = particles.sliceDensity();
    auto nofail = particles.sliceNoFail();
    const double keep_low = bottom.low[1] + horizon + 1e-10;
    const double keep_high = top.high[1] - horizon - 1e-10;
    particles.update(exec_space{}, KOKKOS_LAMBDA(const int p) {
        rho(p) = rho0;
        if (x(p, 1) <= keep_low || x(p, 1) >= keep_high) nofail(p) = 1;
    });

    CabanaPD::Solver solver(inputs, particles, model);

    const double b0 = sigma0 / dy;
    auto f = solver.particles.sliceForce();
    x = solver.particles.sliceReferencePosition();
    auto pull = KOKKOS_LAMBDA(const int p, const double) {
        const double y = x(p, 1);
        f(p, 1) += b0 * (std::abs(y) / y);
    };
    auto traction = createBoundaryCondition(pull, exec_space{}, solver.particles, true, bottom, top);

    solver.init(traction, notches);
    solver.run(traction);
    std::cout << std::setprecision(17) << "strain energy: " << solver.totalStrainEnergy()
              << " damage: " << solver.totalDamage() << std::endl;
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        std::cerr << "usage: random_cracks <input.json>\n";
        return 2;
    }
    Kokkos::initialize(argc, argv);
    run(argv[1]);
    Kokkos::finalize();
    return 0;
}
