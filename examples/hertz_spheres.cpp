// Two spheres colliding head-on under Hertzian contact with damping, written
// against the CabanaPD API (HertzianModel as the only force model, as
// CabanaPD's DEM programs use it), built on the cabanapd_b200 front end.
// Usage: hertz_spheres <input.json>
//
// The domain is two cells along x, so the two cell-centre particles sit at
// x = +-dx/2 on the axis; they approach each other at the input speed. The
// program prints the coefficient of restitution sqrt(KE_end / KE_start),
// which the model's restitution input should reproduce.
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
    const double vol0 = inputs["volume"];
    const double radius = inputs["radius"];
    const double extend = inputs["radius_extend"];
    const double nu = inputs["poisson_ratio"];
    const double E = inputs["elastic_modulus"];
    const double e = inputs["restitution"];
    const double speed = inputs["impact_speed"];

    CabanaPD::HertzianModel contact(radius, extend, nu, E, e);

    CabanaPD::Particles particles(memory_space{}, CabanaPD::HertzianModel{},
                                  CabanaPD::BaseOutput{});
    particles.domain(inputs);
    particles.create(exec_space{});

    auto x = particles.sliceReferencePosition();
    auto v = particles.sliceVelocity();
    auto rho = particles.sliceDensity();
    auto vol = particles.sliceVolume();
    particles.update(exec_space{}, KOKKOS_LAMBDA(const int p) {
        rho(p) = rho0;
        vol(p) = vol0;
        v(p, 0) = x(p, 0) > 0.0 ? -speed : speed;
    });

    CabanaPD::Solver solver(inputs, particles, contact);
    auto kinetic = KOKKOS_LAMBDA(const int p, const double) {
        return 0.5 * rho(p) * vol(p) * (v(p, 0) * v(p, 0) + v(p, 1) * v(p, 1) + v(p, 2) * v(p, 2));
    };
    double ke0 = 0.0;
    for (std::size_t p = 0; p < particles.size(); p++) ke0 += kinetic(static_cast<int>(p), 0.0);

    std::array<double, 3> lo = inputs["low_corner"], hi = inputs["high_corner"];
    CabanaPD::Region<CabanaPD::RectangularPrism> box(lo, hi);
    auto energy = CabanaPD::createOutputTimeSeries(
        "output_kinetic_energy.txt", inputs, exec_space{}, solver.particles, kinetic, box);

    solver.init();
    solver.run(energy);
    std::cout << std::setprecision(17) << "restitution: " << std::sqrt(energy.values().back() / ke0)
              << std::endl;
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        std::cerr << "usage: hertz_spheres <input.json>\n";
        return 2;
    }
    Kokkos::initialize(argc, argv);
    run(argv[1]);
    Kokkos::finalize();
    return 0;
}
