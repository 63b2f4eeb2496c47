// Kalthoff-Winkler impact on a double-notched steel plate, written against
// the CabanaPD API (the program shape of CabanaPD's
// examples/mechanics/kalthoff_winkler.cpp), built on the cabanapd_b200 front
// end. Usage: kalthoff_winkler <input.json>
//
// A strip between the two notches starts at the impactor speed and is held
// there by a zero-force boundary condition; the crack tip's largest |y| among
// particles with damage above 0.3 is written every output step to
// output_kw_crack_y.txt.
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
    const double E = inputs["elastic_modulus"];
    const double nu = 1.0 / 3.0;
    const double K = E / (3.0 * (1.0 - 2.0 * nu));
    const double G0 = inputs["fracture_energy"];
    const double horizon = static_cast<double>(inputs["horizon"]) + 1e-10;
    const double v_impact = inputs["impactor_velocity"];

    const std::array<double, 3> lo = inputs["low_corner"];
    const std::array<double, 3> hi = inputs["high_corner"];
    const std::array<int, 3> cells = inputs["num_cells"];
    const std::array<double, 3> size = inputs["system_size"];
    const int halo = static_cast<int>(std::floor(horizon / ((hi[0] - lo[0]) / cells[0]))) + 1;

    // Two notches from the impacted edge, a quarter of the width apart,
    // through the whole thickness.
    const double notch_y = size[1] / 8.0;
    Kokkos::Array<double, 3> along = {size[0] / 2.0, 0.0, 0.0};
    Kokkos::Array<double, 3> through = {0.0, 0.0, size[2]};
    Kokkos::Array<Kokkos::Array<double, 3>, 2> corners = {
        Kokkos::Array<double, 3>{lo[0], -notch_y, lo[2]},
        Kokkos::Array<double, 3>{lo[0], notch_y, lo[2]}};
    CabanaPD::Prenotch<2> notches(along, through, corners);

    CabanaPD::ForceModel model(CabanaPD::PMB{}, horizon, K, G0);

    CabanaPD::Particles particles(memory_space{}, CabanaPD::PMB{});
    particles.domain(lo, hi, cells, halo);
    particles.create(exec_space{});

    auto x = particles.sliceReferencePosition();
    auto v = particles.sliceVelocity();
    auto rho = particles.sliceDensity();
    const double dx = particles.dx[0];
    const double edge = lo[0];
    particles.update(exec_space{}, KOKKOS_LAMBDA(const int p) {
        rho(p) = rho0;
        if (x(p, 1) > -notch_y && x(p, 1) < notch_y && x(p, 0) < edge + dx) v(p, 0) = v_impact;
    });

    CabanaPD::Solver solver(inputs, particles, model);

    CabanaPD::Region<CabanaPD::RectangularPrism> impact_face(
        edge - dx, edge + dx, -notch_y - 0.25 * dx, notch_y + 0.25 * dx, -size[2], size[2]);
    auto hold = createBoundaryCondition(CabanaPD::ForceValueBCTag{}, 0.0, exec_space{},
                                        solver.particles, impact_face);

    auto damage = solver.particles.sliceDamage();
    auto crack_y = KOKKOS_LAMBDA(const int p, const double) {
        return damage(p) > 0.3 ? x(p, 1) : 0.0;
    };
    CabanaPD::Region<CabanaPD::RectangularPrism> plate(lo, hi);
    auto crack_output = CabanaPD::createOutputTimeSeries<Kokkos::Max<double>>(
        "output_kw_crack_y.txt", inputs, exec_space{}, solver.particles, crack_y, plate);

    solver.init(hold, notches);
    solver.run(hold, crack_output);
    std::cout << std::setprecision(17) << "max crack y: " << crack_output.values().back()
              << std::endl;
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        std::cerr << "usage: kalthoff_winkler <input.json>\n";
        return 2;
    }
    Kokkos::initialize(argc, argv);
    run(argv[1]);
    Kokkos::finalize();
    return 0;
}
