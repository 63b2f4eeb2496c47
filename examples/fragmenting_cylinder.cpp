// A hollow steel cylinder thrown outward until it fragments, written against
// the CabanaPD API (the program shape of CabanaPD's
// examples/mechanics/fragmenting_cylinder.cpp), built on the cabanapd_b200
// front end. Usage: fragmenting_cylinder <input.json>
//
// PMB with critical-stretch fracture inside the shell; with use_contact the
// fragments also repel each other through normal-repulsion contact searched
// on current positions, rebuilt whenever a particle has moved more than the
// search extension since the last build. Particles sit at a random point of
// their grid cell and are kept inside the shell. The program writes the
// initial positions and velocities to cylinder_initial.txt and prints the
// final strain energy and damage.
#include <array>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>

#include <CabanaPD.hpp>

template <class ContactTag>
static void run(CabanaPD::Inputs& inputs, ContactTag)
{
    using exec_space = Kokkos::DefaultExecutionSpace;
    using memory_space = exec_space::memory_space;
    constexpr bool with_contact = !std::is_same<ContactTag, CabanaPD::PMB>::value;

    const double rho0 = inputs["density"];
    const double K = inputs["bulk_modulus"];
    const double sc = inputs["critical_stretch"];
    const double horizon = static_cast<double>(inputs["horizon"]) + 1e-10;
    // Critical stretch to fracture energy, PMB (influence 1) form.
    const double G0 = 9 * K * horizon * (sc * sc) / 5;

    const std::array<double, 3> lo = inputs["low_corner"];
    const std::array<double, 3> hi = inputs["high_corner"];
    const std::array<int, 3> nc = inputs["num_cells"];
    const int m = static_cast<int>(std::floor(horizon / ((hi[0] - lo[0]) / nc[0])));

    CabanaPD::ForceModel model(CabanaPD::PMB{}, horizon, K, G0);

    const double xc = 0.5 * (lo[0] + hi[0]);
    const double yc = 0.5 * (lo[1] + hi[1]);
    const double zc = 0.5 * (lo[2] + hi[2]);
    const double r_out = inputs["cylinder_outer_radius"];
    const double r_in = inputs["cylinder_inner_radius"];
    const double H = inputs["cylinder_height"];
    auto in_shell = KOKKOS_LAMBDA(const int, const double px[3])
    {
        const double rsq = (px[0] - xc) * (px[0] - xc) + (px[1] - yc) * (px[1] - yc);
        return !(rsq < r_in * r_in || rsq > r_out * r_out || px[2] > zc + 0.5 * H ||
                 px[2] < zc - 0.5 * H);
    };

    CabanaPD::Particles particles(memory_space{}, ContactTag{});
    particles.domain(lo, hi, nc, m + 1);
    particles.create(exec_space{}, Cabana::InitRandom{}, in_shell);

    auto x = particles.sliceReferencePosition();
    auto v = particles.sliceVelocity();
    auto rho = particles.sliceDensity();
    const double vr_max = inputs["max_radial_velocity"];
    const double vr_min = inputs["min_radial_velocity"];
    const double vz_max = inputs["max_vertical_velocity"];
    const double z_min = zc - 0.5 * H;
    particles.update(exec_space{}, KOKKOS_LAMBDA(const int p) {
        rho(p) = rho0;
        const double zf = ((x(p, 2) - z_min) / (0.5 * H)) - 1;
        const double vr = vr_max - vr_min * zf * zf;
        const double angle = Kokkos::atan2(x(p, 1), x(p, 0));
        v(p, 0) = vr * Kokkos::cos(angle);
        v(p, 1) = vr * Kokkos::sin(angle);
        v(p, 2) = vz_max * zf;
    });
    {
        std::ofstream out("cylinder_initial.txt");
        out << std::setprecision(17);
        for (std::size_t p = 0; p < particles.size(); p++) {
            const int i = static_cast<int>(p);
            out << x(i, 0) << " " << x(i, 1) << " " << x(i, 2) << " " << v(i, 0) << " "
                << v(i, 1) << " " << v(i, 2) << "\n";
        }
    }

    double W, D;
    if constexpr (with_contact) {
        // Contact radius and search extension in units of the spacing: two
        // particles first touch at dx / 2 each.
        const double dx = particles.dx[0];
        const double r_c = static_cast<double>(inputs["contact_horizon_factor"]) * dx / 2.0;
        const double r_extend = static_cast<double>(inputs["contact_horizon_extend_factor"]) * dx;
        CabanaPD::NormalRepulsionModel contact(horizon, r_c, r_extend, K);
        CabanaPD::Solver solver(inputs, particles, model, contact);
        solver.init();
        solver.run();
        W = solver.totalStrainEnergy();
        D = solver.totalDamage();
    } else {
        CabanaPD::Solver solver(inputs, particles, model);
        solver.init();
        solver.run();
        W = solver.totalStrainEnergy();
        D = solver.totalDamage();
    }
    std::cout << std::setprecision(17) << "particles: " << particles.size() << "\n"
              << "strain energy: " << W << " damage: " << D << std::endl;
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        std::cerr << "usage: fragmenting_cylinder <input.json>\n";
        return 2;
    }
    Kokkos::initialize(argc, argv);
    {
        CabanaPD::Inputs inputs(argv[1]);
        if (static_cast<bool>(inputs["use_contact"]))
            run(inputs, CabanaPD::NormalRepulsionModel{});
        else
            run(inputs, CabanaPD::PMB{});
    }
    Kokkos::finalize();
    return 0;
}
