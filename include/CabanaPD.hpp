// CabanaPD-compatible C++ front end over the cabanapd_b200 C ABI.
//
// A Kokkos-free restatement of the user-facing template API of CabanaPD
// (src/CabanaPD.hpp and the headers it includes) for the per-timestep
// mechanics path: Inputs, ForceModel (PMB, LPS, LinearPMB, LinearLPS with
// and without fracture), HertzianModel, NormalRepulsionModel, Particles
// (with output), Region, Prenotch, createBoundaryCondition, BodyTerm,
// Solver, createOutputTimeSeries and createDisplacementProfile keep their
// names, argument meaning and call
// order, so a program written against CabanaPD builds against this header
// (nvcc -x cu --extended-lambda -std=c++17) and runs on the B200 kernels.
//
// Execution model:
// * Particles hold host arrays until a Solver is built; Particles::update
//   functors run on the host, as an initialisation pass.
// * Building a Solver creates the cpd_system, uploads the particles and
//   builds the neighbour list. Slices taken from the solver's particles
//   afterwards carry both the device array and a host mirror: device code
//   (custom boundary-condition and body-term functors, launched on the
//   system's stream between library stages) indexes the device array, host
//   code (output functors) the mirror, which the solver refreshes at output
//   steps before it calls the outputs.
// * The library keeps the caller's particle order (CPD_ORDER_INPUT), so a
//   particle index means the same particle on host and device.
// * Precision: CPD_FP64 unless CABANAPD_B200_PRECISION is "exact" (bitwise
//   reference arithmetic) or "mixed".
// Errors raised by the library become std::runtime_error with its message.
#pragma once

#include <cabanapd_b200.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "cabanapd_shim/inputs.hpp"
#include "cabanapd_shim/kokkos.hpp"

#if defined(__CUDACC__)
#include <cuda_runtime.h>
#endif

namespace CabanaPD {

constexpr double pi = 3.14159265358979323846;

inline void cpdCheck(cpd_status s)
{
    if (s != CPD_OK) throw std::runtime_error(cpd_last_error());
}
inline bool print_rank() { return true; }

// ---------------------------------------------------------------------------
// Tags (src/CabanaPD_Types.hpp).
struct Fracture {};
struct NoFracture {};
struct Elastic {};
struct PMB { static constexpr int32_t pd_id = CPD_PD_PMB; };
struct LPS { static constexpr int32_t pd_id = CPD_PD_LPS; };
struct LinearPMB { static constexpr int32_t pd_id = CPD_PD_LINEAR_PMB; };
struct LinearLPS { static constexpr int32_t pd_id = CPD_PD_LINEAR_LPS; };
struct BaseOutput {};
struct EnergyOutput {};
struct EnergyStressOutput {};
struct TemperatureIndependent {};
struct ForceValueBCTag {};
struct ForceUpdateBCTag {};
struct RectangularPrism {};
struct Line {};
struct NoContact {};

// ---------------------------------------------------------------------------
// Peridynamic force models (src/force_models/CabanaPD_PMB.hpp:27-304,
// src/force_models/CabanaPD_LPS.hpp:26-302): the parameters the kernels need;
// the derived constants (c, s0, bond_break_coeff, theta/s coefficients) are
// computed by the library from these.
template <class ModelTag, class FractureTag>
struct ForceModel {
    using model_tag = ModelTag;
    using model_type = ModelTag;
    using fracture_type = FractureTag;
    static constexpr bool is_contact = false;
    double force_horizon = 0.0, K = 0.0, G = 0.0, G0 = 0.0;
    int influence_type = -1;

    // PMB with fracture: (horizon, K, G0[, influence]).
    ForceModel(ModelTag, double h, double k, double g0, int infl = 1)
        : force_horizon(h), K(k), G0(g0), influence_type(infl) {}
    ForceModel(ModelTag t, Elastic, double h, double k, double g0, int infl = 1)
        : ForceModel(t, h, k, g0, infl) {}
    ForceModel(ModelTag t, Elastic, Fracture, double h, double k, double g0, int infl = 1)
        : ForceModel(t, h, k, g0, infl) {}
    // PMB without fracture: (NoFracture, horizon, K).
    ForceModel(ModelTag, NoFracture, double h, double k) : force_horizon(h), K(k) {}
    ForceModel(ModelTag, Elastic, NoFracture, double h, double k) : force_horizon(h), K(k) {}
    // LPS without fracture: (NoFracture, horizon, K, G[, influence]).
    ForceModel(ModelTag, NoFracture, double h, double k, double g, int infl = 0)
        : force_horizon(h), K(k), G(g), influence_type(infl) {}
    ForceModel(ModelTag, Elastic, NoFracture, double h, double k, double g, int infl = 0)
        : force_horizon(h), K(k), G(g), influence_type(infl) {}
    // LPS with fracture: (horizon, K, G, G0[, influence]).
    ForceModel(ModelTag, double h, double k, double g, double g0, int infl = 0)
        : force_horizon(h), K(k), G(g), G0(g0), influence_type(infl) {}

    void fill(cpd_params& p) const
    {
        p.pd_model = ModelTag::pd_id;
        p.fracture = std::is_same<FractureTag, Fracture>::value ? 1 : 0;
        p.influence_type = influence_type;
        p.horizon = force_horizon;
        p.K = K;
        p.G = G;
        p.G0 = G0;
    }
};

template <class Tag>
ForceModel(Tag, double, double, double) -> ForceModel<Tag, Fracture>;
template <class Tag>
ForceModel(Tag, double, double, double, int) -> ForceModel<Tag, Fracture>;
template <class Tag>
ForceModel(Tag, Elastic, double, double, double) -> ForceModel<Tag, Fracture>;
template <class Tag>
ForceModel(Tag, Elastic, Fracture, double, double, double) -> ForceModel<Tag, Fracture>;
template <class Tag>
ForceModel(Tag, NoFracture, double, double) -> ForceModel<Tag, NoFracture>;
template <class Tag>
ForceModel(Tag, Elastic, NoFracture, double, double) -> ForceModel<Tag, NoFracture>;
template <class Tag>
ForceModel(Tag, NoFracture, double, double, double) -> ForceModel<Tag, NoFracture>;
template <class Tag>
ForceModel(Tag, NoFracture, double, double, double, int) -> ForceModel<Tag, NoFracture>;
template <class Tag>
ForceModel(Tag, Elastic, NoFracture, double, double, double) -> ForceModel<Tag, NoFracture>;
template <class Tag>
ForceModel(Tag, Elastic, NoFracture, double, double, double, int) -> ForceModel<Tag, NoFracture>;
template <class Tag>
ForceModel(Tag, double, double, double, double) -> ForceModel<Tag, Fracture>;
template <class Tag>
ForceModel(Tag, double, double, double, double, int) -> ForceModel<Tag, Fracture>;

// Hertzian contact (src/force_models/CabanaPD_Hertzian.hpp:23-88): radius,
// search-radius extension, Poisson ratio, Young's modulus, restitution.
struct HertzianModel {
    using model_tag = HertzianModel;
    using model_type = HertzianModel;
    using fracture_type = NoFracture;
    static constexpr bool is_contact = true;
    double radius = 0.0, radius_extend = 0.0, nu = 0.0, E = 0.0, e = 0.0;
    HertzianModel() = default;
    HertzianModel(double r, double extend, double nu_, double E_, double e_)
        : radius(r), radius_extend(extend), nu(nu_), E(E_), e(e_) {}
    void fill(cpd_params& p) const
    {
        p.contact_model = CPD_CONTACT_HERTZ;
        p.contact_radius = radius;
        p.radius_extend = radius_extend;
        p.nu = nu;
        p.E = E;
        p.restitution = e;
    }
};

// Normal repulsion contact (src/force_models/CabanaPD_Contact.hpp:54-89):
// (delta, contact radius, search-radius extension, K). Pairs closer than the
// contact radius repel with 15 c (r - radius) / delta vol_j, c as PMB's.
struct NormalRepulsionModel {
    using model_tag = NormalRepulsionModel;
    using model_type = NormalRepulsionModel;
    using fracture_type = NoFracture;
    static constexpr bool is_contact = true;
    double delta = 0.0, radius = 0.0, radius_extend = 0.0, K = 0.0, c = 0.0;
    NormalRepulsionModel() = default;
    NormalRepulsionModel(double delta_, double radius_, double extend, double K_)
        : delta(delta_), radius(radius_), radius_extend(extend), K(K_),
          c(18.0 * K_ / (pi * delta_ * delta_ * delta_ * delta_)) {}
    double cutoff() const { return 2.0 * radius + radius_extend; }
    double extend() const { return radius_extend; }
    void fill(cpd_params& p) const
    {
        p.contact_model = CPD_CONTACT_NORMAL_REPULSION;
        p.contact_radius = radius;
        p.radius_extend = radius_extend;
        p.contact_horizon = delta;
        p.contact_K = K;
    }
};

// ---------------------------------------------------------------------------
// Slices: operator()(i[, d]) reads the device array in device code and the
// host mirror in host code. Vector fields are component-major on both sides.
template <class T>
struct Slice {
    T* host = nullptr;
    int64_t hstride = 0;
    T* dev = nullptr;
    int64_t dstride = 0;
    int64_t n = 0;
    CPD_HD T& operator()(int64_t i, int d = 0) const
    {
#if defined(__CUDA_ARCH__)
        return dev[d * dstride + i];
#else
        return host[d * hstride + i];
#endif
    }
    // Tensor fields (stress): component (a, b) is column 3 a + b.
    CPD_HD T& operator()(int64_t i, int a, int b) const { return (*this)(i, 3 * a + b); }
    std::size_t size() const { return static_cast<std::size_t>(n); }
};

namespace detail {

// Host copy of every particle field plus, once a solver owns the particles,
// the system handle and the device field pointers.
struct ParticleData {
    int64_t n = 0, frozen = 0;
    std::array<double, 3> lo{}, hi{}, dx{};
    std::array<int, 3> nc{};
    std::vector<double> x, u, v, f, vol, rho, W, phi;
    std::vector<int> nofail;
    // EnergyStressOutput particles: the stress mirror, [9][n] (component
    // 3 a + b), refreshed with the others.
    bool with_stress = false;
    std::vector<double> stress;
    cpd_system* sys = nullptr;
    int64_t dstride = 0;
    double *d_x = nullptr, *d_u = nullptr, *d_v = nullptr, *d_f = nullptr, *d_vol = nullptr,
           *d_rho = nullptr, *d_W = nullptr, *d_phi = nullptr, *d_stress = nullptr;

    ParticleData() = default;
    ParticleData(const ParticleData&) = delete;
    ParticleData& operator=(const ParticleData&) = delete;
    ~ParticleData()
    {
        if (sys) cpd_system_destroy(sys);
    }

    // Grow or shrink to m particles keeping the first min(n, m); new ones
    // are zeroed with rho = 1.
    void resize(int64_t m)
    {
        auto resize3 = [&](std::vector<double>& a) {
            std::vector<double> b(3 * m, 0.0);
            for (int d = 0; d < 3; d++)
                for (int64_t i = 0; i < std::min(n, m); i++) b[d * m + i] = a[d * n + i];
            a.swap(b);
        };
        resize3(x);
        resize3(u);
        resize3(v);
        resize3(f);
        vol.resize(m, 0.0);
        rho.resize(m, 1.0);
        W.resize(m, 0.0);
        phi.resize(m, 0.0);
        nofail.resize(m, 0);
        if (with_stress) stress.assign(9 * m, 0.0);
        n = m;
    }
    std::vector<double> interleaved(const std::vector<double>& soa) const
    {
        std::vector<double> a(3 * n);
        for (int64_t i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) a[3 * i + d] = soa[d * n + i];
        return a;
    }
    void download3(int32_t field, std::vector<double>& dst, std::vector<double>& tmp)
    {
        tmp.resize(3 * n);
        cpdCheck(cpd_download(sys, field, tmp.data()));
        for (int64_t i = 0; i < n; i++)
            for (int d = 0; d < 3; d++) dst[d * n + i] = tmp[3 * i + d];
    }
    // Refresh the host mirrors in place (slices keep pointing at them).
    void refresh_mirrors()
    {
        if (!sys) return;
        std::vector<double> tmp;
        download3(CPD_FIELD_U, u, tmp);
        download3(CPD_FIELD_V, v, tmp);
        download3(CPD_FIELD_F, f, tmp);
        cpdCheck(cpd_download(sys, CPD_FIELD_W, W.data()));
        cpdCheck(cpd_download(sys, CPD_FIELD_PHI, phi.data()));
        if (with_stress && d_stress) {
            tmp.resize(9 * n);
            cpdCheck(cpd_download(sys, CPD_FIELD_STRESS, tmp.data()));
            for (int64_t i = 0; i < n; i++)
                for (int c = 0; c < 9; c++) stress[c * n + i] = tmp[9 * i + c];
        }
    }
    // CabanaPD_Force.hpp:222-235 computeStress, for EnergyStressOutput
    // particles (Solver.hpp:243, 486: at init and output steps).
    void compute_stress()
    {
        if (!with_stress || !sys) return;
        cpdCheck(cpd_compute_stress(sys));
        if (!d_stress) {
            void* ptr = nullptr;
            int64_t stride = 0;
            cpdCheck(cpd_device_field(sys, CPD_FIELD_STRESS, &ptr, &stride));
            d_stress = static_cast<double*>(ptr);
        }
    }
};

template <class T>
struct is_init : std::integral_constant<bool, std::is_same<T, Cabana::InitUniform>::value ||
                                                  std::is_same<T, Cabana::InitRandom>::value> {};

// Particle output. The reference writes each output step through Cabana's
// HDF5 (or SILO) particle writer when Cabana was built with one, else it
// only logs that no output is enabled (CabanaPD_Particles.hpp:622-652). Here
// the same fields go to an XDMF file with its heavy data in one raw binary
// file (readable by ParaView and VisIt), when CABANAPD_B200_PARTICLE_OUTPUT
// is set to anything but "0".
inline bool particle_output_enabled()
{
    const char* e = std::getenv("CABANAPD_B200_PARTICLE_OUTPUT");
    return e && *e && std::string(e) != "0";
}

// One output field: its name (the reference's slice label), components per
// particle (1, 3 or 9) and its values in [n][components] order.
struct OutputField {
    std::string name;
    int components = 1;
    std::vector<double> values;
    std::vector<int32_t> ints;  // used instead of values when not empty
};

// <prefix>_<step>.xmf and <prefix>_<step>.bin: a polyvertex grid at time
// `time` with the geometry from `positions` ([n][3]) and one node attribute
// per field, all stored back to back in the .bin file.
inline void write_xdmf_particles(const std::string& prefix, int step, double time, int64_t n,
                                 const OutputField& positions,
                                 const std::vector<OutputField>& fields)
{
    const std::string base = prefix + "_" + std::to_string(step);
    const std::string bin_name = base + ".bin";
    std::ofstream bin(bin_name, std::ios::binary | std::ios::trunc);
    if (!bin) throw std::runtime_error("particle output: cannot write " + bin_name);
    const uint16_t probe = 1;
    const char* endian = (*reinterpret_cast<const unsigned char*>(&probe) == 1) ? "Little" : "Big";
    std::ostringstream xml;
    int64_t offset = 0;
    auto data_item = [&](const OutputField& fld) {
        const bool is_int = !fld.ints.empty();
        const size_t count = static_cast<size_t>(n) * fld.components;
        if ((is_int ? fld.ints.size() : fld.values.size()) != count)
            throw std::runtime_error("particle output: field " + fld.name + " has the wrong size");
        const size_t bytes = count * (is_int ? sizeof(int32_t) : sizeof(double));
        bin.write(is_int ? reinterpret_cast<const char*>(fld.ints.data())
                         : reinterpret_cast<const char*>(fld.values.data()),
                  static_cast<std::streamsize>(bytes));
        xml << "        <DataItem Format=\"Binary\" Dimensions=\"" << n;
        if (fld.components > 1) xml << " " << fld.components;
        xml << "\" NumberType=\"" << (is_int ? "Int" : "Float") << "\" Precision=\""
            << (is_int ? 4 : 8) << "\" Endian=\"" << endian << "\" Seek=\"" << offset << "\">"
            << bin_name.substr(bin_name.find_last_of('/') + 1) << "</DataItem>\n";
        offset += static_cast<int64_t>(bytes);
    };
    xml << "<?xml version=\"1.0\" ?>\n<Xdmf Version=\"3.0\">\n  <Domain>\n"
        << "    <Grid Name=\"particles\" GridType=\"Uniform\">\n"
        << "      <Time Value=\"" << std::setprecision(17) << time << "\"/>\n"
        << "      <Topology TopologyType=\"Polyvertex\" NumberOfElements=\"" << n << "\"/>\n"
        << "      <Geometry GeometryType=\"XYZ\">\n";
    data_item(positions);
    xml << "      </Geometry>\n";
    for (const OutputField& fld : fields) {
        const char* kind = fld.components == 1 ? "Scalar" : fld.components == 3 ? "Vector" : "Tensor";
        xml << "      <Attribute Name=\"" << fld.name << "\" AttributeType=\"" << kind
            << "\" Center=\"Node\">\n";
        data_item(fld);
        xml << "      </Attribute>\n";
    }
    xml << "    </Grid>\n  </Domain>\n</Xdmf>\n";
    if (!bin) throw std::runtime_error("particle output: writing " + bin_name + " failed");
    std::ofstream(base + ".xmf", std::ios::trunc) << xml.str();
}

}  // namespace detail

// ---------------------------------------------------------------------------
// Particles (src/CabanaPD_Particles.hpp:81-686).
template <class MemorySpace = Kokkos::CudaSpace, class ModelTag = PMB, class... Rest>
class Particles {
  public:
    using memory_space = MemorySpace;
    using execution_space = typename MemorySpace::execution_space;
    static constexpr int dim = 3;
    Kokkos::Array<double, 3> dx{};
    Kokkos::Array<double, 3> local_mesh_lo{}, local_mesh_hi{};
    Kokkos::Array<double, 3> ghost_mesh_lo{}, ghost_mesh_hi{};

    Particles(MemorySpace, ModelTag, Rest...) : d_(std::make_shared<detail::ParticleData>())
    {
        d_->with_stress = (std::is_same<Rest, EnergyStressOutput>::value || ... || false);
    }

    void domain(std::array<double, 3> low, std::array<double, 3> high, std::array<int, 3> num_cells,
                int /*halo_width*/)
    {
        d_->lo = low;
        d_->hi = high;
        d_->nc = num_cells;
        for (int d = 0; d < 3; d++) {
            d_->dx[d] = (high[d] - low[d]) / num_cells[d];
            dx[d] = d_->dx[d];
            local_mesh_lo[d] = ghost_mesh_lo[d] = low[d];
            local_mesh_hi[d] = ghost_mesh_hi[d] = high[d];
        }
    }
    void domain(const Inputs& inputs, int halo_width = 1)
    {
        std::array<double, 3> lo = inputs["low_corner"], hi = inputs["high_corner"];
        std::array<int, 3> nc = inputs["num_cells"];
        domain(lo, hi, nc, halo_width);
    }

    // One particle per cell at the cell centre (x index fastest), kept where
    // user(pid, px) is true; vol = cell volume, rho = 1, nofail = 0, u = v =
    // f = 0 (CabanaPD_Particles.hpp:242-307). Cabana::InitRandom places the
    // particle at a seeded uniform random point of its cell instead.
    template <class ExecSpace>
    void create(const ExecSpace&)
    {
        create_cells(Cabana::InitUniform{}, AllCells{}, 0, false);
    }
    template <class ExecSpace, class UserFunctor,
              class = typename std::enable_if<!detail::is_init<UserFunctor>::value>::type>
    void create(const ExecSpace&, UserFunctor user, std::size_t num_previous = 0,
                bool create_frozen = false)
    {
        create_cells(Cabana::InitUniform{}, user, num_previous, create_frozen);
    }
    template <class ExecSpace, class InitType, class UserFunctor,
              class = typename std::enable_if<detail::is_init<InitType>::value>::type>
    void create(const ExecSpace&, InitType init, UserFunctor user, std::size_t num_previous = 0,
                bool create_frozen = false)
    {
        create_cells(init, user, num_previous, create_frozen);
    }

    // Runs functor(pid) on the host for pid in [frozen, n) (or [0, n)).
    template <class ExecSpace, class Functor>
    void update(const ExecSpace&, Functor functor, bool update_frozen = false)
    {
        if (d_->sys)
            throw std::runtime_error("Particles::update after the solver was built is not supported");
        const int64_t start = update_frozen ? 0 : d_->frozen;
        for (int64_t p = start; p < d_->n; p++) functor(static_cast<int>(p));
    }

    Slice<double> sliceReferencePosition() const { return slice(d_->x, d_->d_x); }
    Slice<double> sliceDisplacement() const { return slice(d_->u, d_->d_u); }
    Slice<double> sliceVelocity() const { return slice(d_->v, d_->d_v); }
    Slice<double> sliceForce() const { return slice(d_->f, d_->d_f); }
    Slice<double> sliceVolume() const { return slice(d_->vol, d_->d_vol); }
    Slice<double> sliceDensity() const { return slice(d_->rho, d_->d_rho); }
    Slice<double> sliceStrainEnergy() const { return slice(d_->W, d_->d_W); }
    Slice<double> sliceDamage() const { return slice(d_->phi, d_->d_phi); }
    // Particles built with EnergyStressOutput: stress(i, a, b), computed at
    // init and output steps.
    Slice<double> sliceStress() const
    {
        if (!d_->with_stress)
            throw std::runtime_error("sliceStress: particles were not built with EnergyStressOutput");
        return slice(d_->stress, d_->d_stress);
    }
    // Host-only: the no-fail flags are uploaded with the particles.
    Slice<int> sliceNoFail() const
    {
        Slice<int> s;
        s.host = d_->nofail.data();
        s.hstride = d_->n;
        s.n = d_->n;
        return s;
    }

    std::size_t numLocal() const { return static_cast<std::size_t>(d_->n - d_->frozen); }
    std::size_t numFrozen() const { return static_cast<std::size_t>(d_->frozen); }
    std::size_t frozenOffset() const { return static_cast<std::size_t>(d_->frozen); }
    std::size_t localOffset() const { return static_cast<std::size_t>(d_->n); }
    std::size_t referenceOffset() const { return static_cast<std::size_t>(d_->n); }
    std::size_t size() const { return static_cast<std::size_t>(d_->n); }
    unsigned long long numGlobal() const { return static_cast<unsigned long long>(d_->n); }
    int rank() const { return 0; }

    const std::shared_ptr<detail::ParticleData>& data() const { return d_; }

    // Particles::output (CabanaPD_Particles.hpp:622-652 with the field lists
    // of :785-791, :1192-1199, :1323-1331): positions (reference or current),
    // forces, displacements, velocities and type, then strain energy and
    // damage, the LPS weighted volume and dilatation, and the stress of
    // EnergyStressOutput particles, as particles_<output_step>.xmf / .bin
    // when CABANAPD_B200_PARTICLE_OUTPUT is set (else a one-time notice, as
    // the reference logs without an output library). The solver calls it at
    // init and at output steps with the host mirrors refreshed.
    void output(int output_step, double output_time, bool use_reference) const
    {
        if (!detail::particle_output_enabled()) {
            static bool told = false;
            if (!told) std::cout << "No particle output enabled." << std::endl;
            told = true;
            return;
        }
        const int64_t n = d_->n;
        auto aos = [&](const std::vector<double>& soa, int comps) {
            std::vector<double> a(static_cast<size_t>(n) * comps);
            for (int64_t i = 0; i < n; i++)
                for (int c = 0; c < comps; c++) a[comps * i + c] = soa[c * n + i];
            return a;
        };
        detail::OutputField pos{use_reference ? "reference_positions" : "current_positions", 3,
                                aos(d_->x, 3), {}};
        if (!use_reference)
            for (int64_t i = 0; i < n; i++)
                for (int c = 0; c < 3; c++) pos.values[3 * i + c] += d_->u[c * n + i];
        std::vector<detail::OutputField> fields;
        fields.push_back({"forces", 3, aos(d_->f, 3), {}});
        fields.push_back({"displacements", 3, aos(d_->u, 3), {}});
        fields.push_back({"velocities", 3, aos(d_->v, 3), {}});
        fields.push_back({"type", 1, {}, std::vector<int32_t>(static_cast<size_t>(n), 0)});
        fields.push_back({"strain_energy", 1, d_->W, {}});
        fields.push_back({"damage", 1, d_->phi, {}});
        constexpr bool lps = std::is_same<ModelTag, LPS>::value ||
                             std::is_same<ModelTag, LinearLPS>::value;
        if (lps && d_->sys) {
            std::vector<double> m(static_cast<size_t>(n)), theta(static_cast<size_t>(n));
            cpdCheck(cpd_download(d_->sys, CPD_FIELD_M, m.data()));
            cpdCheck(cpd_download(d_->sys, CPD_FIELD_THETA, theta.data()));
            fields.push_back({"weighted_volume", 1, std::move(m), {}});
            fields.push_back({"dilatation", 1, std::move(theta), {}});
        }
        if (d_->with_stress) fields.push_back({"stress", 9, aos(d_->stress, 9), {}});
        detail::write_xdmf_particles("particles", output_step, output_time, n, pos, fields);
    }

  private:
    struct AllCells {
        bool operator()(int, const double*) const { return true; }
    };

    Slice<double> slice(std::vector<double>& host, double* dev) const
    {
        Slice<double> s;
        s.host = host.data();
        s.hstride = d_->n;
        s.dev = dev;
        s.dstride = d_->dstride;
        s.n = d_->n;
        return s;
    }

    template <class InitType, class UserFunctor>
    void create_cells(InitType, UserFunctor user, std::size_t num_previous, bool create_frozen)
    {
        if (d_->nc[0] <= 0 || d_->nc[1] <= 0 || d_->nc[2] <= 0)
            throw std::runtime_error("Cannot create() particles without calling domain() first.");
        if (d_->sys) throw std::runtime_error("Cannot create() particles after the solver was built.");
        if (static_cast<int64_t>(num_previous) > d_->n)
            throw std::runtime_error("create(): num_previous exceeds the existing particles");
        constexpr bool random = std::is_same<InitType, Cabana::InitRandom>::value;
        std::mt19937_64 gen(0x5eed2024ULL + num_previous);
        std::uniform_real_distribution<double> unif(0.0, 1.0);
        std::vector<double> pos;
        const double cell_vol = d_->dx[0] * d_->dx[1] * d_->dx[2];
        int pid = static_cast<int>(num_previous);
        for (int k = 0; k < d_->nc[2]; k++)
            for (int j = 0; j < d_->nc[1]; j++)
                for (int i = 0; i < d_->nc[0]; i++) {
                    const int idx[3] = {i, j, k};
                    double px[3];
                    for (int d = 0; d < 3; d++) {
                        const double lo = d_->lo[d] + idx[d] * d_->dx[d];
                        const double hi = d_->lo[d] + (idx[d] + 1.0) * d_->dx[d];
                        const double t = random ? unif(gen) : 0.5;
                        px[d] = lo + t * (hi - lo);
                    }
                    if (user(pid, px)) {
                        pos.insert(pos.end(), px, px + 3);
                        pid++;
                    }
                }
        const int64_t added = static_cast<int64_t>(pos.size() / 3);
        const int64_t base = static_cast<int64_t>(num_previous);
        d_->resize(base);
        d_->resize(base + added);
        const int64_t m = d_->n;
        for (int64_t p = 0; p < added; p++) {
            for (int d = 0; d < 3; d++) d_->x[d * m + base + p] = pos[3 * p + d];
            d_->vol[base + p] = cell_vol;
        }
        if (create_frozen) d_->frozen = m;
    }

    std::shared_ptr<detail::ParticleData> d_;
};

// ---------------------------------------------------------------------------
// Regions (src/CabanaPD_Geometry.hpp:54-168).
template <class Kind>
struct Region;

template <>
struct Region<RectangularPrism> {
    Kokkos::Array<double, 3> low, high;
    Region(double lx, double hx, double ly, double hy, double lz, double hz)
    {
        low[0] = lx;
        high[0] = hx;
        low[1] = ly;
        high[1] = hy;
        low[2] = lz;
        high[2] = hz;
    }
    template <class A>
    Region(const A& lo, const A& hi)
    {
        for (int d = 0; d < 3; d++) {
            low[d] = lo[d];
            high[d] = hi[d];
        }
    }
    template <class S>
    CPD_HD bool inside(const S& x, int64_t pid) const
    {
        return x(pid, 0) >= low[0] && x(pid, 0) <= high[0] && x(pid, 1) >= low[1] &&
               x(pid, 1) <= high[1] && x(pid, 2) >= low[2] && x(pid, 2) <= high[2];
    }
};

template <>
struct Region<Line> {
    Kokkos::Array<int, 2> dims;
    Kokkos::Array<double, 2> half_dx;
    template <class A>
    Region(int profile_dim, const A& dx)
    {
        dims[0] = (profile_dim + 1) % 3;
        dims[1] = (profile_dim + 2) % 3;
        half_dx[0] = dx[dims[0]] / 2.0;
        half_dx[1] = dx[dims[1]] / 2.0;
    }
    template <class S>
    CPD_HD bool inside(const S& x, int64_t pid) const
    {
        return x(pid, dims[0]) < half_dx[0] && x(pid, dims[0]) > -half_dx[0] &&
               x(pid, dims[1]) < half_dx[1] && x(pid, dims[1]) > -half_dx[1];
    }
};

// ParticleSteeringVector (CabanaPD_Geometry.hpp:170-273): ascending indices
// of the particles in [frozen, n) inside any of the regions.
template <class ParticleType, class... R>
std::vector<int64_t> steeringIndices(const ParticleType& particles, const R&... regions)
{
    std::vector<int64_t> idx;
    const auto x = particles.sliceReferencePosition();
    for (int64_t p = static_cast<int64_t>(particles.frozenOffset());
         p < static_cast<int64_t>(particles.localOffset()); p++) {
        bool in = false;
        ((in = in || regions.inside(x, p)), ...);
        if (in) idx.push_back(p);
    }
    return idx;
}

// ---------------------------------------------------------------------------
// Pre-notches (src/CabanaPD_Prenotch.hpp:174-213): one orientation for all
// notches, or one per notch.
template <std::size_t NumNotch>
struct Prenotch {
    std::vector<double> v1, v2, p0;
    Prenotch() = default;
    Prenotch(Kokkos::Array<double, 3> a, Kokkos::Array<double, 3> b,
             Kokkos::Array<Kokkos::Array<double, 3>, NumNotch> o)
    {
        for (std::size_t k = 0; k < NumNotch; k++)
            for (int d = 0; d < 3; d++) {
                v1.push_back(a[d]);
                v2.push_back(b[d]);
                p0.push_back(o[k][d]);
            }
    }
    Prenotch(Kokkos::Array<Kokkos::Array<double, 3>, NumNotch> a,
             Kokkos::Array<Kokkos::Array<double, 3>, NumNotch> b,
             Kokkos::Array<Kokkos::Array<double, 3>, NumNotch> o)
    {
        for (std::size_t k = 0; k < NumNotch; k++)
            for (int d = 0; d < 3; d++) {
                v1.push_back(a[k][d]);
                v2.push_back(b[k][d]);
                p0.push_back(o[k][d]);
            }
    }
};

// ---------------------------------------------------------------------------
// Boundary conditions (src/CabanaPD_Boundary.hpp:34-204) and body terms
// (src/CabanaPD_BodyTerm.hpp:25-69). ForceValue / ForceUpdate run inside the
// library; custom functors f(pid, time) run as device kernels on the system
// stream: after the force for force-update conditions, before it otherwise.
template <class Kind>
struct BoundaryCondition {
    Kind user;
    std::vector<int64_t> indices;
    bool force_update = true;
    bool forceUpdate() const { return force_update; }
};
template <>
struct BoundaryCondition<ForceValueBCTag> {
    double value = 0.0;
    std::vector<int64_t> indices;
    bool forceUpdate() const { return true; }
};
template <>
struct BoundaryCondition<ForceUpdateBCTag> {
    double value = 0.0;
    std::vector<int64_t> indices;
    bool forceUpdate() const { return true; }
};

template <class ExecSpace, class ParticleType, class... R>
BoundaryCondition<ForceValueBCTag> createBoundaryCondition(ForceValueBCTag, double value, ExecSpace,
                                                           const ParticleType& p, R... regions)
{
    return {value, steeringIndices(p, regions...)};
}
template <class ExecSpace, class ParticleType, class... R>
BoundaryCondition<ForceUpdateBCTag> createBoundaryCondition(ForceUpdateBCTag, double value,
                                                            ExecSpace, const ParticleType& p,
                                                            R... regions)
{
    return {value, steeringIndices(p, regions...)};
}
template <class UserFunctor, class ExecSpace, class ParticleType, class... R,
          class = typename std::enable_if<!std::is_same<UserFunctor, ForceValueBCTag>::value &&
                                          !std::is_same<UserFunctor, ForceUpdateBCTag>::value>::type>
BoundaryCondition<UserFunctor> createBoundaryCondition(UserFunctor user, ExecSpace,
                                                       const ParticleType& p, bool force_update,
                                                       R... regions)
{
    return {user, steeringIndices(p, regions...), force_update};
}

template <class UserFunctor>
struct BodyTerm {
    UserFunctor user;
    std::size_t particle_count;
    bool force_update;
    bool update_frozen;
    BodyTerm(UserFunctor u, std::size_t count, bool force, bool frozen = false)
        : user(u), particle_count(count), force_update(force), update_frozen(frozen) {}
    bool forceUpdate() const { return force_update; }
};

namespace detail {

template <class T>
struct is_builtin_bc : std::false_type {};
template <>
struct is_builtin_bc<BoundaryCondition<ForceValueBCTag>> : std::true_type {
    static constexpr int32_t kind = CPD_BC_FORCE_VALUE;
};
template <>
struct is_builtin_bc<BoundaryCondition<ForceUpdateBCTag>> : std::true_type {
    static constexpr int32_t kind = CPD_BC_FORCE_UPDATE;
};
template <class T>
struct is_body_term : std::false_type {};
template <class U>
struct is_body_term<BodyTerm<U>> : std::true_type {};
template <class T>
struct is_condition : std::false_type {};
template <class U>
struct is_condition<BoundaryCondition<U>> : std::true_type {};
template <class U>
struct is_condition<BodyTerm<U>> : std::true_type {};

#if defined(__CUDACC__)
template <class F>
__global__ void apply_indexed(F f, const int64_t* idx, int64_t count, double time)
{
    const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (b < count) f(static_cast<int>(idx[b]), time);
}
template <class F>
__global__ void apply_range(F f, int64_t begin, int64_t end, double time)
{
    const int64_t p = begin + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p < end) f(static_cast<int>(p), time);
}
inline void check_launch()
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("boundary kernel launch failed: ") +
                                 cudaGetErrorString(e));
}
#endif

// A custom boundary condition or body term bound to one system.
class UserStage {
  public:
    virtual ~UserStage() = default;
    virtual void apply(double time) = 0;
    bool force_update = true;
};

template <class BC>
class UserStageImpl final : public UserStage {
  public:
    UserStageImpl(const BC& bc, cpd_system* sys, int64_t frozen, int64_t n)
        : bc_(bc), sys_(sys), frozen_(frozen), n_(n)
    {
        force_update = bc.forceUpdate();
#if defined(__CUDACC__)
        if constexpr (!is_body_term<BC>::value) {
            count_ = static_cast<int64_t>(bc_.indices.size());
            if (count_ > 0) {
                if (cudaMalloc(&d_idx_, sizeof(int64_t) * count_) != cudaSuccess)
                    throw std::runtime_error("cudaMalloc of boundary indices failed");
                if (cudaMemcpy(d_idx_, bc_.indices.data(), sizeof(int64_t) * count_,
                               cudaMemcpyHostToDevice) != cudaSuccess)
                    throw std::runtime_error("copy of boundary indices failed");
            }
        }
#else
        throw std::runtime_error(
            "custom boundary conditions and body terms run as device functors: build with nvcc "
            "--extended-lambda");
#endif
    }
    ~UserStageImpl() override
    {
#if defined(__CUDACC__)
        if (d_idx_) cudaFree(d_idx_);
#endif
    }
    void apply(double time) override
    {
#if defined(__CUDACC__)
        void* st = nullptr;
        cpdCheck(cpd_get_stream(sys_, &st));
        const cudaStream_t stream = static_cast<cudaStream_t>(st);
        if constexpr (is_body_term<BC>::value) {
            const int64_t begin = bc_.update_frozen ? 0 : frozen_;
            if (n_ > begin) {
                apply_range<<<static_cast<unsigned>((n_ - begin + 255) / 256), 256, 0, stream>>>(
                    bc_.user, begin, n_, time);
                check_launch();
            }
        } else if (count_ > 0) {
            apply_indexed<<<static_cast<unsigned>((count_ + 255) / 256), 256, 0, stream>>>(
                bc_.user, d_idx_, count_, time);
            check_launch();
        }
#else
        (void)time;
#endif
    }

  private:
    BC bc_;
    cpd_system* sys_;
    int64_t frozen_, n_;
    int64_t count_ = 0;
    int64_t* d_idx_ = nullptr;
};

}  // namespace detail

// ---------------------------------------------------------------------------
// Outputs (src/CabanaPD_OutputProfiles.hpp:27-215), evaluated on the host
// from the mirrors the solver refreshes at output steps.
template <class Reducer, class Functor>
class OutputTimeSeries {
  public:
    OutputTimeSeries(std::string name, std::vector<int64_t> idx, Functor f)
        : name_(std::move(name)), idx_(std::move(idx)), f_(f) {}
    void update(double time)
    {
        double acc = Reducer::identity();
        for (int64_t p : idx_) acc = Reducer::join(acc, f_(static_cast<int>(p), time));
        values_.push_back(acc);
    }
    // "value  value/num_particles" per output step, appended to the file.
    void print() const
    {
        std::ofstream out(name_, std::ios::app);
        for (double v : values_)
            out << std::fixed << std::setprecision(15) << v << "  "
                << v / static_cast<double>(idx_.size()) << "\n";
    }
    const std::vector<double>& values() const { return values_; }

  private:
    std::string name_;
    std::vector<int64_t> idx_;
    Functor f_;
    std::vector<double> values_;
};

template <class Functor, class ExecSpace, class ParticleType, class Geometry>
OutputTimeSeries<Kokkos::Sum<double>, Functor> createOutputTimeSeries(std::string name,
                                                                      const Inputs&, ExecSpace,
                                                                      const ParticleType& p,
                                                                      Functor user,
                                                                      const Geometry& geom)
{
    return OutputTimeSeries<Kokkos::Sum<double>, Functor>(name, steeringIndices(p, geom), user);
}
template <class Reducer, class Functor, class ExecSpace, class ParticleType, class Geometry>
OutputTimeSeries<Reducer, Functor> createOutputTimeSeries(std::string name, const Inputs&,
                                                          ExecSpace, const ParticleType& p,
                                                          Functor user, const Geometry& geom)
{
    return OutputTimeSeries<Reducer, Functor>(name, steeringIndices(p, geom), user);
}

// "rank x value" lines for the particles on the line through the origin
// along profile_dim (CabanaPD_OutputProfiles.hpp:27-84), appended to file.
template <class ParticleType, class UserFunctor>
void createOutputProfile(const std::string& file, ParticleType particles, int profile_dim,
                         UserFunctor user)
{
    particles.data()->refresh_mirrors();
    Region<Line> line(profile_dim, particles.dx);
    const auto x = particles.sliceReferencePosition();
    std::ofstream out(file, std::ios::app);
    out << std::setprecision(17);
    for (int64_t p : steeringIndices(particles, line))
        out << particles.rank() << " " << x(p, profile_dim) << " " << user(static_cast<int>(p))
            << "\n";
}
template <class ParticleType>
void createDisplacementProfile(const std::string& file, ParticleType particles, int profile_dim,
                               int displacement_dim = -1)
{
    if (displacement_dim == -1) displacement_dim = profile_dim;
    const auto u = particles.sliceDisplacement();
    createOutputProfile(file, particles, profile_dim,
                        [=](int p) { return u(p, displacement_dim); });
}
template <class ParticleType>
void createDisplacementMagnitudeProfile(const std::string& file, ParticleType particles,
                                        int profile_dim)
{
    const auto u = particles.sliceDisplacement();
    createOutputProfile(file, particles, profile_dim, [=](int p) {
        return std::sqrt(u(p, 0) * u(p, 0) + u(p, 1) * u(p, 1) + u(p, 2) * u(p, 2));
    });
}

// ---------------------------------------------------------------------------
// Solver (src/CabanaPD_Solver.hpp:87-657). Each step runs the library's four
// stages with any custom boundary functor between them, in runStep's order
// (Solver.hpp:332-375); energy and damage are computed every
// output_frequency steps (Solver.hpp:479-495).
template <class ParticleType, class ForceModelType, class ContactModelType = NoContact>
class Solver {
  public:
    ParticleType particles;
    int num_steps = 0;
    int output_frequency = 1;
    double dt = 0.0;

    Solver(Inputs inputs, ParticleType p, ForceModelType model)
        : particles(p), inputs_(std::move(inputs))
    {
        cpd_params prm{};
        model.fill(prm);
        setup(prm, !ForceModelType::is_contact);
    }
    Solver(Inputs inputs, ParticleType p, ForceModelType model, ContactModelType contact)
        : particles(p), inputs_(std::move(inputs))
    {
        cpd_params prm{};
        model.fill(prm);
        contact.fill(prm);
        setup(prm, !ForceModelType::is_contact);
    }
    Solver(const Solver&) = delete;
    Solver& operator=(const Solver&) = delete;

    void init(bool initial_output = true)
    {
        initial_output_ = initial_output;
        init_stages(static_cast<NoCondition*>(nullptr));
    }
    template <std::size_t N>
    void init(const Prenotch<N>& notch, bool initial_output = true)
    {
        apply_prenotch(notch);
        init(initial_output);
    }
    template <class BC, class = typename std::enable_if<detail::is_condition<BC>::value>::type>
    void init(BC& bc, bool initial_output = true)
    {
        initial_output_ = initial_output;
        init_stages(&bc);
    }
    template <class BC, std::size_t N>
    void init(BC& bc, const Prenotch<N>& notch, bool initial_output = true)
    {
        initial_output_ = initial_output;
        apply_prenotch(notch);
        init_stages(&bc);
    }

    void run() { run_steps(); }
    // run(bc, outputs...) as in the reference; a condition not given to
    // init() is attached here and acts from the first step.
    template <class First, class... Out>
    void run(First& first, Out&... outputs)
    {
        if constexpr (detail::is_condition<First>::value) {
            if (!bc_bound_) bind(first);
            run_steps(outputs...);
        } else {
            run_steps(first, outputs...);
        }
    }

    // Drop the particles in [frozen, n) (or [0, n)) whose force magnitude
    // exceeds threshold, keeping the others' state and forces
    // (Solver.hpp:298-330). The library system is rebuilt for the remaining
    // particles; call it before attaching boundary conditions.
    void remove(double threshold, bool use_frozen = false)
    {
        const auto& d = particles.data();
        if (bc_bound_)
            throw std::runtime_error("Solver::remove after a boundary condition was attached");
        d->refresh_mirrors();
        const int64_t n = d->n, first = use_frozen ? 0 : d->frozen;
        std::vector<int64_t> kept;
        int64_t frozen_kept = 0;
        for (int64_t p = 0; p < n; p++) {
            const bool drop =
                p >= first &&
                std::hypot(d->f[p], d->f[n + p], d->f[2 * n + p]) > threshold;
            if (drop) continue;
            kept.push_back(p);
            if (p < d->frozen) frozen_kept++;
        }
        const int64_t m = static_cast<int64_t>(kept.size());
        if (m == n) return;
        auto pick3 = [&](std::vector<double>& a) {
            std::vector<double> b(3 * m);
            for (int dd = 0; dd < 3; dd++)
                for (int64_t k = 0; k < m; k++) b[dd * m + k] = a[dd * n + kept[k]];
            a.swap(b);
        };
        auto pick = [&](auto& a) {
            std::remove_reference_t<decltype(a)> b(m);
            for (int64_t k = 0; k < m; k++) b[k] = a[kept[k]];
            a.swap(b);
        };
        pick3(d->x);
        pick3(d->u);
        pick3(d->v);
        pick3(d->f);
        pick(d->vol);
        pick(d->rho);
        pick(d->W);
        pick(d->phi);
        pick(d->nofail);
        d->n = m;
        d->frozen = frozen_kept;
        cpdCheck(cpd_system_destroy(d->sys));
        d->sys = nullptr;
        const std::vector<double> f_kept = d->f;
        setup_system();
        if (initialized_) {
            cpdCheck(cpd_init(d->sys));
#if defined(__CUDACC__)
            for (int dd = 0; dd < 3; dd++)
                if (cudaMemcpy(d->d_f + dd * d->dstride, f_kept.data() + dd * m,
                               sizeof(double) * m, cudaMemcpyHostToDevice) != cudaSuccess)
                    throw std::runtime_error("restoring forces after remove failed");
#else
            throw std::runtime_error("Solver::remove needs the nvcc build of this header");
#endif
        }
    }

    // Totals of the last energy evaluation (output steps and init).
    double totalStrainEnergy() const { return last_W_; }
    double totalDamage() const { return last_D_; }

  private:
    struct NoCondition {};

    void setup(cpd_params prm, bool mechanics)
    {
        const auto t0 = std::chrono::steady_clock::now();
        const auto& d = particles.data();
        if (d->sys) throw std::runtime_error("these particles already belong to a solver");
        if (d->n == 0) throw std::runtime_error("no particles: call Particles::create first");
        if (mechanics) inputs_.computeCriticalTimeStep();
        num_steps = inputs_["num_steps"];
        output_frequency = inputs_["output_frequency"];
        dt = inputs_["timestep"];
        prm.dt = dt;
        prm.precision = precision_from_env();
        prm.ordering = CPD_ORDER_INPUT;
        params_ = prm;
        setup_system();
        int32_t max_n = 0;
        int64_t total = 0;
        cpdCheck(cpd_neighbor_stats(d->sys, &max_n, &total));
        output_file_ = inputs_.contains("output_file") ? static_cast<std::string>(inputs_["output_file"])
                                                       : std::string("cabanaPD.out");
        output_reference_ = inputs_.contains("output_reference")
                                ? static_cast<bool>(inputs_["output_reference"])
                                : true;
        std::ofstream out(output_file_, std::ofstream::app);
        const std::time_t now = std::time(nullptr);
        out << "CabanaPD (cabanapd_b200) " << std::ctime(&now) << "\n"
            << "Local particles, Ghosted particles, Global particles\n"
            << particles.numLocal() << ", 0, " << particles.numGlobal() << "\n"
            << "Maximum neighbors: " << max_n << ", Total neighbors: " << total << "\n\n";
        init_time_ += seconds_since(t0);
    }

    // Create the library system from params_ and the host particle arrays,
    // build the neighbour list and record the device field pointers.
    void setup_system()
    {
        const auto& d = particles.data();
        cpdCheck(cpd_system_create(&params_, &d->sys));
        d->d_stress = nullptr;
        const int64_t n = d->n;
        const std::vector<double> xi = d->interleaved(d->x);
        const std::vector<int32_t> nofail(d->nofail.begin(), d->nofail.end());
        cpdCheck(cpd_upload_particles(d->sys, n, d->frozen, xi.data(), d->vol.data(),
                                      d->rho.data(), nofail.data(), nullptr));
        const std::vector<double> ui = d->interleaved(d->u);
        const std::vector<double> vi = d->interleaved(d->v);
        cpdCheck(cpd_set_state(d->sys, ui.data(), vi.data()));
        cpdCheck(cpd_build_neighbors(d->sys));
        const std::pair<int32_t, double**> fields[] = {
            {CPD_FIELD_X, &d->d_x},     {CPD_FIELD_U, &d->d_u},     {CPD_FIELD_V, &d->d_v},
            {CPD_FIELD_F, &d->d_f},     {CPD_FIELD_VOL, &d->d_vol}, {CPD_FIELD_RHO, &d->d_rho},
            {CPD_FIELD_W, &d->d_W},     {CPD_FIELD_PHI, &d->d_phi}};
        for (const auto& fp : fields) {
            void* ptr = nullptr;
            int64_t stride = 0;
            cpdCheck(cpd_device_field(d->sys, fp.first, &ptr, &stride));
            *fp.second = static_cast<double*>(ptr);
            d->dstride = stride;
        }
    }

    template <class BC>
    void bind(BC& bc)
    {
        bc_bound_ = true;
        const auto& d = particles.data();
        if constexpr (detail::is_builtin_bc<BC>::value) {
            const double value = bc.value;
            cpdCheck(cpd_add_boundary_condition(d->sys, detail::is_builtin_bc<BC>::kind, 0,
                                                static_cast<int64_t>(bc.indices.size()),
                                                bc.indices.data(), &value));
        } else {
            stage_ = std::make_unique<detail::UserStageImpl<BC>>(bc, d->sys, d->frozen, d->n);
        }
    }

    template <class BC>
    void init_stages(BC* bc)
    {
        const auto t0 = std::chrono::steady_clock::now();
        const auto& d = particles.data();
        if constexpr (!std::is_same<BC, NoCondition>::value) bind(*bc);
        // Non-force conditions act before the initial force, force
        // conditions after it (Solver.hpp:251-281).
        if (stage_ && !stage_->force_update) stage_->apply(0.0);
        cpdCheck(cpd_init(d->sys));
        initialized_ = true;
        if (stage_ && stage_->force_update) stage_->apply(0.0);
        if (d->with_stress) d->compute_stress();
        if (d->with_stress || (initial_output_ && detail::particle_output_enabled()))
            d->refresh_mirrors();
        cpdCheck(cpd_synchronize(d->sys));
        // Solver.hpp:245-246: the initial particle output.
        if (initial_output_) particles.output(0, 0.0, output_reference_);
        init_time_ += seconds_since(t0);
    }

    template <class... Out>
    void run_steps(Out&... outputs)
    {
        const auto& d = particles.data();
        {
            std::ofstream out(output_file_, std::ofstream::app);
            out << "Init-Time(s): " << init_time_ << "\n"
                << "#Timestep/Total-steps Simulation-time Total-strain-energy Total-Damage "
                   "Cumulative-Time(s) Particle*steps/s\n";
        }
        const auto t_start = std::chrono::steady_clock::now();
        for (int step = 1; step <= num_steps; step++) {
            bool energy_done = false;
            if (!stage_) {
                // No device functor runs between stages: the steps up to the
                // next output step go to the library in one call (its fused
                // step where the model has one; bit-identical to the stages),
                // with the output step's energy when it ends on one.
                const int next_out = std::min(num_steps, (step / output_frequency + 1) *
                                                             output_frequency);
                const int last = step % output_frequency == 0 ? step : next_out;
                if (last % output_frequency == 0) {
                    cpdCheck(cpd_step_energy(d->sys, last - step + 1, &last_W_, &last_D_));
                    energy_done = true;
                } else {
                    cpdCheck(cpd_step(d->sys, last - step + 1));
                }
                step = last;
            } else {
                const double time = step * dt;
                cpdCheck(cpd_step_stage(d->sys, CPD_STAGE_INITIAL_HALF));
                if (!stage_->force_update) stage_->apply(time);
                cpdCheck(cpd_step_stage(d->sys, CPD_STAGE_FORCE));
                cpdCheck(cpd_step_stage(d->sys, CPD_STAGE_FORCE_BC));
                if (stage_->force_update) stage_->apply(time);
                cpdCheck(cpd_step_stage(d->sys, CPD_STAGE_FINAL_HALF));
            }
            if (step % output_frequency == 0) {
                const double time = step * dt;
                if (!energy_done) cpdCheck(cpd_compute_energy(d->sys, &last_W_, &last_D_));
                d->compute_stress();
                const bool write = detail::particle_output_enabled();
                if (sizeof...(Out) > 0 || d->with_stress || write) d->refresh_mirrors();
                // Solver.hpp:479-494: energy, stress, then the particle output.
                particles.output(step / output_frequency, time, output_reference_);
                if constexpr (sizeof...(Out) > 0) (outputs.update(time), ...);
                const double elapsed = seconds_since(t_start);
                std::ofstream out(output_file_, std::ofstream::app);
                out << step << "/" << num_steps << " " << std::scientific << std::setprecision(2)
                    << time << " " << last_W_ << " " << last_D_ << " " << std::fixed
                    << std::setprecision(4) << elapsed << " " << std::scientific
                    << std::setprecision(2)
                    << static_cast<double>(particles.numGlobal()) * step / std::max(elapsed, 1e-12)
                    << "\n";
            }
        }
        cpdCheck(cpd_synchronize(d->sys));
        const double total = seconds_since(t_start);
        {
            std::ofstream out(output_file_, std::ofstream::app);
            out << "\n#Steps/s Particle-steps/s\n"
                << std::scientific << std::setprecision(4) << num_steps / total << " "
                << static_cast<double>(particles.numGlobal()) * num_steps / total << "\n";
        }
        (outputs.print(), ...);
    }

    static int32_t precision_from_env()
    {
        const char* e = std::getenv("CABANAPD_B200_PRECISION");
        if (!e) return CPD_FP64;
        const std::string s(e);
        if (s == "exact") return CPD_FP64_EXACT;
        if (s == "mixed") return CPD_MIXED;
        if (s == "fp64") return CPD_FP64;
        throw std::runtime_error("CABANAPD_B200_PRECISION must be exact, fp64 or mixed");
    }
    static double seconds_since(std::chrono::steady_clock::time_point t0)
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    template <std::size_t N>
    void apply_prenotch(const Prenotch<N>& notch)
    {
        cpdCheck(cpd_prenotch(particles.data()->sys, static_cast<int32_t>(N), notch.v1.data(),
                              notch.v2.data(), notch.p0.data()));
    }

    Inputs inputs_;
    cpd_params params_{};
    std::string output_file_;
    double init_time_ = 0.0;
    double last_W_ = 0.0, last_D_ = 0.0;
    bool bc_bound_ = false;
    bool initialized_ = false;
    bool initial_output_ = true;
    bool output_reference_ = true;
    std::unique_ptr<detail::UserStage> stage_;
};

template <class P, class F>
Solver(Inputs, P, F) -> Solver<P, F>;
template <class P, class F, class C>
Solver(Inputs, P, F, C) -> Solver<P, F, C>;

}  // namespace CabanaPD
