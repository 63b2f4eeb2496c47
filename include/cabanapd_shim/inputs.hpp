// CabanaPD::Inputs: a JSON input deck ({"key": {"value": ..., "unit": ...}})
// with the keys the reference derives in its constructor
// (src/CabanaPD_Input.hpp:30-215) and the mechanics critical time step
// (src/CabanaPD_Input.hpp:217-301, 385-399).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "json.hpp"

namespace CabanaPD {

class Inputs {
    using Json = cabanapd_shim::Json;

  public:
    // One entry's "value", converting like the reference's json values do:
    // to double, int, bool, std::string or std::array<T, N>.
    class Value {
      public:
        explicit Value(const Json& j) : j_(j) {}
        operator double() const { return j_.number(); }
        operator int() const { return static_cast<int>(j_.number()); }
        operator bool() const { return j_.boolean(); }
        operator std::string() const { return j_.string(); }
        template <class T, std::size_t N>
        operator std::array<T, N>() const
        {
            if (!j_.is_array() || j_.size() != N)
                throw std::runtime_error("input value is not an array of the expected size");
            std::array<T, N> a{};
            for (std::size_t i = 0; i < N; i++) a[i] = static_cast<T>(j_[i].number());
            return a;
        }
        Value operator[](std::size_t i) const { return Value(j_[i]); }

      private:
        Json j_;
    };

    explicit Inputs(const std::string& filename)
    {
        in_ = Json::parse_file(filename);
        setupSize();
        const double tf = number("final_time");
        double dt = number("timestep");
        // Mass scaling, applied once (CabanaPD_Input.hpp:43-61).
        if (in_.contains("mass_scaling_factor") && !in_.contains("density_input")) {
            const double ms = number("mass_scaling_factor");
            const double rho0 = number("density");
            in_["density_input"]["value"] = Json(rho0);
            in_["density"]["value"] = Json(rho0 * ms);
            in_["timestep_input"]["value"] = Json(dt);
            dt *= std::sqrt(ms);
            in_["timestep"]["value"] = Json(dt);
        }
        if (in_.contains("horizon") && in_.contains("m"))
            throw std::runtime_error("Cannot input both horizon and m.");
        const double dx = in_.at("dx").at("value")[0].number();
        if (in_.contains("horizon")) {
            const double horizon = number("horizon");
            const int m = static_cast<int>(std::floor(horizon / dx));
            if (horizon < dx)
                throw std::runtime_error(
                    "Input horizon must be greater than or equal to dx to result in any "
                    "neighbour-particles");
            in_["m"]["value"] = Json(static_cast<double>(m));
        } else if (in_.contains("m")) {
            const int m = static_cast<int>(number("m"));
            if (m < 1) throw std::runtime_error("Input m must be greater than or equal to 1.");
            in_["horizon"]["value"] = Json(static_cast<double>(m) * dx + 0.01 * dx);
        }
        if (!in_.contains("timestep_safety_factor"))
            in_["timestep_safety_factor"]["value"] = Json(0.85);
        if (!in_.contains("bulk_modulus") && !in_.contains("elastic_modulus"))
            throw std::runtime_error("Must input either bulk_modulus or elastic_modulus.");
        // C++ int conversion truncates toward zero.
        in_["num_steps"]["value"] = Json(static_cast<double>(static_cast<int>(tf / dt)));
        if (!in_.contains("output_file"))
            in_["output_file"]["value"] = Json(std::string("cabanaPD.out"));
        if (!in_.contains("error_file"))
            in_["error_file"]["value"] = Json(std::string("cabanaPD.err"));
        in_["input_file"]["value"] = Json(filename);
        if (!in_.contains("output_reference")) in_["output_reference"]["value"] = Json(true);
        std::ofstream("cabanaPD.in.json") << in_.dump();
    }

    Value operator[](const std::string& key) const { return Value(in_.at(key).at("value")); }
    bool contains(const std::string& key) const { return in_.contains(key); }
    std::vector<double> getVector(const std::string& key) const
    {
        const Json& v = in_.at(key).at("value");
        std::vector<double> out;
        if (v.is_array())
            for (std::size_t i = 0; i < v.size(); i++) out.push_back(v[i].number());
        else
            out.push_back(v.number());
        return out;
    }

    // Silling & Askari stable step summed over the lattice neighbourhood of a
    // bulk point, with K from bulk_modulus (or E / (3 (1 - 2 * 0.25))) and
    // the smallest rho / K over materials. Warns when the input step is
    // larger than safety * dt_crit, stores that product as
    // critical_timestep_mechanics and returns dt_crit.
    double computeCriticalTimeStep()
    {
        const double dx = in_.at("dx").at("value")[0].number();
        const double dy = in_.at("dx").at("value")[1].number();
        const double dz = in_.at("dx").at("value")[2].number();
        const double v_p = dx * dy * dz;
        std::vector<double> K;
        if (in_.contains("bulk_modulus")) {
            K = getVector("bulk_modulus");
        } else {
            const double denom = 3.0 * (1.0 - 2.0 * 0.25);
            for (double e : getVector("elastic_modulus")) K.push_back(e / denom);
        }
        const std::vector<double> rho = getVector("density");
        std::size_t imin = 0;
        for (std::size_t i = 1; i < rho.size() && i < K.size(); i++)
            if (rho[i] / K[i] < rho[imin] / K[imin]) imin = i;
        const int m = static_cast<int>(number("m"));
        const double horizon = number("horizon");
        const double c = 18.0 * K[imin] / (3.14159265358979323846 * horizon * horizon * horizon * horizon);
        double sum = 0.0;
        for (int i = -(m + 1); i < m + 2; i++) {
            const double xi_1 = i * dx;
            for (int j = -(m + 1); j < m + 2; j++) {
                const double xi_2 = j * dy;
                for (int k = -(m + 1); k < m + 2; k++) {
                    const double xi_3 = k * dz;
                    const double r2 = xi_1 * xi_1 + xi_2 * xi_2 + xi_3 * xi_3;
                    if (r2 < horizon * horizon + 1e-10 && r2 > 0) sum += v_p * c / std::sqrt(r2);
                }
            }
        }
        const double dt_crit = std::sqrt(2.0 * rho[imin] / sum);
        const double safety = number("timestep_safety_factor");
        const double dt = number("timestep");
        if (dt > safety * dt_crit)
            std::cout << "WARNING: timestep (" << dt
                      << ") is larger than estimated stable timestep for mechanics ("
                      << safety * dt_crit << "), using safety factor of " << safety << ".\n";
        in_["critical_timestep_mechanics"]["value"] = Json(safety * dt_crit);
        return dt_crit;
    }

  private:
    double number(const std::string& key) const { return in_.at(key).at("value").number(); }

    // CabanaPD_Input.hpp:130-215.
    void setupSize()
    {
        if (in_.contains("system_size")) {
            const Json s = in_.at("system_size").at("value");
            if (s.size() != 3) throw std::runtime_error("CabanaPD requires 3d (system_size).");
            for (std::size_t d = 0; d < 3; d++) {
                in_["low_corner"]["value"].at_index(d) = Json(-0.5 * s[d].number());
                in_["high_corner"]["value"].at_index(d) = Json(0.5 * s[d].number());
            }
        } else if (in_.contains("low_corner") && in_.contains("high_corner")) {
            const Json lo = in_.at("low_corner").at("value");
            const Json hi = in_.at("high_corner").at("value");
            if (lo.size() != 3 || hi.size() != 3)
                throw std::runtime_error("CabanaPD requires 3d (low_corner/high_corner).");
            for (std::size_t d = 0; d < 3; d++)
                in_["system_size"]["value"].at_index(d) = Json(hi[d].number() - lo[d].number());
        } else {
            throw std::runtime_error(
                "Must input either system_size or both low_corner and high_corner.");
        }
        const Json s = in_.at("system_size").at("value");
        if (in_.contains("dx")) {
            const Json dx = in_.at("dx").at("value");
            if (dx.size() != 3) throw std::runtime_error("CabanaPD requires 3d (dx).");
            for (std::size_t d = 0; d < 3; d++)
                in_["num_cells"]["value"].at_index(d) =
                    Json(static_cast<double>(static_cast<int>(s[d].number() / dx[d].number())));
        } else if (in_.contains("num_cells")) {
            const Json nc = in_.at("num_cells").at("value");
            if (nc.size() != 3) throw std::runtime_error("CabanaPD requires 3d (num_cells).");
            for (std::size_t d = 0; d < 3; d++)
                in_["dx"]["value"].at_index(d) =
                    Json(s[d].number() / static_cast<double>(static_cast<int>(nc[d].number())));
        } else {
            throw std::runtime_error("Must input either num_cells or dx.");
        }
    }

    Json in_;
};

}  // namespace CabanaPD
