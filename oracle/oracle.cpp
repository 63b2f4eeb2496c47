// CPU oracle for the CabanaPD per-timestep hot path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path and the
// timed CPU baseline. The product never links this file. See oracle.h.
//
// Every kernel below restates one reference function; the citation on each
// names the reference file:line (paths relative to the CabanaPD source tree).
// Expressions keep the reference's operand order so that, compiled with
// -ffp-contract=off, each per-bond value rounds exactly as the reference's
// scalar code does.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

int fail(const std::string& msg)
{
    g_err = msg;
    return 1;
}

// CabanaPD_Constants.hpp: pi = Kokkos::numbers::pi_v<double>.
constexpr double kPi = 3.14159265358979323846;

struct Model {
    int pd = ORC_PD_NONE;
    int fracture = 0;
    int influence = 1;
    int contact = ORC_CONTACT_NONE;
    double horizon = 0, K = 0, G = 0, G0 = 0;
    // force_models/CabanaPD_PMB.hpp:41-47
    double c = 0;
    // force_models/CabanaPD_LPS.hpp:64-75 (single-material coefficients)
    double theta_coeff = 0, s_coeff = 0;
    // CabanaPD_ForceModels.hpp:93-102
    double s0 = 0, bond_break_coeff = 0;
    // force_models/CabanaPD_Contact.hpp:40-48, CabanaPD_Hertzian.hpp:40-56
    double radius = 0, radius_extend = 0, nu = 0, E = 0, e = 0;
    double Rs = 0, Es = 0, beta = 0, coeff_h_n = 0, coeff_h_d = 0;
    int per_particle_radius = 0;
    // force_models/CabanaPD_Contact.hpp:70-79 (normal repulsion)
    double contact_horizon = 0, c_contact = 0;
};

// Full neighbour list: rows for i in [begin, n), padded to max_n columns,
// each row sorted by ascending neighbour index (the oracle's fixed order;
// Cabana's own in-row order is not part of the reference's contract).
struct NList {
    int32_t max_n = 0;
    int64_t total = 0;
    std::vector<int32_t> count;
    std::vector<int32_t> idx;
};

struct BC {
    int kind;
    int component;
    std::vector<int64_t> idx;
    std::vector<double> values;
};

}  // namespace

struct orc_system {
    Model model;
    int64_t n = 0, frozen = 0;
    std::vector<double> x, u, v, f, vol, rho, m, theta, W, phi, radius, u_neigh;
    std::vector<double> stress;  // [n][3][3]
    std::vector<int32_t> nofail;
    NList pd_list;
    std::vector<int32_t> mu;  // [n][pd_list.max_n], 1 = intact
    NList contact_list;
    bool have_contact_list = false;
    double dt = 0;
    double max_displacement = 0;
    int32_t rebuild_every = 0;
    int64_t steps_since_rebuild = 0;
    int64_t rebuilds = 0;
    std::vector<BC> bcs;
    bool ready = false;
};

namespace {

// ---------------------------------------------------------------------------
// CabanaPD_Force.hpp:74-93 getDistance.
inline void get_distance(const double* x, const double* u, int64_t i,
                         int64_t j, double& xi, double& r, double& s,
                         double& rx, double& ry, double& rz, double& xi_x,
                         double& xi_y, double& xi_z)
{
    xi_x = x[3 * j + 0] - x[3 * i + 0];
    const double eta_u = u[3 * j + 0] - u[3 * i + 0];
    xi_y = x[3 * j + 1] - x[3 * i + 1];
    const double eta_v = u[3 * j + 1] - u[3 * i + 1];
    xi_z = x[3 * j + 2] - x[3 * i + 2];
    const double eta_w = u[3 * j + 2] - u[3 * i + 2];
    rx = xi_x + eta_u;
    ry = xi_y + eta_v;
    rz = xi_z + eta_w;
    r = std::sqrt(rx * rx + ry * ry + rz * rz);
    xi = std::sqrt(xi_x * xi_x + xi_y * xi_y + xi_z * xi_z);
    s = (r - xi) / xi;
}

// CabanaPD_Force.hpp:114-129 getLinearizedDistance.
inline void get_linearized_distance(const double* x, const double* u,
                                    int64_t i, int64_t j, double& xi,
                                    double& s, double& xi_x, double& xi_y,
                                    double& xi_z)
{
    xi_x = x[3 * j + 0] - x[3 * i + 0];
    const double eta_u = u[3 * j + 0] - u[3 * i + 0];
    xi_y = x[3 * j + 1] - x[3 * i + 1];
    const double eta_v = u[3 * j + 1] - u[3 * i + 1];
    xi_z = x[3 * j + 2] - x[3 * i + 2];
    const double eta_w = u[3 * j + 2] - u[3 * i + 2];
    xi = std::sqrt(xi_x * xi_x + xi_y * xi_y + xi_z * xi_z);
    s = (xi_x * eta_u + xi_y * eta_v + xi_z * eta_w) / (xi * xi);
}

// force_models/CabanaPD_LPS.hpp:85-98 influence function.
inline double influence(const Model& md, double xi)
{
    if (md.influence == 1) return 1.0 / xi;
    return 1.0;
}

// force_models/CabanaPD_LPS.hpp:118-134 ForceCoeffTag (single material:
// theta_coeff[0] == theta_coeff[1], s_coeff[0] == s_coeff[1]).
inline double lps_force_coeff(const Model& md, double s, double xi,
                              double vol_j, double m_i, double m_j,
                              double theta_i, double theta_j)
{
    const double infl = influence(md, xi);
    return (md.theta_coeff * theta_i / m_i + md.theta_coeff * theta_j / m_j +
            s * (md.s_coeff / m_i + md.s_coeff / m_j)) *
           infl * xi * vol_j;
}

// force_models/CabanaPD_LPS.hpp:136-148 EnergyTag.
inline double lps_energy(const Model& md, double s, double xi, double vol_j,
                         double m_i, double theta_i, double num_bonds)
{
    const double infl = influence(md, xi);
    return 1.0 / num_bonds * 0.5 * md.theta_coeff / 3.0 * (theta_i * theta_i) +
           0.5 * (md.s_coeff / m_i) * infl * s * s * xi * xi * vol_j;
}

// ---------------------------------------------------------------------------
// Linked-cell full neighbour list. Restates what Neighbor's constructor gets
// from Cabana::VerletList<FullNeighborTag> (CabanaPD_Neighbor.hpp:44-66):
// every particle in [0, n) is a candidate, rows exist for [begin, n), and a
// pair is listed when its squared distance is <= cutoff^2.
void build_list(const std::vector<double>& pos, int64_t n, int64_t begin,
                double cutoff, NList& nl)
{
    nl.count.assign(n, 0);
    nl.idx.clear();
    nl.max_n = 0;
    nl.total = 0;
    if (n == 0) return;
    double lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = pos[d];
        hi[d] = pos[d];
    }
    for (int64_t p = 0; p < n; p++)
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], pos[3 * p + d]);
            hi[d] = std::max(hi[d], pos[3 * p + d]);
        }
    // Cells are at least the cutoff wide (so the 27-cell stencil is
    // complete) and grow when a tiny cutoff would make the grid much larger
    // than the particle count.
    int64_t nc[3];
    double cell = cutoff;
    for (;;) {
        for (int d = 0; d < 3; d++) {
            double span = (hi[d] - lo[d]) / cell;
            nc[d] = std::max<int64_t>(1, std::min<int64_t>((int64_t)span + 1, 1 << 20));
        }
        if ((double)nc[0] * (double)nc[1] * (double)nc[2] <= 4.0 * (double)n + 4096.0) break;
        cell *= 2.0;
    }
    auto cell_of = [&](int64_t p, int64_t c[3]) {
        for (int d = 0; d < 3; d++) {
            int64_t k = (int64_t)std::floor((pos[3 * p + d] - lo[d]) / cell);
            c[d] = std::min<int64_t>(std::max<int64_t>(k, 0), nc[d] - 1);
        }
    };
    const int64_t ncell = nc[0] * nc[1] * nc[2];
    std::vector<int64_t> start(ncell + 1, 0);
    std::vector<int64_t> cid(n);
    for (int64_t p = 0; p < n; p++) {
        int64_t c[3];
        cell_of(p, c);
        cid[p] = c[0] + nc[0] * (c[1] + nc[1] * c[2]);
        start[cid[p] + 1]++;
    }
    for (int64_t c = 0; c < ncell; c++) start[c + 1] += start[c];
    std::vector<int64_t> fillp(start.begin(), start.end() - 1);
    std::vector<int64_t> order(n);
    for (int64_t p = 0; p < n; p++) order[fillp[cid[p]]++] = p;

    const double rsqr = cutoff * cutoff;
    auto visit = [&](int64_t i, auto&& emit) {
        int64_t c[3];
        cell_of(i, c);
        for (int64_t dz = -1; dz <= 1; dz++)
            for (int64_t dy = -1; dy <= 1; dy++)
                for (int64_t dx = -1; dx <= 1; dx++) {
                    int64_t a = c[0] + dx, b = c[1] + dy, cc = c[2] + dz;
                    if (a < 0 || b < 0 || cc < 0 || a >= nc[0] || b >= nc[1] ||
                        cc >= nc[2])
                        continue;
                    int64_t cell = a + nc[0] * (b + nc[1] * cc);
                    for (int64_t q = start[cell]; q < start[cell + 1]; q++) {
                        int64_t j = order[q];
                        if (j == i) continue;
                        double ddx = pos[3 * j + 0] - pos[3 * i + 0];
                        double ddy = pos[3 * j + 1] - pos[3 * i + 1];
                        double ddz = pos[3 * j + 2] - pos[3 * i + 2];
                        double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                        if (d2 <= rsqr) emit(j);
                    }
                }
    };
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = begin; i < n; i++) {
        int32_t cnt = 0;
        visit(i, [&](int64_t) { cnt++; });
        nl.count[i] = cnt;
    }
    int32_t mx = 0;
    int64_t tot = 0;
    for (int64_t i = 0; i < n; i++) {
        mx = std::max(mx, nl.count[i]);
        tot += nl.count[i];
    }
    nl.max_n = mx;
    nl.total = tot;
    nl.idx.assign((size_t)n * (size_t)std::max(mx, 1), -1);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = begin; i < n; i++) {
        int32_t* row = &nl.idx[(size_t)i * mx];
        int32_t k = 0;
        visit(i, [&](int64_t j) { row[k++] = (int32_t)j; });
        std::sort(row, row + k);
    }
}

// ---------------------------------------------------------------------------
// PD kernels. Each loops i over [frozen, n) (Neighbor::makePolicy,
// CabanaPD_Neighbor.hpp:182-187) and walks row i in ascending-j order.

// force/CabanaPD_LPS.hpp:89-112 (NoFracture) and :287-329 (Fracture).
void lps_weighted_volume(orc_system& s)
{
    const Model& md = s.model;
    const NList& nl = s.pd_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    std::fill(s.m.begin(), s.m.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        double mi = 0.0;
        for (int32_t nn = 0; nn < nl.count[i]; nn++) {
            int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            double xi, r, st, rx, ry, rz, xx, xy, xz;
            get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
            // force_models/CabanaPD_LPS.hpp:100-106 WeightedVolumeTag
            double wv = influence(md, xi) * xi * xi * s.vol[j];
            if (md.fracture)
                mi += s.mu[(size_t)i * nl.max_n + nn] * wv;
            else
                mi += wv;
        }
        s.m[i] = mi;
    }
}

// force/CabanaPD_LPS.hpp:114-141 (NoFracture) and :331-378 (Fracture).
void lps_dilatation(orc_system& s)
{
    const Model& md = s.model;
    const NList& nl = s.pd_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    std::fill(s.theta.begin(), s.theta.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        double th = 0.0;
        const double m_i = s.m[i];
        for (int32_t nn = 0; nn < nl.count[i]; nn++) {
            int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            double xi, r, st, rx, ry, rz, xx, xy, xz;
            get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
            // force_models/CabanaPD_LPS.hpp:108-116 DilatationTag
            double theta_i = influence(md, xi) * st * xi * xi * s.vol[j];
            double term = 3.0 * theta_i / m_i;
            if (md.fracture) {
                if (m_i > 0) th += s.mu[(size_t)i * nl.max_n + nn] * term;
            } else {
                th += term;
            }
        }
        s.theta[i] = th;
    }
}

// force/CabanaPD_PMB.hpp:89-125 (NoFracture), :222-287 (Fracture),
// :406-455 (LinearPMB); force/CabanaPD_LPS.hpp:143-181 (NoFracture),
// :380-447 (Fracture). f is zeroed first (CabanaPD_Force.hpp:187-189).
// LinearLPS systems reach here as LPS (see orc_create).
void pd_force(orc_system& s)
{
    const Model& md = s.model;
    const NList& nl = s.pd_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    const bool linear = md.pd == ORC_PD_LINEAR_PMB;
    const bool lps = md.pd == ORC_PD_LPS;
    std::fill(s.f.begin(), s.f.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int32_t nn = 0; nn < nl.count[i]; nn++) {
            int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            if (linear) {
                double xi, ls, xx, xy, xz;
                get_linearized_distance(x, u, i, j, xi, ls, xx, xy, xz);
                const double coeff = md.c * ls * s.vol[j];
                fx += coeff * xx / xi;
                fy += coeff * xy / xi;
                fz += coeff * xz / xi;
                continue;
            }
            double xi, r, st, rx, ry, rz, xx, xy, xz;
            get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
            if (md.fracture) {
                int32_t& mu = s.mu[(size_t)i * nl.max_n + nn];
                // CabanaPD_ForceModels.hpp:123-128 CriticalStretchTag.
                // LPS tests nofail(i) twice (force/CabanaPD_LPS.hpp:417-418);
                // PMB tests nofail(i) and nofail(j) (force/CabanaPD_PMB.hpp:260-261).
                bool critical = r * r >= md.bond_break_coeff * xi * xi;
                bool nofail_other = lps ? (s.nofail[i] != 0) : (s.nofail[j] != 0);
                if (critical && !s.nofail[i] && !nofail_other) {
                    mu = 0;
                } else if (mu > 0) {
                    double coeff;
                    if (lps)
                        coeff = lps_force_coeff(md, st, xi, s.vol[j], s.m[i],
                                                s.m[j], s.theta[i], s.theta[j]);
                    else
                        coeff = md.c * st * s.vol[j];
                    double muij = mu;
                    fx += muij * coeff * rx / r;
                    fy += muij * coeff * ry / r;
                    fz += muij * coeff * rz / r;
                }
            } else {
                double coeff;
                if (lps)
                    coeff = lps_force_coeff(md, st, xi, s.vol[j], s.m[i], s.m[j],
                                            s.theta[i], s.theta[j]);
                else
                    coeff = md.c * st * s.vol[j];
                fx += coeff * rx / r;
                fy += coeff * ry / r;
                fz += coeff * rz / r;
            }
        }
        s.f[3 * i + 0] = fx;
        s.f[3 * i + 1] = fy;
        s.f[3 * i + 2] = fz;
    }
}

// force/CabanaPD_PMB.hpp:127-155, :289-339, :458-491;
// force/CabanaPD_LPS.hpp:183-219, :449-504.
// W is reset first (CabanaPD_Force.hpp:213-214). Per-particle W_i and phi_i
// are exact restatements; the totals are summed serially over i.
void pd_energy(orc_system& s, double& total_W, double& total_D)
{
    const Model& md = s.model;
    const NList& nl = s.pd_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    const bool linear = md.pd == ORC_PD_LINEAR_PMB;
    const bool lps = md.pd == ORC_PD_LPS;
    std::fill(s.W.begin(), s.W.end(), 0.0);
    std::vector<double> phi_contrib(s.n, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        const int32_t cnt = nl.count[i];
        double Wi = 0.0;
        double Phi_i = 0.0;  // sum of w * vol(i) (NoFracture accumulation order)
        double num_bonds = static_cast<double>(cnt);
        if (md.fracture && lps) {
            num_bonds = 0.0;
            for (int32_t nn = 0; nn < cnt; nn++)
                num_bonds += static_cast<double>(s.mu[(size_t)i * nl.max_n + nn]);
        }
        double phi_i = 0.0, vol_H_i = 0.0;
        for (int32_t nn = 0; nn < cnt; nn++) {
            int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            double w;
            if (linear) {
                double xi, ls, xx, xy, xz;
                get_linearized_distance(x, u, i, j, xi, ls, xx, xy, xz);
                w = 0.25 * md.c * ls * ls * xi * s.vol[j];
            } else {
                double xi, r, st, rx, ry, rz, xx, xy, xz;
                get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
                if (lps)
                    w = lps_energy(md, st, xi, s.vol[j], s.m[i], s.theta[i],
                                   num_bonds);
                else
                    // force_models/CabanaPD_PMB.hpp:64-71 EnergyTag
                    w = 0.25 * md.c * st * st * xi * s.vol[j];
            }
            if (md.fracture) {
                int32_t mu = s.mu[(size_t)i * nl.max_n + nn];
                w = mu * w;
                Wi += w;
                phi_i += mu * s.vol[j];
                vol_H_i += s.vol[j];
            } else {
                Wi += w;
                Phi_i += w * s.vol[i];
            }
        }
        s.W[i] = Wi;
        if (md.fracture) {
            s.phi[i] = 1 - phi_i / vol_H_i;
            phi_contrib[i] = Wi * s.vol[i];
        } else {
            phi_contrib[i] = Phi_i;
        }
    }
    double Phi = 0.0, D = 0.0;
    for (int64_t i = s.frozen; i < s.n; i++) {
        Phi += phi_contrib[i];
        if (md.fracture) D += s.phi[i];
    }
    total_W = Phi;
    total_D = D;
}

// force/CabanaPD_PMB.hpp:157-202 (NoFracture), :341-401 (Fracture),
// :492-537 (LinearPMB); force/CabanaPD_LPS.hpp:221-267 (NoFracture),
// :506-572 (Fracture: intact bonds only). Half the pair force times the
// reference bond vector, stress(i, a, b) += f_a xi_b, accumulated over the
// row in row order after the tensor is zeroed (CabanaPD_Force.hpp:222-235).
void pd_stress(orc_system& s)
{
    const Model& md = s.model;
    const NList& nl = s.pd_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    const bool linear = md.pd == ORC_PD_LINEAR_PMB;
    const bool lps = md.pd == ORC_PD_LPS;
    std::fill(s.stress.begin(), s.stress.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        double* S = &s.stress[9 * (size_t)i];
        for (int32_t nn = 0; nn < nl.count[i]; nn++) {
            const int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            double fx, fy, fz, xx, xy, xz;
            if (linear) {
                double xi, ls;
                get_linearized_distance(x, u, i, j, xi, ls, xx, xy, xz);
                const double coeff = 0.5 * (md.c * ls * s.vol[j]);
                fx = coeff * xx / xi;
                fy = coeff * xy / xi;
                fz = coeff * xz / xi;
            } else {
                double xi, r, st, rx, ry, rz;
                get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
                const int32_t mu = md.fracture ? s.mu[(size_t)i * nl.max_n + nn] : 1;
                if (md.fracture && lps && !(mu > 0)) continue;
                double coeff;
                if (lps) {
                    coeff = lps_force_coeff(md, st, xi, s.vol[j], s.m[i], s.m[j], s.theta[i],
                                            s.theta[j]);
                    coeff *= 0.5;
                } else {
                    coeff = 0.5 * (md.c * st * s.vol[j]);
                }
                if (md.fracture) {
                    const double muij = mu;
                    fx = muij * coeff * rx / r;
                    fy = muij * coeff * ry / r;
                    fz = muij * coeff * rz / r;
                } else {
                    fx = coeff * rx / r;
                    fy = coeff * ry / r;
                    fz = coeff * rz / r;
                }
            }
            S[0] += fx * xx;
            S[4] += fy * xy;
            S[8] += fz * xz;
            S[1] += fx * xy;
            S[3] += fy * xx;
            S[2] += fx * xz;
            S[6] += fz * xx;
            S[5] += fy * xz;
            S[7] += fz * xy;
        }
    }
}

// ---------------------------------------------------------------------------
// Hertzian contact: force/CabanaPD_Contact.hpp:119-168 with the model of
// force_models/CabanaPD_Hertzian.hpp:58-87. With per_particle_radius the
// model is generalised to R* = R_i (R_j / (R_i + R_j)), overlap
// r - (R_i + R_j), m* = m_i (m_j / (m_i + m_j)); for R_i == R_j every one of
// these rounds to the reference's single-radius value.
void hertz_force(orc_system& s, bool reset)
{
    const Model& md = s.model;
    const NList& nl = s.contact_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    const double* v = s.v.data();
    if (reset) std::fill(s.f.begin(), s.f.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        double fx = s.f[3 * i + 0], fy = s.f[3 * i + 1], fz = s.f[3 * i + 2];
        for (int32_t nn = 0; nn < nl.count[i]; nn++) {
            int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            double xi, r, st, rx, ry, rz, xx, xy, xz;
            get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
            double nx = rx / r, ny = ry / r, nz = rz / r;
            double vx = v[3 * j + 0] - v[3 * i + 0];
            double vy = v[3 * j + 1] - v[3 * i + 1];
            double vz = v[3 * j + 2] - v[3 * i + 2];
            double vn = vx * nx + vy * ny + vz * nz;
            // normalForce(r, vn, vol(i), rho(i))
            double sum_r, Rs, coeff_h_n, ms;
            const double vol_i = s.vol[i];
            const double rho_i = s.rho[i];
            if (md.per_particle_radius) {
                double Ri = s.radius[i], Rj = s.radius[j];
                sum_r = Ri + Rj;
                Rs = Ri * (Rj / (Ri + Rj));
                coeff_h_n = 4.0 / 3.0 * md.Es * std::sqrt(Rs);
                double mi = rho_i * vol_i;
                double mj = s.rho[j] * s.vol[j];
                ms = mi * (mj / (mi + mj));
            } else {
                sum_r = 2.0 * md.radius;
                Rs = md.Rs;
                coeff_h_n = md.coeff_h_n;
                ms = (rho_i * vol_i) / 2.0;
            }
            const double delta_n = (r - sum_r);
            double coeff = 0.0;
            if (delta_n < 0.0)
                coeff = std::min(0.0, -coeff_h_n * std::pow(std::fabs(delta_n), 3.0 / 2.0));
            coeff /= vol_i;
            double Sn = 0.0;
            if (delta_n < 0.0) Sn = 2.0 * md.Es * std::sqrt(Rs * std::fabs(delta_n));
            coeff -= md.coeff_h_d * std::sqrt(Sn * ms) * vn / vol_i;
            const double fn = coeff;
            fx += fn * nx;
            fy += fn * ny;
            fz += fn * nz;
            // tangentialForce is a no-op (CabanaPD_Hertzian.hpp:83-87); the
            // reference then adds ft = 0.0 to each component.
            fx += 0.0;
            fy += 0.0;
            fz += 0.0;
        }
        s.f[3 * i + 0] = fx;
        s.f[3 * i + 1] = fy;
        s.f[3 * i + 2] = fz;
    }
}

// Normal repulsion: force/CabanaPD_Contact.hpp:52-92 computeForceFull with
// NormalRepulsionModel::forceCoeff (force_models/CabanaPD_Contact.hpp:82-88).
void repulsion_force(orc_system& s, bool reset)
{
    const Model& md = s.model;
    const NList& nl = s.contact_list;
    const double* x = s.x.data();
    const double* u = s.u.data();
    if (reset) std::fill(s.f.begin(), s.f.end(), 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        double fx = s.f[3 * i + 0], fy = s.f[3 * i + 1], fz = s.f[3 * i + 2];
        for (int32_t nn = 0; nn < nl.count[i]; nn++) {
            int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
            double fcx = 0.0, fcy = 0.0, fcz = 0.0;
            double xi, r, st, rx, ry, rz, xx, xy, xz;
            get_distance(x, u, i, j, xi, r, st, rx, ry, rz, xx, xy, xz);
            if (r < md.radius) {
                const double sc = (r - md.radius) / md.contact_horizon;
                const double coeff = 15.0 * md.c_contact * sc * s.vol[j];
                fcx = coeff * rx / r;
                fcy = coeff * ry / r;
                fcz = coeff * rz / r;
            }
            fx += fcx;
            fy += fcy;
            fz += fcz;
        }
        s.f[3 * i + 0] = fx;
        s.f[3 * i + 1] = fy;
        s.f[3 * i + 2] = fz;
    }
}

void contact_force(orc_system& s, bool reset)
{
    if (s.model.contact == ORC_CONTACT_NORMAL_REPULSION)
        repulsion_force(s, reset);
    else
        hertz_force(s, reset);
}

void build_contact_list(orc_system& s, double cutoff)
{
    // CabanaPD_Particles.hpp:534-553 current positions y = x + u.
    std::vector<double> y(3 * s.n);
    for (int64_t p = 0; p < 3 * s.n; p++) y[p] = s.x[p] + s.u[p];
    build_list(y, s.n, s.frozen, cutoff, s.contact_list);
    s.have_contact_list = true;
    // CabanaPD_Neighbor.hpp:127-130 reset the rebuild displacement.
    s.u_neigh = s.u;
    s.rebuilds++;
    s.steps_since_rebuild = 0;
}

// CabanaPD_Neighbor.hpp:107-132 Neighbor::update (contact list rebuild on
// displacement), or the fixed-interval variant when rebuild_every > 0.
void contact_update(orc_system& s)
{
    const Model& md = s.model;
    bool rebuild;
    if (s.rebuild_every > 0)
        rebuild = s.steps_since_rebuild >= s.rebuild_every;
    else
        rebuild = s.max_displacement > md.radius_extend;
    if (rebuild) build_contact_list(s, 2.0 * md.radius + md.radius_extend);
}

// ---------------------------------------------------------------------------
// CabanaPD_Integrate.hpp:89-116 (NoContact) and :151-193 (Contact).
void vv_initial(orc_system& s)
{
    const double dt = s.dt, half_dt = 0.5 * s.dt;
    const bool contact = s.model.contact != ORC_CONTACT_NONE;
    double maxu = 0.0;
#pragma omp parallel for schedule(static) reduction(max : maxu)
    for (int64_t i = s.frozen; i < s.n; i++) {
        const double half_dt_m = half_dt / s.rho[i];
        for (int d = 0; d < 3; d++) s.v[3 * i + d] += half_dt_m * s.f[3 * i + d];
        for (int d = 0; d < 3; d++) s.u[3 * i + d] += dt * s.v[3 * i + d];
        if (contact) {
            double um = std::hypot(s.u[3 * i + 0] - s.u_neigh[3 * i + 0],
                                   s.u[3 * i + 1] - s.u_neigh[3 * i + 1],
                                   s.u[3 * i + 2] - s.u_neigh[3 * i + 2]);
            if (um > maxu) maxu = um;
        }
    }
    if (contact) s.max_displacement = maxu;
    s.steps_since_rebuild++;
}

// CabanaPD_Integrate.hpp:119-141.
void vv_final(orc_system& s)
{
    const double half_dt = 0.5 * s.dt;
#pragma omp parallel for schedule(static)
    for (int64_t i = s.frozen; i < s.n; i++) {
        const double half_dt_m = half_dt / s.rho[i];
        for (int d = 0; d < 3; d++) s.v[3 * i + d] += half_dt_m * s.f[3 * i + d];
    }
}

// CabanaPD_Boundary.hpp:94-113 (ForceValueBCTag), :138-157
// (ForceUpdateBCTag), and the custom-functor form :52-69 used as
// f(pid, component) += value (random_cracks.cpp:173-178, BodyTerm gravity).
void apply_force_bcs(orc_system& s)
{
    for (const BC& bc : s.bcs) {
        for (size_t b = 0; b < bc.idx.size(); b++) {
            int64_t p = bc.idx[b];
            if (bc.kind == ORC_BC_FORCE_VALUE)
                for (int d = 0; d < 3; d++) s.f[3 * p + d] = bc.values[0];
            else if (bc.kind == ORC_BC_FORCE_UPDATE)
                for (int d = 0; d < 3; d++) s.f[3 * p + d] += bc.values[0];
            else
                s.f[3 * p + bc.component] += bc.values[b];
        }
    }
}

bool has_pd(const orc_system& s) { return s.model.pd != ORC_PD_NONE; }
bool is_lps(const orc_system& s)
{
    return s.model.pd == ORC_PD_LPS;
}

// CabanaPD_Solver.hpp:462-477 updateForce, plus the contact force
// (Solver.hpp:361-363, reset=false) or the DEM-only force (reset=true).
void update_force(orc_system& s)
{
    if (has_pd(s)) {
        if (is_lps(s)) {
            if (s.model.fracture) lps_weighted_volume(s);
            lps_dilatation(s);
        }
        pd_force(s);
    }
    if (s.model.contact != ORC_CONTACT_NONE) {
        contact_update(s);
        contact_force(s, !has_pd(s));
    }
}

// ---------------------------------------------------------------------------
// Pre-notch geometry: CabanaPD_Prenotch.hpp:24-172.
struct V3 {
    double a[3];
};
inline double dot3(V3 a, V3 b)
{
    double v = 0;
    for (int d = 0; d < 3; d++) v += (a.a[d]) * (b.a[d]);
    return v;
}
inline double norm3(V3 a) { return std::sqrt(dot3(a, a)); }
inline V3 cross3(V3 a, V3 b)
{
    V3 c;
    c.a[0] = a.a[1] * b.a[2] - a.a[2] * b.a[1];
    c.a[1] = -(a.a[0] * b.a[2] - a.a[2] * b.a[0]);
    c.a[2] = a.a[0] * b.a[1] - a.a[1] * b.a[0];
    return c;
}
inline V3 scale3(V3 a, double nn)
{
    for (int d = 0; d < 3; d++) a.a[d] *= nn;
    return a;
}
inline V3 diff3(V3 a, V3 b)
{
    V3 c;
    for (int d = 0; d < 3; d++) c.a[d] = a.a[d] - b.a[d];
    return c;
}
inline V3 sum3(V3 a, V3 b)
{
    V3 c;
    for (int d = 0; d < 3; d++) c.a[d] = a.a[d] + b.a[d];
    return c;
}
inline int line_plane(V3 p0, V3 n, V3 l0, V3 l, double tol = 1e-10)
{
    if (std::fabs(dot3(l, n)) < tol) {
        if (std::fabs(dot3(diff3(p0, l0), n)) < tol) return 1;
        return 2;
    }
    return 3;
}
int bond_prenotch_intersection(V3 v1, V3 v2, V3 p0, V3 x_i, V3 x_j,
                               double tol = 1e-10)
{
    V3 cv = cross3(v1, v2);
    double ncv = norm3(cv);
    V3 n = scale3(cv, 1.0 / ncv);
    V3 l0 = x_i;
    V3 l = diff3(x_j, x_i);
    int flag = line_plane(p0, n, l0, l);
    int keep = 1;
    if (flag == 1) {
        double n2 = ncv * ncv;
        double li1 = dot3(cross3(diff3(x_i, p0), v2), cv) / n2;
        double li2 = -dot3(cross3(diff3(x_i, p0), v1), cv) / n2;
        double lj1 = dot3(cross3(diff3(x_j, p0), v2), cv) / n2;
        double lj2 = -dot3(cross3(diff3(x_j, p0), v1), cv) / n2;
        if (!(std::fmin(li1, lj1) > 1 + tol || std::fmax(li1, lj1) < -tol ||
              std::fmin(li2, lj2) > 1 + tol || std::fmax(li2, lj2) < -tol))
            keep = 0;
    } else if (flag == 3) {
        double dd = dot3(diff3(p0, l0), n) / dot3(l, n);
        if (-tol < dd && dd < 1 + tol) {
            V3 p = sum3(l0, scale3(l, dd));
            double n2 = ncv * ncv;
            double l1 = dot3(cross3(diff3(p, p0), v2), cv) / n2;
            double l2 = -dot3(cross3(diff3(p, p0), v1), cv) / n2;
            if (-tol < std::fmin(l1, l2) && std::fmax(l1, l2) < 1 + tol) keep = 0;
        }
    }
    return keep;
}

}  // namespace

// ===========================================================================
extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

orc_system* orc_create(const orc_params* p)
{
    if (!p) {
        fail("null params");
        return nullptr;
    }
    if (p->pd_model == ORC_PD_NONE && p->contact_model == ORC_CONTACT_NONE) {
        fail("need a PD model or a contact model");
        return nullptr;
    }
    if (p->pd_model == ORC_PD_LINEAR_PMB && p->fracture) {
        // Force<LinearPMB, Fracture> is not defined (force/CabanaPD_PMB.hpp:407).
        fail("LinearPMB has no fracture variant");
        return nullptr;
    }
    orc_system* s = new orc_system();
    Model& md = s->model;
    // LinearLPS computes with the LPS kernels: ForceModel<LinearLPS>
    // (force_models/CabanaPD_LPS.hpp:255-272) keeps the base model's
    // force_tag = LPS (:32), and the Solver and the unit tests instantiate
    // Force<memory_space, force_tag, fracture_type> (CabanaPD_Solver.hpp:96-99,
    // unit_test/tstForce.hpp:927), so Force<LinearLPS> is never selected.
    md.pd = p->pd_model == ORC_PD_LINEAR_LPS ? ORC_PD_LPS : p->pd_model;
    md.fracture = p->fracture;
    md.contact = p->contact_model;
    md.horizon = p->horizon;
    md.K = p->K;
    md.G = p->G;
    md.G0 = p->G0;
    const bool lps = md.pd == ORC_PD_LPS;
    md.influence = p->influence_type >= 0 ? p->influence_type : (lps ? 0 : 1);
    if (md.pd != ORC_PD_NONE) {
        const double h = md.horizon;
        // force_models/CabanaPD_PMB.hpp:41-47
        md.c = 18.0 * md.K / (kPi * h * h * h * h);
        // force_models/CabanaPD_LPS.hpp:64-75
        md.theta_coeff = 3.0 * md.K - 5.0 * md.G;
        md.s_coeff = 15.0 * md.G;
        if (md.fracture) {
            // CabanaPD_ForceModels.hpp:93-102 (and LPS ctor :209-223)
            md.s0 = std::sqrt(5.0 * md.G0 / 9.0 / md.K / h);
            if (md.influence == 0) md.s0 = std::sqrt(8.0 * md.G0 / 15.0 / md.K / h);
            md.bond_break_coeff = (1.0 + md.s0) * (1.0 + md.s0);
        }
    }
    if (md.contact == ORC_CONTACT_HERTZ) {
        // force_models/CabanaPD_Hertzian.hpp:40-56
        md.radius = p->contact_radius;
        md.radius_extend = p->radius_extend;
        md.nu = p->nu;
        md.E = p->E;
        md.e = p->restitution;
        md.Rs = 0.5 * md.radius;
        md.Es = md.E / (2.0 * (1.0 - std::pow(md.nu, 2.0)));
        double ln_e = std::log(md.e);
        md.beta = -ln_e / std::sqrt(std::pow(ln_e, 2.0) + std::pow(kPi, 2.0));
        md.coeff_h_n = 4.0 / 3.0 * md.Es * std::sqrt(md.Rs);
        md.coeff_h_d = -2.0 * std::sqrt(5.0 / 6.0) * md.beta;
        md.per_particle_radius = p->per_particle_radius;
    }
    if (md.contact == ORC_CONTACT_NORMAL_REPULSION) {
        // force_models/CabanaPD_Contact.hpp:70-79: c as the PMB model's, from
        // the contact model's own delta and K.
        md.radius = p->contact_radius;
        md.radius_extend = p->radius_extend;
        md.contact_horizon = p->contact_horizon;
        const double h = md.contact_horizon;
        md.c_contact = 18.0 * p->contact_K / (kPi * h * h * h * h);
    }
    s->dt = p->dt;
    s->rebuild_every = p->rebuild_every;
    return s;
}

void orc_destroy(orc_system* s) { delete s; }

int orc_model_constants(const orc_system* s, double* o)
{
    const Model& m = s->model;
    double v[10] = {m.c,     m.s0, m.bond_break_coeff, m.theta_coeff, m.s_coeff,
                    m.Rs,    m.Es, m.beta,             m.coeff_h_n,   m.coeff_h_d};
    std::memcpy(o, v, sizeof(v));
    return 0;
}

int orc_set_particles(orc_system* s, int64_t n, int64_t n_frozen,
                      const double* x, const double* vol, const double* rho,
                      const int32_t* nofail, const double* radius)
{
    if (n <= 0 || n_frozen < 0 || n_frozen > n || !x || !vol)
        return fail("orc_set_particles: bad arguments");
    s->n = n;
    s->frozen = n_frozen;
    s->x.assign(x, x + 3 * n);
    s->vol.assign(vol, vol + n);
    if (rho)
        s->rho.assign(rho, rho + n);
    else
        s->rho.assign(n, 1.0);
    if (nofail)
        s->nofail.assign(nofail, nofail + n);
    else
        s->nofail.assign(n, 0);
    if (radius)
        s->radius.assign(radius, radius + n);
    else
        s->radius.assign(n, s->model.radius);
    s->u.assign(3 * n, 0.0);
    s->v.assign(3 * n, 0.0);
    s->f.assign(3 * n, 0.0);
    s->u_neigh.assign(3 * n, 0.0);
    s->m.assign(n, 0.0);
    s->theta.assign(n, 0.0);
    s->W.assign(n, 0.0);
    s->phi.assign(n, 0.0);
    s->stress.assign(9 * (size_t)n, 0.0);
    s->ready = false;
    return 0;
}

int orc_set_state(orc_system* s, const double* u, const double* v)
{
    if (s->n == 0) return fail("orc_set_state: no particles");
    if (u) s->u.assign(u, u + 3 * s->n);
    if (v) s->v.assign(v, v + 3 * s->n);
    return 0;
}

// Overwrites a whole vector field (u, v or f): the sharding tests write
// ghost rows between steps.
int orc_set_field(orc_system* s, int32_t field, const double* in)
{
    if (s->n == 0) return fail("orc_set_field: no particles");
    std::vector<double>* dst = nullptr;
    switch (field) {
    case ORC_FIELD_U: dst = &s->u; break;
    case ORC_FIELD_V: dst = &s->v; break;
    case ORC_FIELD_F: dst = &s->f; break;
    default: return fail("orc_set_field: only u, v and f");
    }
    dst->assign(in, in + 3 * s->n);
    return 0;
}

int orc_build_neighbors(orc_system* s)
{
    if (s->n == 0) return fail("orc_build_neighbors: no particles");
    const Model& md = s->model;
    if (md.pd != ORC_PD_NONE) {
        // CabanaPD_Neighbor.hpp:56-59: reference positions, cutoff + 1e-14.
        build_list(s->x, s->n, s->frozen, md.horizon + 1e-14, s->pd_list);
        s->mu.assign((size_t)s->n * std::max(s->pd_list.max_n, 1), 1);
    }
    if (md.contact != ORC_CONTACT_NONE) {
        // CabanaPD_Neighbor.hpp:60-63: current positions, cutoff + 1e-14.
        build_contact_list(*s, 2.0 * md.radius + md.radius_extend + 1e-14);
        s->rebuilds = 0;
    }
    return 0;
}

int orc_neighbor_stats(const orc_system* s, int32_t* max_n, int64_t* total)
{
    const NList& nl = s->model.pd != ORC_PD_NONE ? s->pd_list : s->contact_list;
    if (max_n) *max_n = nl.max_n;
    if (total) *total = nl.total;
    return 0;
}

int orc_get_neighbors(const orc_system* s, int32_t* counts, int32_t* idx,
                      int32_t* mu)
{
    const bool pd = s->model.pd != ORC_PD_NONE;
    const NList& nl = pd ? s->pd_list : s->contact_list;
    for (int64_t i = 0; i < s->n; i++) {
        if (counts) counts[i] = nl.count[i];
        for (int32_t k = 0; k < nl.max_n; k++) {
            size_t o = (size_t)i * nl.max_n + k;
            if (idx) idx[o] = k < nl.count[i] ? nl.idx[o] : -1;
            if (mu) mu[o] = (pd && k < nl.count[i] && !s->mu.empty()) ? s->mu[o] : 0;
        }
    }
    return 0;
}

// The broken-bond state packed as the product stores it (for comparing
// large systems without the full neighbour arrays): bits[w][n], bit b of
// word w of row i = mu of slot 32 w + b (1 = intact).
int orc_get_bond_bits(const orc_system* s, uint32_t* bits)
{
    const NList& nl = s->pd_list;
    if (s->mu.empty()) return fail("orc_get_bond_bits: no bond state");
    const int32_t words = (nl.max_n + 31) / 32;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < s->n; i++)
        for (int32_t w = 0; w < words; w++) {
            uint32_t v = 0;
            for (int32_t b = 0; b < 32; b++) {
                const int32_t k = 32 * w + b;
                if (k < nl.count[i] && s->mu[(size_t)i * nl.max_n + k] > 0) v |= 1u << b;
            }
            bits[(size_t)w * s->n + i] = v;
        }
    return 0;
}

// CabanaPD_Prenotch.hpp:215-263 Prenotch::create: i over [0, local).
int orc_prenotch(orc_system* s, int32_t k, const double* v1, const double* v2,
                 const double* p0)
{
    if (s->mu.empty()) return fail("orc_prenotch: needs a fracture model with neighbors");
    const NList& nl = s->pd_list;
    for (int32_t p = 0; p < k; p++) {
        V3 a{{v1[3 * p], v1[3 * p + 1], v1[3 * p + 2]}};
        V3 b{{v2[3 * p], v2[3 * p + 1], v2[3 * p + 2]}};
        V3 o{{p0[3 * p], p0[3 * p + 1], p0[3 * p + 2]}};
#pragma omp parallel for schedule(dynamic, 1024)
        for (int64_t i = 0; i < s->n; i++) {
            V3 xi{{s->x[3 * i], s->x[3 * i + 1], s->x[3 * i + 2]}};
            for (int32_t nn = 0; nn < nl.count[i]; nn++) {
                int64_t j = nl.idx[(size_t)i * nl.max_n + nn];
                V3 xj{{s->x[3 * j], s->x[3 * j + 1], s->x[3 * j + 2]}};
                if (!bond_prenotch_intersection(a, b, o, xi, xj))
                    s->mu[(size_t)i * nl.max_n + nn] = 0;
            }
        }
    }
    return 0;
}

int orc_add_bc(orc_system* s, int32_t kind, int32_t component, int64_t count,
               const int64_t* idx, const double* values)
{
    if (kind < 0 || kind > 2 || count < 0 || (count > 0 && !idx) || !values)
        return fail("orc_add_bc: bad arguments");
    if (kind == ORC_BC_FORCE_ADD && (component < 0 || component > 2))
        return fail("orc_add_bc: component must be 0..2");
    BC bc;
    bc.kind = kind;
    bc.component = component;
    bc.idx.assign(idx, idx + count);
    for (int64_t b = 0; b < count; b++)
        if (bc.idx[b] < 0 || bc.idx[b] >= s->n) return fail("orc_add_bc: index out of range");
    if (kind == ORC_BC_FORCE_ADD)
        bc.values.assign(values, values + count);
    else
        bc.values.assign(values, values + 1);
    s->bcs.push_back(std::move(bc));
    return 0;
}

int orc_compute_weighted_volume(orc_system* s)
{
    if (is_lps(*s)) lps_weighted_volume(*s);
    return 0;
}
int orc_compute_dilatation(orc_system* s)
{
    if (is_lps(*s)) lps_dilatation(*s);
    return 0;
}
int orc_compute_force(orc_system* s)
{
    if (has_pd(*s)) pd_force(*s);
    if (s->model.contact != ORC_CONTACT_NONE) contact_force(*s, !has_pd(*s));
    return 0;
}
int orc_compute_energy(orc_system* s, double* total_W, double* total_D)
{
    double Wt = 0, Dt = 0;
    if (has_pd(*s)) pd_energy(*s, Wt, Dt);
    if (total_W) *total_W = Wt;
    if (total_D) *total_D = Dt;
    return 0;
}

int orc_compute_stress(orc_system* s)
{
    if (has_pd(*s)) pd_stress(*s);
    return 0;
}

// CabanaPD_Solver.hpp:229-279 init(bc): weighted volume once without
// fracture, updateForce, energy, then the force BCs at t = 0.
int orc_init(orc_system* s)
{
    if (s->n == 0) return fail("orc_init: no particles");
    if (has_pd(*s) && is_lps(*s) && !s->model.fracture) lps_weighted_volume(*s);
    if (has_pd(*s)) {
        if (is_lps(*s)) {
            if (s->model.fracture) lps_weighted_volume(*s);
            lps_dilatation(*s);
        }
        pd_force(*s);
    }
    // Solver::init calls updateForce only: with a PD model the contact force
    // first appears in runStep (Solver.hpp:361-363); a DEM-only solver's
    // force model is the contact model (reset = true, list just built).
    if (!has_pd(*s) && s->model.contact != ORC_CONTACT_NONE) contact_force(*s, true);
    double W, D;
    if (has_pd(*s)) pd_energy(*s, W, D);
    apply_force_bcs(*s);
    s->ready = true;
    return 0;
}

// CabanaPD_Solver.hpp:332-375 runStep(step, bc), num_steps times.
int orc_run(orc_system* s, int32_t num_steps)
{
    if (!s->ready) return fail("orc_run: call orc_init first");
    for (int32_t k = 0; k < num_steps; k++) {
        vv_initial(*s);
        update_force(*s);
        apply_force_bcs(*s);
        vv_final(*s);
    }
    return 0;
}

int orc_get(const orc_system* s, int32_t field, double* out)
{
    const std::vector<double>* src = nullptr;
    switch (field) {
    case ORC_FIELD_X: src = &s->x; break;
    case ORC_FIELD_U: src = &s->u; break;
    case ORC_FIELD_V: src = &s->v; break;
    case ORC_FIELD_F: src = &s->f; break;
    case ORC_FIELD_VOL: src = &s->vol; break;
    case ORC_FIELD_RHO: src = &s->rho; break;
    case ORC_FIELD_M: src = &s->m; break;
    case ORC_FIELD_THETA: src = &s->theta; break;
    case ORC_FIELD_W: src = &s->W; break;
    case ORC_FIELD_PHI: src = &s->phi; break;
    case ORC_FIELD_RADIUS: src = &s->radius; break;
    case ORC_FIELD_STRESS: src = &s->stress; break;
    default: return fail("orc_get: unknown field");
    }
    std::memcpy(out, src->data(), src->size() * sizeof(double));
    return 0;
}

double orc_max_displacement(const orc_system* s) { return s->max_displacement; }
int64_t orc_contact_rebuilds(const orc_system* s) { return s->rebuilds; }

// CabanaPD_Input.hpp:217-301 computeCriticalTimeStep (mechanics part).
double orc_critical_timestep(double dx, double dy, double dz, int32_t m,
                             double horizon, double K, double rho)
{
    double v_p = dx * dy * dz;
    double sum = 0;
    double c = 18.0 * K / (kPi * horizon * horizon * horizon * horizon);
    for (int i = -(m + 1); i < m + 2; i++) {
        double xi_1 = i * dx;
        for (int j = -(m + 1); j < m + 2; j++) {
            double xi_2 = j * dy;
            for (int k = -(m + 1); k < m + 2; k++) {
                double xi_3 = k * dz;
                double r2 = xi_1 * xi_1 + xi_2 * xi_2 + xi_3 * xi_3;
                if (r2 < horizon * horizon + 1e-10) {
                    if (r2 > 0) {
                        double xi = std::sqrt(r2);
                        sum += v_p * c / xi;
                    }
                }
            }
        }
    }
    return std::sqrt(2.0 * rho / sum);
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_num_threads(int32_t n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

}  // extern "C"
