// Plain-FP64 particle kernels of the hot path.
//
// This translation unit is compiled with --fmad=false: every per-bond
// expression is evaluated with separately rounded IEEE double operations in
// the reference's operand order, so per-particle sums walked in the same
// neighbour order are bit-identical to a scalar CPU evaluation of the
// reference's code. sqrt and '/' on doubles are the IEEE-rounded CUDA
// operations.
//
// Work decomposition: one thread per particle row. A thread keeps particle
// i's position, displacement and running force in registers and walks its
// padded-ELL row; the k-th loads of a warp's 32 consecutive rows are
// contiguous in the column-major list, and neighbour gathers of a lattice in
// x-fastest order are contiguous as well. Broken-bond state is one bit per
// bond, read and written a 32-bond word at a time.
#include <cuda_runtime.h>

#include "cpd_internal.cuh"
#include "cpd_epilogue.cuh"

namespace cpd {
namespace {

constexpr int kBlock = 256;

inline int blocks_for(int64_t rows) { return (int)((rows + kBlock - 1) / kBlock); }

struct ModelDev {
    double c, theta_coeff, s_coeff, bond_break_coeff;
    double Rs, Es, coeff_h_n, coeff_h_d, radius;
};

ModelDev to_dev(const Model& m)
{
    return ModelDev{m.c,  m.theta_coeff, m.s_coeff,   m.bond_break_coeff, m.Rs,
                    m.Es, m.coeff_h_n,   m.coeff_h_d, m.radius};
}

// CabanaPD_Force.hpp:74-93 getDistance for the pair (i, j); particle i's
// position and displacement are already in registers.
__device__ __forceinline__ void bond_geometry(
    const double* __restrict__ x, const double* __restrict__ u, int64_t np,
    int64_t j, double xi0, double xi1, double xi2, double ui0, double ui1,
    double ui2, double& xi, double& r, double& s, double& rx, double& ry,
    double& rz, double& xx, double& xy, double& xz)
{
    xx = __ldg(x + j) - xi0;
    const double eta_u = __ldg(u + j) - ui0;
    xy = __ldg(x + np + j) - xi1;
    const double eta_v = __ldg(u + np + j) - ui1;
    xz = __ldg(x + 2 * np + j) - xi2;
    const double eta_w = __ldg(u + 2 * np + j) - ui2;
    rx = xx + eta_u;
    ry = xy + eta_v;
    rz = xz + eta_w;
    r = sqrt(rx * rx + ry * ry + rz * rz);
    xi = sqrt(xx * xx + xy * xy + xz * xz);
    s = (r - xi) / xi;
}

// CabanaPD_Force.hpp:114-129 getLinearizedDistance.
__device__ __forceinline__ void bond_linearized(
    const double* __restrict__ x, const double* __restrict__ u, int64_t np,
    int64_t j, double xi0, double xi1, double xi2, double ui0, double ui1,
    double ui2, double& xi, double& s, double& xx, double& xy, double& xz)
{
    xx = __ldg(x + j) - xi0;
    const double eta_u = __ldg(u + j) - ui0;
    xy = __ldg(x + np + j) - xi1;
    const double eta_v = __ldg(u + np + j) - ui1;
    xz = __ldg(x + 2 * np + j) - xi2;
    const double eta_w = __ldg(u + 2 * np + j) - ui2;
    xi = sqrt(xx * xx + xy * xy + xz * xz);
    s = (xx * eta_u + xy * eta_v + xz * eta_w) / (xi * xi);
}

// force_models/CabanaPD_LPS.hpp:85-98.
template <int INFL>
__device__ __forceinline__ double influence(double xi)
{
    if (INFL == 1) return 1.0 / xi;
    return 1.0;
}

// ---------------------------------------------------------------------------
// LPS weighted volume: force/CabanaPD_LPS.hpp:89-112 (NoFracture) and
// :287-329 (Fracture). m_i = sum_k mu_k * omega(xi) xi^2 vol_j.
template <int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock)
    k_lps_weighted_volume(ParticleView p, EllView nl)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const int cnt = nl.count[i];
    double mi = 0.0;
    uint32_t word = 0;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) word = nl.mu[(int64_t)(k >> 5) * np + i];
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        double xi, r, s, rx, ry, rz, xx, xy, xz;
        bond_geometry(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, r, s, rx,
                      ry, rz, xx, xy, xz);
        const double wv = influence<INFL>(xi) * xi * xi * __ldg(p.vol + j);
        if (FRACTURE)
            mi += (double)((word >> (k & 31)) & 1u) * wv;
        else
            mi += wv;
    }
    p.m[i] = mi;
}

// LPS dilatation: force/CabanaPD_LPS.hpp:114-141 (NoFracture), :331-378
// (Fracture). Also stores the per-particle factors of the force coefficient
// (force_models/CabanaPD_LPS.hpp:118-134): a = theta_coeff*theta/m and
// b = s_coeff/m, the exact subexpressions the force loop would otherwise
// recompute for every bond.
template <int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock)
    k_lps_dilatation(ParticleView p, EllView nl, ModelDev md)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const double m_i = p.m[i];
    const int cnt = nl.count[i];
    double th = 0.0;
    uint32_t word = 0;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) word = nl.mu[(int64_t)(k >> 5) * np + i];
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        double xi, r, s, rx, ry, rz, xx, xy, xz;
        bond_geometry(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, r, s, rx,
                      ry, rz, xx, xy, xz);
        const double theta_i = influence<INFL>(xi) * s * xi * xi * __ldg(p.vol + j);
        const double term = 3.0 * theta_i / m_i;
        if (FRACTURE) {
            if (m_i > 0) th += (double)((word >> (k & 31)) & 1u) * term;
        } else {
            th += term;
        }
    }
    p.theta[i] = th;
    p.lps_a[i] = md.theta_coeff * th / m_i;
    p.lps_b[i] = md.s_coeff / m_i;
}

// ---------------------------------------------------------------------------
// PD force. PMB: force/CabanaPD_PMB.hpp:89-125 (NoFracture), :222-287
// (Fracture); LinearPMB :406-455; LPS: force/CabanaPD_LPS.hpp:143-181
// (NoFracture), :380-447 (Fracture). LinearLPS systems run as LPS.
// The force is written (not accumulated): CabanaPD_Force.hpp:187-189 zeroes
// f before the kernel, and 0.0 + t == t.
enum { M_PMB = 0, M_LPS = 1, M_LINEAR_PMB = 2 };

template <int MODEL, int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock)
    k_pd_force(ParticleView p, EllView nl, ModelDev md)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    constexpr bool lps = MODEL == M_LPS;
    constexpr bool linear = MODEL == M_LINEAR_PMB;
    double a_i = 0.0, b_i = 0.0;
    if (lps) {
        a_i = p.lps_a[i];
        b_i = p.lps_b[i];
    }
    const bool nofail_i = FRACTURE ? (p.nofail[i] != 0) : false;
    const int cnt = nl.count[i];
    double fx = 0.0, fy = 0.0, fz = 0.0;
    uint32_t word = 0;
    bool dirty = false;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) {
            if (dirty) nl.mu[(int64_t)((k >> 5) - 1) * np + i] = word;
            dirty = false;
            word = nl.mu[(int64_t)(k >> 5) * np + i];
        }
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        const double vol_j = __ldg(p.vol + j);
        if (linear) {
            double xi, ls, xx, xy, xz;
            bond_linearized(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, ls,
                            xx, xy, xz);
            const double coeff = md.c * ls * vol_j;
            fx += coeff * xx / xi;
            fy += coeff * xy / xi;
            fz += coeff * xz / xi;
            continue;
        }
        double xi, r, s, rx, ry, rz, xx, xy, xz;
        bond_geometry(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, r, s, rx,
                      ry, rz, xx, xy, xz);
        bool intact = true;
        if (FRACTURE) {
            // CabanaPD_ForceModels.hpp:123-128. LPS tests nofail(i) twice
            // (force/CabanaPD_LPS.hpp:417-418), PMB nofail(i) and nofail(j).
            const bool critical = r * r >= md.bond_break_coeff * xi * xi;
            const bool nofail_other = lps ? nofail_i : (__ldg(p.nofail + j) != 0);
            const uint32_t bit = 1u << (k & 31);
            if (critical && !nofail_i && !nofail_other) {
                if (word & bit) {
                    word &= ~bit;
                    dirty = true;
                }
                intact = false;
            } else {
                intact = (word & bit) != 0;
            }
        }
        if (intact) {
            double coeff;
            if (lps) {
                const double a_j = __ldg(p.lps_a + j), b_j = __ldg(p.lps_b + j);
                coeff = (a_i + a_j + s * (b_i + b_j)) * influence<INFL>(xi) * xi * vol_j;
            } else {
                coeff = md.c * s * vol_j;
            }
            // mu == 1 here, and 1.0 * coeff == coeff.
            fx += coeff * rx / r;
            fy += coeff * ry / r;
            fz += coeff * rz / r;
        }
    }
    if (FRACTURE && dirty && cnt > 0) nl.mu[(int64_t)((cnt - 1) >> 5) * np + i] = word;
    p.f[i] = fx;
    p.f[np + i] = fy;
    p.f[2 * np + i] = fz;
}

// ---------------------------------------------------------------------------
// Strain energy density and damage: force/CabanaPD_PMB.hpp:127-155
// (NoFracture), :289-339 (Fracture), :458-491 (LinearPMB);
// force/CabanaPD_LPS.hpp:183-219, :449-504.
// Per particle W_i and phi_i are exact; the block partial sums of
// (sum_k w_k vol_i or W_i vol_i, phi_i) are reduced in a fixed tree order.
template <int MODEL, int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock)
    k_pd_energy(ParticleView p, EllView nl, ModelDev md, double* partials)
{
    __shared__ double s_phi[kBlock];
    __shared__ double s_dmg[kBlock];
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double Phi_i = 0.0, dmg_i = 0.0;
    if (i < p.n) {
        const int64_t np = p.npad;
        const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
        const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
        constexpr bool lps = MODEL == M_LPS;
        constexpr bool linear = MODEL == M_LINEAR_PMB;
        const int cnt = nl.count[i];
        const double vol_i = p.vol[i];
        double m_i = 0.0, th_i = 0.0;
        if (lps) {
            m_i = p.m[i];
            th_i = p.theta[i];
        }
        double num_bonds = (double)cnt;
        if (FRACTURE && lps) {
            num_bonds = 0.0;
            for (int k = 0; k < cnt; ++k) {
                const uint32_t word = nl.mu[(int64_t)(k >> 5) * np + i];
                num_bonds += (double)((word >> (k & 31)) & 1u);
            }
        }
        double Wi = 0.0, phi_sum = 0.0, vol_H = 0.0;
        uint32_t word = 0;
        for (int k = 0; k < cnt; ++k) {
            if (FRACTURE && (k & 31) == 0) word = nl.mu[(int64_t)(k >> 5) * np + i];
            const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
            const double vol_j = __ldg(p.vol + j);
            double s, xi;
            if (linear) {
                double xx, xy, xz;
                bond_linearized(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, s,
                                xx, xy, xz);
            } else {
                double r, rx, ry, rz, xx, xy, xz;
                bond_geometry(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, r, s,
                              rx, ry, rz, xx, xy, xz);
            }
            double w;
            if (lps) {
                // force_models/CabanaPD_LPS.hpp:136-148
                w = 1.0 / num_bonds * 0.5 * md.theta_coeff / 3.0 * (th_i * th_i) +
                    0.5 * (md.s_coeff / m_i) * influence<INFL>(xi) * s * s * xi * xi *
                        vol_j;
            } else {
                // force_models/CabanaPD_PMB.hpp:64-71
                w = 0.25 * md.c * s * s * xi * vol_j;
            }
            if (FRACTURE) {
                const double mu = (double)((word >> (k & 31)) & 1u);
                w = mu * w;
                Wi += w;
                phi_sum += mu * vol_j;
                vol_H += vol_j;
            } else {
                Wi += w;
                Phi_i += w * vol_i;
            }
        }
        p.W[i] = Wi;
        if (FRACTURE) {
            dmg_i = 1 - phi_sum / vol_H;
            p.phi[i] = dmg_i;
            Phi_i = Wi * vol_i;
        }
    }
    s_phi[threadIdx.x] = Phi_i;
    s_dmg[threadIdx.x] = dmg_i;
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s_phi[threadIdx.x] += s_phi[threadIdx.x + w];
            s_dmg[threadIdx.x] += s_dmg[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x + 0] = s_phi[0];
        partials[2 * blockIdx.x + 1] = s_dmg[0];
    }
}

// Per-particle stress: force/CabanaPD_PMB.hpp:157-202 (NoFracture), :341-401
// (Fracture), :492-537 (LinearPMB); force/CabanaPD_LPS.hpp:221-267
// (NoFracture), :506-572 (Fracture: intact bonds only). Half the pair force
// times the reference bond vector, sigma(i, a, b) = sum_k f_a xi_b over the
// row in row order (the caller zeroes sigma first, CabanaPD_Force.hpp:
// 229-231). Component-major: sigma[(3 a + b) npad + i]. LPS uses the factors
// a = theta_coeff theta / m and b = s_coeff / m of the last force update,
// exact subexpressions of the reference's coefficient.
template <int MODEL, int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock)
    k_pd_stress(ParticleView p, EllView nl, ModelDev md, double* __restrict__ sigma)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    constexpr bool lps = MODEL == M_LPS;
    constexpr bool linear = MODEL == M_LINEAR_PMB;
    double a_i = 0.0, b_i = 0.0;
    if (lps) {
        a_i = p.lps_a[i];
        b_i = p.lps_b[i];
    }
    const int cnt = nl.count[i];
    double S[9] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    uint32_t word = 0;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) word = nl.mu[(int64_t)(k >> 5) * np + i];
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        const double vol_j = __ldg(p.vol + j);
        double fx, fy, fz, xx, xy, xz;
        if (linear) {
            double xi, ls;
            bond_linearized(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, ls, xx, xy,
                            xz);
            const double coeff = 0.5 * (md.c * ls * vol_j);
            fx = coeff * xx / xi;
            fy = coeff * xy / xi;
            fz = coeff * xz / xi;
        } else {
            const double mu = FRACTURE ? (double)((word >> (k & 31)) & 1u) : 1.0;
            if (FRACTURE && lps && !(mu > 0.0)) continue;
            double xi, r, s, rx, ry, rz;
            bond_geometry(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, r, s, rx, ry,
                          rz, xx, xy, xz);
            double coeff;
            if (lps) {
                const double a_j = __ldg(p.lps_a + j), b_j = __ldg(p.lps_b + j);
                coeff = (a_i + a_j + s * (b_i + b_j)) * influence<INFL>(xi) * xi * vol_j;
                coeff *= 0.5;
            } else {
                coeff = 0.5 * (md.c * s * vol_j);
            }
            if (FRACTURE) {
                fx = mu * coeff * rx / r;
                fy = mu * coeff * ry / r;
                fz = mu * coeff * rz / r;
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
    for (int c = 0; c < 9; ++c) sigma[(int64_t)c * np + i] = S[c];
}

// Single-block fixed-order sum of [nblocks][ncols] partials.
__global__ void __launch_bounds__(kBlock)
    k_sum_partials(const double* partials, int nblocks, int ncols, double* out)
{
    __shared__ double s[kBlock];
    for (int c = 0; c < ncols; ++c) {
        double acc = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += kBlock) acc += partials[(int64_t)b * ncols + c];
        s[threadIdx.x] = acc;
        __syncthreads();
        for (int w = kBlock / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = s[0];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock)
    k_max_partials(const double* partials, int nblocks, double* out)
{
    __shared__ double s[kBlock];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kBlock) acc = fmax(acc, partials[b]);
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s[0];
}

// ---------------------------------------------------------------------------
// Hertzian contact: force/CabanaPD_Contact.hpp:119-168 with
// force_models/CabanaPD_Hertzian.hpp:58-87 (normalForce; tangentialForce is
// a no-op that adds 0.0). With per-particle radii the pair uses
// R* = R_i (R_j / (R_i + R_j)), overlap r - (R_i + R_j) and
// m* = m_i (m_j / (m_i + m_j)), which round to the single-radius values when
// R_i == R_j.
// EPI: a contact-only fused step; the epilogue finishes the row (force BC,
// half steps, next displacement and velocity into the second buffers).
template <bool PER_PARTICLE, bool EPI = false>
__global__ void __launch_bounds__(kBlock, 3)
    k_hertz_force(ParticleView p, EllView nl, ModelDev md, bool reset, StepEpilogue ep)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const double vi0 = p.v[i], vi1 = p.v[np + i], vi2 = p.v[2 * np + i];
    const double vol_i = p.vol[i], rho_i = p.rho[i];
    const double R_i = PER_PARTICLE ? p.radius[i] : 0.0;
    double fx = reset ? 0.0 : p.f[i];
    double fy = reset ? 0.0 : p.f[np + i];
    double fz = reset ? 0.0 : p.f[2 * np + i];
    const int cnt = nl.count[i];
    for (int k = 0; k < cnt; ++k) {
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        double xi, r, s, rx, ry, rz, xx, xy, xz;
        bond_geometry(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, xi, r, s, rx,
                      ry, rz, xx, xy, xz);
        const double R_j = PER_PARTICLE ? p.radius[j] : 0.0;
        const double sum_r = PER_PARTICLE ? R_i + R_j : 2.0 * md.radius;
        const double delta_n = r - sum_r;
        // Without overlap the pair adds a zero: skip it (the sum is unchanged;
        // at most a zero sum keeps the sign the reference's + 0.0 would
        // clear).
        if (!(delta_n < 0.0)) continue;
        const double nx = rx / r, ny = ry / r, nz = rz / r;
        const double vx = p.v[j] - vi0;
        const double vy = p.v[np + j] - vi1;
        const double vz = p.v[2 * np + j] - vi2;
        const double vn = vx * nx + vy * ny + vz * nz;
        double Rs, coeff_h_n, ms;
        if (PER_PARTICLE) {
            Rs = R_i * (R_j / (R_i + R_j));
            coeff_h_n = 4.0 / 3.0 * md.Es * sqrt(Rs);
            const double mi = rho_i * vol_i;
            const double mj = p.rho[j] * p.vol[j];
            ms = mi * (mj / (mi + mj));
        } else {
            Rs = md.Rs;
            coeff_h_n = md.coeff_h_n;
            ms = (rho_i * vol_i) / 2.0;
        }
        double coeff = 0.0;
        if (delta_n < 0.0) {
            const double h = -coeff_h_n * pow(fabs(delta_n), 3.0 / 2.0);
            coeff = (h < 0.0) ? h : 0.0;
        }
        coeff /= vol_i;
        double Sn = 0.0;
        if (delta_n < 0.0) Sn = 2.0 * md.Es * sqrt(Rs * fabs(delta_n));
        coeff -= md.coeff_h_d * sqrt(Sn * ms) * vn / vol_i;
        fx += coeff * nx;
        fy += coeff * ny;
        fz += coeff * nz;
        fx += 0.0;
        fy += 0.0;
        fz += 0.0;
    }
    if (EPI) {
        step_epilogue<false>(p, ep, i, fx, fy, fz);
        return;
    }
    p.f[i] = fx;
    p.f[np + i] = fy;
    p.f[2 * np + i] = fz;
}

// ---------------------------------------------------------------------------
// Normal repulsion: force/CabanaPD_Contact.hpp:52-92 with
// NormalRepulsionModel::forceCoeff (force_models/CabanaPD_Contact.hpp:82-88).
// A pair whose current distance r is below the contact radius adds
// ((15 c) sc) vol_j r_d / r per component, sc = (r - radius) / delta_c; the
// coefficient is negative, so the pair pushes i away from j. Pairs farther
// apart add a zero and are skipped (only the sign of a zero sum can differ).
// The reference distance and stretch of getDistance are not used here.
__global__ void __launch_bounds__(kBlock)
    k_repulsion_force(ParticleView p, EllView nl, double radius, double c15,
                      double delta, bool reset)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    double fx = reset ? 0.0 : p.f[i];
    double fy = reset ? 0.0 : p.f[np + i];
    double fz = reset ? 0.0 : p.f[2 * np + i];
    const int cnt = nl.count[i];
    for (int k = 0; k < cnt; ++k) {
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        const double xx = __ldg(p.x + j) - xi0;
        const double eu = __ldg(p.u + j) - ui0;
        const double xy = __ldg(p.x + np + j) - xi1;
        const double ev = __ldg(p.u + np + j) - ui1;
        const double xz = __ldg(p.x + 2 * np + j) - xi2;
        const double ew = __ldg(p.u + 2 * np + j) - ui2;
        const double rx = xx + eu, ry = xy + ev, rz = xz + ew;
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        if (!(r < radius)) continue;
        const double sc = (r - radius) / delta;
        const double coeff = c15 * sc * p.vol[j];
        fx += coeff * rx / r;
        fy += coeff * ry / r;
        fz += coeff * rz / r;
    }
    p.f[i] = fx;
    p.f[np + i] = fy;
    p.f[2 * np + i] = fz;
}

// ---------------------------------------------------------------------------
// Velocity Verlet: CabanaPD_Integrate.hpp:89-116 (NoContact), :151-193
// (Contact: also the largest displacement since the last list build).
template <bool TRACK>
__global__ void __launch_bounds__(kBlock)
    k_vv_initial(ParticleView p, double dt, double half_dt, double* block_max, double* u_out)
{
    __shared__ double s_max[kBlock];
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double um = 0.0;
    if (i < p.n) {
        const int64_t np = p.npad;
        const double half_dt_m = half_dt / p.rho[i];
        double v0 = p.v[i] + half_dt_m * p.f[i];
        double v1 = p.v[np + i] + half_dt_m * p.f[np + i];
        double v2 = p.v[2 * np + i] + half_dt_m * p.f[2 * np + i];
        p.v[i] = v0;
        p.v[np + i] = v1;
        p.v[2 * np + i] = v2;
        const double u0 = p.u[i] + dt * v0;
        const double u1 = p.u[np + i] + dt * v1;
        const double u2 = p.u[2 * np + i] + dt * v2;
        u_out[i] = u0;
        u_out[np + i] = u1;
        u_out[2 * np + i] = u2;
        if (TRACK)
            um = norm3d(u0 - p.u_neigh[i], u1 - p.u_neigh[np + i],
                        u2 - p.u_neigh[2 * np + i]);
    }
    if (TRACK) {
        s_max[threadIdx.x] = um;
        __syncthreads();
        for (int w = kBlock / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w)
                s_max[threadIdx.x] = fmax(s_max[threadIdx.x], s_max[threadIdx.x + w]);
            __syncthreads();
        }
        if (threadIdx.x == 0) block_max[blockIdx.x] = s_max[0];
    }
}

__global__ void __launch_bounds__(kBlock) k_vv_final(ParticleView p, double half_dt)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double half_dt_m = half_dt / p.rho[i];
    p.v[i] += half_dt_m * p.f[i];
    p.v[np + i] += half_dt_m * p.f[np + i];
    p.v[2 * np + i] += half_dt_m * p.f[2 * np + i];
}

// CabanaPD_Boundary.hpp:94-113, :138-157 and the custom-functor form.
__global__ void __launch_bounds__(kBlock)
    k_force_bc(ParticleView p, int kind, int comp, int64_t count, const int32_t* idx,
               const double* values, double value)
{
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= count) return;
    const int64_t q = idx[b];
    const int64_t np = p.npad;
    if (kind == CPD_BC_FORCE_VALUE) {
        for (int d = 0; d < 3; d++) p.f[d * np + q] = value;
    } else if (kind == CPD_BC_FORCE_UPDATE) {
        for (int d = 0; d < 3; d++) p.f[d * np + q] += value;
    } else {
        p.f[comp * np + q] += values[b];
    }
}

// ---------------------------------------------------------------------------
// Pre-notch: CabanaPD_Prenotch.hpp:24-172 geometry, :215-263 create.
struct V3 {
    double a[3];
};
__device__ __forceinline__ double dot3(V3 a, V3 b)
{
    double v = 0;
    for (int d = 0; d < 3; d++) v += (a.a[d]) * (b.a[d]);
    return v;
}
__device__ __forceinline__ double norm3(V3 a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ V3 cross3(V3 a, V3 b)
{
    V3 c;
    c.a[0] = a.a[1] * b.a[2] - a.a[2] * b.a[1];
    c.a[1] = -(a.a[0] * b.a[2] - a.a[2] * b.a[0]);
    c.a[2] = a.a[0] * b.a[1] - a.a[1] * b.a[0];
    return c;
}
__device__ __forceinline__ V3 scale3(V3 a, double n)
{
    for (int d = 0; d < 3; d++) a.a[d] *= n;
    return a;
}
__device__ __forceinline__ V3 diff3(V3 a, V3 b)
{
    V3 c;
    for (int d = 0; d < 3; d++) c.a[d] = a.a[d] - b.a[d];
    return c;
}
__device__ __forceinline__ V3 sum3(V3 a, V3 b)
{
    V3 c;
    for (int d = 0; d < 3; d++) c.a[d] = a.a[d] + b.a[d];
    return c;
}

__device__ int bond_prenotch_intersection(V3 v1, V3 v2, V3 p0, V3 x_i, V3 x_j)
{
    const double tol = 1e-10;
    V3 cv = cross3(v1, v2);
    double ncv = norm3(cv);
    V3 n = scale3(cv, 1.0 / ncv);
    V3 l0 = x_i;
    V3 l = diff3(x_j, x_i);
    int flag;
    if (fabs(dot3(l, n)) < tol)
        flag = (fabs(dot3(diff3(p0, l0), n)) < tol) ? 1 : 2;
    else
        flag = 3;
    int keep = 1;
    if (flag == 1) {
        double n2 = ncv * ncv;
        double li1 = dot3(cross3(diff3(x_i, p0), v2), cv) / n2;
        double li2 = -dot3(cross3(diff3(x_i, p0), v1), cv) / n2;
        double lj1 = dot3(cross3(diff3(x_j, p0), v2), cv) / n2;
        double lj2 = -dot3(cross3(diff3(x_j, p0), v1), cv) / n2;
        if (!(fmin(li1, lj1) > 1 + tol || fmax(li1, lj1) < -tol ||
              fmin(li2, lj2) > 1 + tol || fmax(li2, lj2) < -tol))
            keep = 0;
    } else if (flag == 3) {
        double dd = dot3(diff3(p0, l0), n) / dot3(l, n);
        if (-tol < dd && dd < 1 + tol) {
            V3 q = sum3(l0, scale3(l, dd));
            double n2 = ncv * ncv;
            double l1 = dot3(cross3(diff3(q, p0), v2), cv) / n2;
            double l2 = -dot3(cross3(diff3(q, p0), v1), cv) / n2;
            if (-tol < fmin(l1, l2) && fmax(l1, l2) < 1 + tol) keep = 0;
        }
    }
    return keep;
}

// One notch per launch (as the reference). Particles whose horizon ball
// cannot reach the notch's bounding box (grown by `margin`) are skipped;
// the test is conservative, so the cut bond set is unchanged.
__global__ void __launch_bounds__(kBlock)
    k_prenotch(ParticleView p, EllView nl, V3 v1, V3 v2, V3 p0, V3 box_lo,
               V3 box_hi)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    V3 xi{{p.x[i], p.x[np + i], p.x[2 * np + i]}};
    for (int d = 0; d < 3; d++)
        if (xi.a[d] < box_lo.a[d] || xi.a[d] > box_hi.a[d]) return;
    const int cnt = nl.count[i];
    for (int w = 0; w * 32 < cnt; ++w) {
        uint32_t word = nl.mu[(int64_t)w * np + i];
        const uint32_t old = word;
        for (int b = 0; b < 32 && w * 32 + b < cnt; ++b) {
            const int k = w * 32 + b;
            const int64_t j = nl.idx[(int64_t)k * np + i];
            V3 xj{{p.x[j], p.x[np + j], p.x[2 * np + j]}};
            if (!bond_prenotch_intersection(v1, v2, p0, xi, xj)) word &= ~(1u << b);
        }
        if (word != old) nl.mu[(int64_t)w * np + i] = word;
    }
}

}  // namespace

// ===========================================================================
// Launchers.
int energy_blocks(int64_t nrows) { return nrows > 0 ? blocks_for(nrows) : 1; }
int vv_blocks(int64_t nrows) { return nrows > 0 ? blocks_for(nrows) : 1; }

int launch_vv_initial(const ParticleView& p, double dt, bool track_max,
                      double* block_max, int, double* u_out, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const double half_dt = 0.5 * dt;
    if (track_max)
        k_vv_initial<true><<<blocks_for(rows), kBlock, 0, st>>>(p, dt, half_dt, block_max, u_out);
    else
        k_vv_initial<false><<<blocks_for(rows), kBlock, 0, st>>>(p, dt, half_dt, nullptr, u_out);
    return 1;
}

int launch_vv_final(const ParticleView& p, double dt, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    k_vv_final<<<blocks_for(rows), kBlock, 0, st>>>(p, 0.5 * dt);
    return 1;
}

int launch_lps_weighted_volume(const ParticleView& p, const EllView& nl,
                               const Model& md, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const int g = blocks_for(rows);
    if (md.influence == 1) {
        if (md.fracture)
            k_lps_weighted_volume<1, true><<<g, kBlock, 0, st>>>(p, nl);
        else
            k_lps_weighted_volume<1, false><<<g, kBlock, 0, st>>>(p, nl);
    } else {
        if (md.fracture)
            k_lps_weighted_volume<0, true><<<g, kBlock, 0, st>>>(p, nl);
        else
            k_lps_weighted_volume<0, false><<<g, kBlock, 0, st>>>(p, nl);
    }
    return 1;
}

int launch_lps_dilatation(const ParticleView& p, const EllView& nl,
                          const Model& md, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const int g = blocks_for(rows);
    const ModelDev d = to_dev(md);
    if (md.influence == 1) {
        if (md.fracture)
            k_lps_dilatation<1, true><<<g, kBlock, 0, st>>>(p, nl, d);
        else
            k_lps_dilatation<1, false><<<g, kBlock, 0, st>>>(p, nl, d);
    } else {
        if (md.fracture)
            k_lps_dilatation<0, true><<<g, kBlock, 0, st>>>(p, nl, d);
        else
            k_lps_dilatation<0, false><<<g, kBlock, 0, st>>>(p, nl, d);
    }
    return 1;
}


#define CPD_PD_DISPATCH(KERNEL, GRID, ...)                                          \
    do {                                                                            \
        const int infl = md.influence == 1 ? 1 : 0;                                 \
        switch (md.pd) {                                                            \
        case CPD_PD_PMB:                                                            \
            if (md.fracture)                                                        \
                KERNEL<M_PMB, 1, true><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);       \
            else                                                                    \
                KERNEL<M_PMB, 1, false><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);      \
            break;                                                                  \
        case CPD_PD_LINEAR_PMB:                                                     \
            KERNEL<M_LINEAR_PMB, 1, false><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);   \
            break;                                                                  \
        case CPD_PD_LPS:                                                            \
            if (md.fracture) {                                                      \
                if (infl)                                                           \
                    KERNEL<M_LPS, 1, true><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);   \
                else                                                                \
                    KERNEL<M_LPS, 0, true><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);   \
            } else {                                                                \
                if (infl)                                                           \
                    KERNEL<M_LPS, 1, false><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);  \
                else                                                                \
                    KERNEL<M_LPS, 0, false><<<GRID, kBlock, 0, st>>>(__VA_ARGS__);  \
            }                                                                       \
            break;                                                                  \
        default:                                                                    \
            return 0;                                                               \
        }                                                                           \
    } while (0)

int launch_pd_force(const ParticleView& p, const EllView& nl, const Model& md,
                    cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const int g = blocks_for(rows);
    const ModelDev d = to_dev(md);
    CPD_PD_DISPATCH(k_pd_force, g, p, nl, d);
    return 1;
}

int launch_pd_energy(const ParticleView& p, const EllView& nl, const Model& md,
                     double* partials, int nblocks, cudaStream_t st)
{
    const ModelDev d = to_dev(md);
    CPD_PD_DISPATCH(k_pd_energy, nblocks, p, nl, d, partials);
    return 1;
}

int launch_pd_stress(const ParticleView& p, const EllView& nl, const Model& md, double* sigma,
                     cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const int g = blocks_for(rows);
    const ModelDev d = to_dev(md);
    CPD_PD_DISPATCH(k_pd_stress, g, p, nl, d, sigma);
    return 1;
}

int launch_sum_partials(const double* partials, int nblocks, int ncols,
                        double* out, cudaStream_t st)
{
    k_sum_partials<<<1, kBlock, 0, st>>>(partials, nblocks, ncols, out);
    return 1;
}

int launch_max_partials(const double* partials, int nblocks, double* out,
                        cudaStream_t st)
{
    k_max_partials<<<1, kBlock, 0, st>>>(partials, nblocks, out);
    return 1;
}

int launch_hertz_force(const ParticleView& p, const EllView& nl,
                       const Model& md, bool reset, cudaStream_t st, const StepEpilogue* ep)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const ModelDev d = to_dev(md);
    const StepEpilogue e = ep ? *ep : StepEpilogue{};
    const int g = blocks_for(rows);
    if (ep) {
        if (md.per_particle_radius)
            k_hertz_force<true, true><<<g, kBlock, 0, st>>>(p, nl, d, true, e);
        else
            k_hertz_force<false, true><<<g, kBlock, 0, st>>>(p, nl, d, true, e);
    } else if (md.per_particle_radius) {
        k_hertz_force<true><<<g, kBlock, 0, st>>>(p, nl, d, reset, e);
    } else {
        k_hertz_force<false><<<g, kBlock, 0, st>>>(p, nl, d, reset, e);
    }
    return 1;
}

int launch_repulsion_force(const ParticleView& p, const EllView& nl, const Model& md,
                           bool reset, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    k_repulsion_force<<<blocks_for(rows), kBlock, 0, st>>>(
        p, nl, md.radius, 15.0 * md.c_contact, md.contact_horizon, reset);
    return 1;
}

int launch_force_bc(const ParticleView& p, const BoundaryCondition& bc,
                    cudaStream_t st)
{
    if (bc.count <= 0) return 0;
    k_force_bc<<<blocks_for(bc.count), kBlock, 0, st>>>(p, bc.kind, bc.component,
                                                       bc.count, bc.idx, bc.values,
                                                       bc.value);
    return 1;
}

int launch_prenotch(const ParticleView& p, const EllView& nl, const double* v1,
                    const double* v2, const double* p0, double margin,
                    cudaStream_t st)
{
    if (p.n <= 0) return 0;
    V3 a{{v1[0], v1[1], v1[2]}}, b{{v2[0], v2[1], v2[2]}}, o{{p0[0], p0[1], p0[2]}};
    V3 lo, hi;
    for (int d = 0; d < 3; d++) {
        double c[4] = {o.a[d], o.a[d] + a.a[d], o.a[d] + b.a[d], o.a[d] + a.a[d] + b.a[d]};
        double mn = c[0], mx = c[0];
        for (int q = 1; q < 4; q++) {
            mn = c[q] < mn ? c[q] : mn;
            mx = c[q] > mx ? c[q] : mx;
        }
        lo.a[d] = mn - margin;
        hi.a[d] = mx + margin;
    }
    k_prenotch<<<blocks_for(p.n), kBlock, 0, st>>>(p, nl, a, b, o, lo, hi);
    return 1;
}

}  // namespace cpd
