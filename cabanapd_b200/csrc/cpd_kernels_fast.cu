// Plain-FP64 particle kernels, throughput form.
//
// Same physics and the same double precision as cpd_kernels_exact.cu, but
// each bond length costs one reciprocal square root and one correction step
// instead of an IEEE square root, and the divisions by xi and r become
// multiplications by the reciprocal square roots:
//   r2, xi2 summed in the reference's order without FMA (as the reference)
//   r  = sqrt(r2)  from y = rsqrt(r2): g = r2 y, e = r2 - g g (exact FMA
//        residual), r = g + e y / 2 -- the Newton-Raphson / Markstein
//        correction of the square root, which returns the correctly rounded
//        root except in rare hard cases (then within one ulp)
//   s  = (r - xi) * rsqrt(xi2)     (r - xi is exact, as in the reference)
//   f += (c s vol_j rsqrt(r2)) * r_vec
// Because r and xi carry the reference's rounding, s differs from the
// reference's (r - xi) / xi by a few ulps of s itself -- no 1/s growth -- and
// forces agree with the bit-exact path to ~1e-15 relative.
//
// Bond breaking stays exact: the reference's test is r * r >=
// (bond_break_coeff * xi) * xi (CabanaPD_ForceModels.hpp:123-128). Inside a
// relative guard band of 1e-12 the test is re-evaluated with correctly
// rounded intrinsics, so broken-bond sets are identical.
#include <cuda_runtime.h>

#include <cstdlib>

#include "cpd_epilogue.cuh"
#include "cpd_internal.cuh"

namespace cpd {
namespace {

constexpr int kBlock = 256;
constexpr double kGuard = 1e-12;

inline int blocks_for(int64_t rows) { return (int)((rows + kBlock - 1) / kBlock); }

// The reference's break test for bond vector xi = (xx, xy, xz) and deformed
// vector r = (rx, ry, rz), with every operation rounded separately.
__device__ __noinline__ bool critical_exact(double xx, double xy, double xz, double rx,
                                            double ry, double rz, double bbc)
{
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)),
                                __dmul_rn(rz, rz));
    const double x2 = __dadd_rn(__dadd_rn(__dmul_rn(xx, xx), __dmul_rn(xy, xy)),
                                __dmul_rn(xz, xz));
    const double r = __dsqrt_rn(r2);
    const double xi = __dsqrt_rn(x2);
    return __dmul_rn(r, r) >= __dmul_rn(__dmul_rn(bbc, xi), xi);
}

// Squared length summed as the reference sums it: (a*a + b*b) + c*c, each
// product and sum rounded (no FMA).
__device__ __forceinline__ double norm2_ref(double a, double b, double c)
{
    return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// sqrt(a) from y ~ 1/sqrt(a): one Newton-Raphson step on g = a y with the
// residual a - g^2 formed exactly by FMA (Markstein's correction).
__device__ __forceinline__ double sqrt_from_rsqrt(double a, double y)
{
    const double g = a * y;
    const double e = fma(-g, g, a);
    return fma(e, 0.5 * y, g);
}

struct Bond {
    double xx, xy, xz, rx, ry, rz;
    double r, xi, rinv, xiinv, s;
};

__device__ __forceinline__ void bond_fast(const double* __restrict__ X,
                                          const double* __restrict__ U, int64_t np,
                                          int64_t j, double xi0, double xi1, double xi2,
                                          double ui0, double ui1, double ui2, Bond& b)
{
    b.xx = __ldg(X + j) - xi0;
    b.xy = __ldg(X + np + j) - xi1;
    b.xz = __ldg(X + 2 * np + j) - xi2;
    b.rx = b.xx + (__ldg(U + j) - ui0);
    b.ry = b.xy + (__ldg(U + np + j) - ui1);
    b.rz = b.xz + (__ldg(U + 2 * np + j) - ui2);
    const double r2 = norm2_ref(b.rx, b.ry, b.rz);
    const double x2 = norm2_ref(b.xx, b.xy, b.xz);
    b.rinv = rsqrt(r2);
    b.xiinv = rsqrt(x2);
    b.r = sqrt_from_rsqrt(r2, b.rinv);
    b.xi = sqrt_from_rsqrt(x2, b.xiinv);
    b.s = (b.r - b.xi) * b.xiinv;
}

__device__ __forceinline__ bool critical_fast(const Bond& b, double bbc)
{
    const double lhs = __dmul_rn(b.r, b.r);
    const double rhs = __dmul_rn(__dmul_rn(bbc, b.xi), b.xi);
    if (fabs(lhs - rhs) <= kGuard * rhs)
        return critical_exact(b.xx, b.xy, b.xz, b.rx, b.ry, b.rz, bbc);
    return lhs >= rhs;
}

// Bond geometry from already-gathered neighbour data.
__device__ __forceinline__ void bond_from(double xj0, double xj1, double xj2, double uj0,
                                          double uj1, double uj2, double xi0, double xi1,
                                          double xi2, double ui0, double ui1, double ui2,
                                          Bond& b)
{
    b.xx = xj0 - xi0;
    b.xy = xj1 - xi1;
    b.xz = xj2 - xi2;
    b.rx = b.xx + (uj0 - ui0);
    b.ry = b.xy + (uj1 - ui1);
    b.rz = b.xz + (uj2 - ui2);
    const double r2 = norm2_ref(b.rx, b.ry, b.rz);
    const double x2 = norm2_ref(b.xx, b.xy, b.xz);
    b.rinv = rsqrt(r2);
    b.xiinv = rsqrt(x2);
    b.r = sqrt_from_rsqrt(r2, b.rinv);
    b.xi = sqrt_from_rsqrt(x2, b.xiinv);
    b.s = (b.r - b.xi) * b.xiinv;
}

// Neighbour data a bond needs, gathered ahead of its arithmetic.
struct Gather {
    double x0, x1, x2, u0, u1, u2, vol;
    bool nofail;
};

template <bool FRACTURE>
__device__ __forceinline__ void gather(const ParticleView& p, int64_t np, int64_t j, Gather& g)
{
    g.x0 = __ldg(p.x + j);
    g.x1 = __ldg(p.x + np + j);
    g.x2 = __ldg(p.x + 2 * np + j);
    g.u0 = __ldg(p.u + j);
    g.u1 = __ldg(p.u + np + j);
    g.u2 = __ldg(p.u + 2 * np + j);
    g.vol = __ldg(p.vol + j);
    g.nofail = FRACTURE ? (__ldg(p.nofail + j) != 0) : false;
}

// Neighbour indices of one ELL row read PF bonds ahead of use (a shift
// register), so the index load of bond k + PF overlaps the work of bond k.
template <int PF>
struct IndexStream {
    const int32_t* __restrict__ idx;
    int64_t np;
    int cnt;
    int32_t q[PF];
    __device__ __forceinline__ IndexStream(const int32_t* row, int64_t stride, int count)
        : idx(row), np(stride), cnt(count)
    {
#pragma unroll
        for (int a = 0; a < PF; ++a) q[a] = a < cnt ? __ldg(idx + (int64_t)a * np) : 0;
    }
    // Index of bond k (called for k = 0, 1, ... in order).
    __device__ __forceinline__ int64_t next(int k)
    {
        const int64_t j = q[0];
#pragma unroll
        for (int a = 0; a + 1 < PF; ++a) q[a] = q[a + 1];
        q[PF - 1] = (k + PF < cnt) ? __ldg(idx + (int64_t)(k + PF) * np) : 0;
        return j;
    }
};

// PMB force (force/CabanaPD_PMB.hpp:89-125, :222-287).
//
// Latency hiding: each bond's work hangs off its neighbour index, which
// streams from HBM; the indices of the next two bonds are loaded two
// iterations ahead (IndexStream), and the kernel is compiled for 4 blocks of
// 256 threads per SM (64 registers). With a warp list the warps take the
// listed chunks of 32 rows (the irregular rows beside the stencil kernel),
// else one thread per row from the first row on.
// Row i's bonds, force boundary condition and step epilogue (the body of
// k_pmb_force_fast and of the batch kernel's PMB rows).
template <bool FRACTURE>
__device__ __forceinline__ void pmb_fast_row(const ParticleView& p, const EllView& nl,
                                             const FastModel& md, const StepEpilogue& ep,
                                             int64_t i)
{
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2v = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const bool nofail_i = FRACTURE ? (p.nofail[i] != 0) : false;
    const int cnt = nl.count[i];
    IndexStream<2> js(nl.idx + i, np, cnt);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    uint32_t word = 0;
    bool dirty = false;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) {
            if (dirty) nl.mu[(int64_t)((k >> 5) - 1) * np + i] = word;
            dirty = false;
            word = nl.mu[(int64_t)(k >> 5) * np + i];
        }
        const int64_t j = js.next(k);
        Gather g;
        gather<FRACTURE>(p, np, j, g);
        Bond b;
        bond_from(g.x0, g.x1, g.x2, g.u0, g.u1, g.u2, xi0, xi1, xi2v, ui0, ui1, ui2, b);
        bool intact = true;
        if (FRACTURE) {
            const uint32_t bit = 1u << (k & 31);
            if (!nofail_i && !g.nofail && critical_fast(b, md.bond_break_coeff)) {
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
            const double kf = md.c * b.s * g.vol * b.rinv;
            fx = fma(kf, b.rx, fx);
            fy = fma(kf, b.ry, fy);
            fz = fma(kf, b.rz, fz);
        }
    }
    if (FRACTURE && dirty && cnt > 0) nl.mu[(int64_t)((cnt - 1) >> 5) * np + i] = word;
    step_epilogue<false>(p, ep, i, fx, fy, fz);
}

template <bool FRACTURE>
__global__ void __launch_bounds__(kBlock, 4)
    k_pmb_force_fast(ParticleView p, EllView nl, FastModel md, StepEpilogue ep,
                     const int32_t* __restrict__ wlist, int64_t wcount)
{
    int64_t i;
    if (wlist) {
        const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        if (slot >= wcount) return;
        i = p.frozen + 32 * (int64_t)wlist[slot] + (threadIdx.x & 31);
    } else {
        i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    }
    if (i >= p.n) return;
    pmb_fast_row<FRACTURE>(p, nl, md, ep, i);
}

// LPS weighted volume and dilatation in ONE pass over the row
// (force/CabanaPD_LPS.hpp:89-141, :287-378): both sums accumulate per bond,
// theta_i = 3 sum(omega s xi^2 vol_j) / m_i at the end (the reference divides
// each term by m_i; the factored division differs by rounding only). With
// WITH_M false, m_i is read (the elastic model computes it once).
template <int INFL, bool FRACTURE, bool WITH_M>
__device__ __forceinline__ void lps_m_theta_row(const ParticleView& p, const EllView& nl,
                                                const FastModel& md, int64_t i)
{
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2v = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const int cnt = nl.count[i];
    IndexStream<2> js(nl.idx + i, np, cnt);
    double mi = WITH_M ? 0.0 : p.m[i];
    double th = 0.0;
    uint32_t word = 0;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) word = nl.mu[(int64_t)(k >> 5) * np + i];
        const int64_t j = js.next(k);
        if (FRACTURE && !((word >> (k & 31)) & 1u)) continue;
        Bond b;
        bond_fast(p.x, p.u, np, j, xi0, xi1, xi2v, ui0, ui1, ui2, b);
        const double vol_j = __ldg(p.vol + j);
        // omega xi^2 (force_models/CabanaPD_LPS.hpp:100-106)
        const double w = INFL == 1 ? b.xi : b.xi * b.xi;
        if (WITH_M) mi = fma(w, vol_j, mi);
        // omega s xi^2 vol_j (force_models/CabanaPD_LPS.hpp:108-116)
        th = fma(w * b.s, vol_j, th);
    }
    if (WITH_M) p.m[i] = mi;
    th = (!FRACTURE || mi > 0) ? 3.0 * th / mi : 0.0;
    p.theta[i] = th;
    p.lps_a[i] = md.theta_coeff * th / mi;
    p.lps_b[i] = md.s_coeff / mi;
}

template <int INFL, bool FRACTURE, bool WITH_M>
__global__ void __launch_bounds__(kBlock, 4)
    k_lps_m_theta_1pass(ParticleView p, EllView nl, FastModel md)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    lps_m_theta_row<INFL, FRACTURE, WITH_M>(p, nl, md, i);
}

// LPS force (force/CabanaPD_LPS.hpp:143-181, :380-447) with the row's
// indices streamed two bonds ahead, compiled for 4 blocks of 256 per SM.
template <int INFL, bool FRACTURE>
__device__ __forceinline__ void lps_force_row(const ParticleView& p, const EllView& nl,
                                              const FastModel& md, const StepEpilogue& ep,
                                              int64_t i)
{
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2v = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const double a_i = p.lps_a[i], b_i = p.lps_b[i];
    const bool nofail_i = FRACTURE ? (p.nofail[i] != 0) : false;
    const int cnt = nl.count[i];
    IndexStream<2> js(nl.idx + i, np, cnt);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    uint32_t word = 0;
    bool dirty = false;
    for (int k = 0; k < cnt; ++k) {
        if (FRACTURE && (k & 31) == 0) {
            if (dirty) nl.mu[(int64_t)((k >> 5) - 1) * np + i] = word;
            dirty = false;
            word = nl.mu[(int64_t)(k >> 5) * np + i];
        }
        const int64_t j = js.next(k);
        Bond b;
        bond_fast(p.x, p.u, np, j, xi0, xi1, xi2v, ui0, ui1, ui2, b);
        bool intact = true;
        if (FRACTURE) {
            // nofail(i) tested twice by the reference (force/CabanaPD_LPS.hpp:417-418).
            const uint32_t bit = 1u << (k & 31);
            if (!nofail_i && critical_fast(b, md.bond_break_coeff)) {
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
            const double a_j = __ldg(p.lps_a + j), b_j = __ldg(p.lps_b + j);
            const double oxi = INFL == 1 ? 1.0 : b.xi;
            const double kf = (a_i + a_j + b.s * (b_i + b_j)) * oxi * __ldg(p.vol + j) * b.rinv;
            fx = fma(kf, b.rx, fx);
            fy = fma(kf, b.ry, fy);
            fz = fma(kf, b.rz, fz);
        }
    }
    if (FRACTURE && dirty && cnt > 0) nl.mu[(int64_t)((cnt - 1) >> 5) * np + i] = word;
    step_epilogue<false>(p, ep, i, fx, fy, fz);
}

template <int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock, 4)
    k_lps_force_pf(ParticleView p, EllView nl, FastModel md, StepEpilogue ep)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    lps_force_row<INFL, FRACTURE>(p, nl, md, ep, i);
}

// Strain energy density and damage at output steps (force/CabanaPD_PMB.hpp:
// 127-155, 289-339; force/CabanaPD_LPS.hpp:183-219, 449-504), for the FP64
// and mixed paths: the per-bond terms and row-order sums of k_pd_energy with
// the bond lengths of bond_fast (correctly rounded square roots from rsqrt
// plus one correction), so W_i agrees with the exact kernel to ~1e-16
// relative per term; broken bonds skip the geometry (their term is zero) but
// count in the damage, which is bit-identical. Block partials of
// (sum W_i vol_i, sum phi_i) in the exact kernel's layout and tree order.
template <bool LPS, int INFL, bool FRACTURE>
__global__ void __launch_bounds__(kBlock)
    k_pd_energy_fast(ParticleView p, EllView nl, FastModel md, double* partials)
{
    __shared__ double s_phi[kBlock];
    __shared__ double s_dmg[kBlock];
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double Phi_i = 0.0, dmg_i = 0.0;
    if (i < p.n) {
        const int64_t np = p.npad;
        const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
        const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
        const int cnt = nl.count[i];
        const double vol_i = p.vol[i];
        double m_i = 0.0, th_i = 0.0;
        if (LPS) {
            m_i = p.m[i];
            th_i = p.theta[i];
        }
        double num_bonds = (double)cnt;
        if (FRACTURE && LPS) {
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
            const bool intact = !FRACTURE || ((word >> (k & 31)) & 1u);
            double w = 0.0;
            if (intact) {
                Bond b;
                bond_fast(p.x, p.u, np, j, xi0, xi1, xi2, ui0, ui1, ui2, b);
                if (LPS) {
                    const double infl = INFL == 1 ? 1.0 / b.xi : 1.0;
                    w = 1.0 / num_bonds * 0.5 * md.theta_coeff / 3.0 * (th_i * th_i) +
                        0.5 * (md.s_coeff / m_i) * infl * b.s * b.s * b.xi * b.xi * vol_j;
                } else {
                    w = 0.25 * md.c * b.s * b.s * b.xi * vol_j;
                }
            }
            if (FRACTURE) {
                Wi += w;
                phi_sum += intact ? vol_j : 0.0;
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

// Batched step over many systems (cpd_batch.cu): persistent blocks take
// tiles grid apart; a tile is up to kBatchTileWarps chunks of 32 rows of one
// instance, whose table entry is staged in shared memory when the block's
// instance changes. Rows run the bodies of the single-system kernels above
// (pass 0: LPS weighted volume when fracture, and dilatation; pass 1: bond
// force and step epilogue) on the instance's current buffer.
__global__ void __launch_bounds__(kBlock, 3)
    k_batch_fast(const BatchInstance* __restrict__ insts, const int32_t* __restrict__ remaining,
                 const BatchTile* __restrict__ tiles, int32_t ntiles, int32_t K, int32_t s,
                 int32_t pass)
{
    static_assert(sizeof(BatchInstance) % 4 == 0 && sizeof(BatchInstance) <= 4 * kBlock,
                  "instance entry staged by one word per thread");
    __shared__ __align__(16) uint32_t dbuf[sizeof(BatchInstance) / 4];
    BatchInstance& d = *reinterpret_cast<BatchInstance*>(dbuf);
    const int w = threadIdx.x >> 5;
    int32_t loaded = -1;
    for (int32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const BatchTile tl = tiles[t];
        if (pass == 0 && !tl.lps) continue;
        const BatchStep bs = batch_step(remaining[tl.inst], K, s);
        if (!bs.run) continue;
        if (tl.inst != loaded) {
            // The instance's entry, with this step's buffers patched in:
            // p.u the current displacement, ep the epilogue of step s.
            __syncthreads();
            const uint32_t* src = reinterpret_cast<const uint32_t*>(insts + tl.inst);
            if (threadIdx.x < sizeof(BatchInstance) / 4) dbuf[threadIdx.x] = src[threadIdx.x];
            __syncthreads();
            if (threadIdx.x == 0) {
                double* const u0 = d.p.u;
                d.p.u = bs.cur ? d.u_alt : u0;
                d.ep.u_next = bs.cur ? u0 : d.u_alt;
                d.ep.mode = bs.mode;
            }
            __syncthreads();
            loaded = tl.inst;
        }
        if (w >= tl.nwarps) continue;
        const int64_t i = d.p.frozen + 32 * (int64_t)(tl.warp0 + w) + (threadIdx.x & 31);
        if (i >= d.p.n) continue;
        const bool infl = d.influence == 1;
        if (pass == 0) {
            if (d.fracture) {
                if (infl) lps_m_theta_row<1, true, true>(d.p, d.nl, d.fm, i);
                else lps_m_theta_row<0, true, true>(d.p, d.nl, d.fm, i);
            } else {
                if (infl) lps_m_theta_row<1, false, false>(d.p, d.nl, d.fm, i);
                else lps_m_theta_row<0, false, false>(d.p, d.nl, d.fm, i);
            }
            continue;
        }
        if (d.pd == CPD_PD_PMB) {
            if (d.fracture) pmb_fast_row<true>(d.p, d.nl, d.fm, d.ep, i);
            else pmb_fast_row<false>(d.p, d.nl, d.fm, d.ep, i);
        } else if (infl) {
            if (d.fracture) lps_force_row<1, true>(d.p, d.nl, d.fm, d.ep, i);
            else lps_force_row<1, false>(d.p, d.nl, d.fm, d.ep, i);
        } else {
            if (d.fracture) lps_force_row<0, true>(d.p, d.nl, d.fm, d.ep, i);
            else lps_force_row<0, false>(d.p, d.nl, d.fm, d.ep, i);
        }
    }
}

}  // namespace

FastModel to_fast(const Model& m)
{
    return FastModel{m.c, m.theta_coeff, m.s_coeff, m.bond_break_coeff};
}

int launch_batch_fast(const BatchInstance* inst, const int32_t* remaining,
                      const BatchTile* tiles, int32_t ntiles, int32_t K, int32_t s,
                      int32_t pass, int grid, cudaStream_t st)
{
    if (ntiles <= 0 || grid <= 0) return 0;
    k_batch_fast<<<grid, kBlock, 0, st>>>(inst, remaining, tiles, ntiles, K, s, pass);
    return 1;
}

int batch_fast_blocks_per_sm()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_fast, kBlock, 0) !=
        cudaSuccess)
        n = 1;
    return n > 0 ? n : 1;
}

bool fast_supported(const Model& md)
{
    return md.pd == CPD_PD_PMB || md.pd == CPD_PD_LPS;
}

int launch_pd_force_fast(const ParticleView& p, const EllView& nl, const Model& md,
                         const StepEpilogue& ep, cudaStream_t st, const int32_t* wlist,
                         int64_t wcount)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0 || (wlist && wcount <= 0)) return 0;
    const int g = wlist ? (int)((wcount + kBlock / 32 - 1) / (kBlock / 32)) : blocks_for(rows);
    const FastModel fm = to_fast(md);
    if (md.pd == CPD_PD_PMB) {
        if (md.fracture)
            k_pmb_force_fast<true><<<g, kBlock, 0, st>>>(p, nl, fm, ep, wlist, wcount);
        else
            k_pmb_force_fast<false><<<g, kBlock, 0, st>>>(p, nl, fm, ep, wlist, wcount);
    } else if (md.influence == 1) {
        if (md.fracture)
            k_lps_force_pf<1, true><<<g, kBlock, 0, st>>>(p, nl, fm, ep);
        else
            k_lps_force_pf<1, false><<<g, kBlock, 0, st>>>(p, nl, fm, ep);
    } else {
        if (md.fracture)
            k_lps_force_pf<0, true><<<g, kBlock, 0, st>>>(p, nl, fm, ep);
        else
            k_lps_force_pf<0, false><<<g, kBlock, 0, st>>>(p, nl, fm, ep);
    }
    return 1;
}

int launch_lps_m_theta_fast(const ParticleView& p, const EllView& nl, const Model& md,
                            bool with_m, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const int g = blocks_for(rows);
    const FastModel fm = to_fast(md);
#define CPD_MT(I, F, W) k_lps_m_theta_1pass<I, F, W><<<g, kBlock, 0, st>>>(p, nl, fm)
    if (md.influence == 1) {
        if (md.fracture) {
            if (with_m) CPD_MT(1, true, true); else CPD_MT(1, true, false);
        } else {
            if (with_m) CPD_MT(1, false, true); else CPD_MT(1, false, false);
        }
    } else {
        if (md.fracture) {
            if (with_m) CPD_MT(0, true, true); else CPD_MT(0, true, false);
        } else {
            if (with_m) CPD_MT(0, false, true); else CPD_MT(0, false, false);
        }
    }
#undef CPD_MT
    return 1;
}

int launch_pd_energy_fast(const ParticleView& p, const EllView& nl, const Model& md,
                          double* partials, int nblocks, cudaStream_t st)
{
    const FastModel fm = to_fast(md);
    const bool infl = md.influence == 1;
    if (md.pd == CPD_PD_PMB) {
        if (md.fracture)
            k_pd_energy_fast<false, 0, true><<<nblocks, kBlock, 0, st>>>(p, nl, fm, partials);
        else
            k_pd_energy_fast<false, 0, false><<<nblocks, kBlock, 0, st>>>(p, nl, fm, partials);
    } else if (md.pd == CPD_PD_LPS) {
        if (md.fracture) {
            if (infl)
                k_pd_energy_fast<true, 1, true><<<nblocks, kBlock, 0, st>>>(p, nl, fm, partials);
            else
                k_pd_energy_fast<true, 0, true><<<nblocks, kBlock, 0, st>>>(p, nl, fm, partials);
        } else {
            if (infl)
                k_pd_energy_fast<true, 1, false><<<nblocks, kBlock, 0, st>>>(p, nl, fm, partials);
            else
                k_pd_energy_fast<true, 0, false><<<nblocks, kBlock, 0, st>>>(p, nl, fm, partials);
        }
    } else {
        return -1;
    }
    return 1;
}

}  // namespace cpd
