// Mixed-precision PMB bond kernel and its supporting passes.
//
// Arithmetic split (what stays FP64 and what goes FP32):
//   FP64  positions, displacements and velocities (integration), the
//         energy / damage reductions, and the break re-test of any bond whose
//         FP32 stretch lies within 1e-4 s0 of s0 (the reference's exact
//         expression on FP64 data), so broken-bond sets match the FP64 path.
//   FP32  bond reference vectors (precomputed once in FP64, stored as FP32),
//         displacement differences, stretch, pairwise force; per-particle
//         force sums with Kahan compensation, converted to FP64 at the end.
//
// Bond reference vectors. On a lattice every bond is one of a few dozen
// offsets (a hx, b hy, c hz). Each bond slot stores a 1-byte code: codes
// below kGeneric index a table (FP32 xi_vec, xi, 1/xi, and the index delta
// j - i, identical for all bonds with that code on an x-fastest lattice),
// kept in shared memory; kGeneric bonds read the 32-bit neighbour index and
// rebuild xi_vec from positions split into FP32 hi + lo parts. The per-bond
// stream is 1 byte (+ the bond bit) instead of 4, and lattice bonds need no
// position gather.
//
// Stencil rows. The table is built in ascending index-delta order, which is
// the sorted row order, so a lattice particle's row is a subset of the table
// in table order (the whole table in the interior). Such rows keep a
// presence bitmask over the table (16 B per particle); a warp whose rows are
// all stencil rows walks the table itself, reading entry k at a warp-uniform
// address and loading no per-bond code. Only warps holding an irregular row
// use the per-bond codes.
//
// Displacements are split the same way (u = hi + lo, both FP32, refreshed
// by the integrator), so eta = u_j - u_i keeps ~1e-7 relative accuracy even
// under large rigid motion. The stretch is formed without cancellation:
//   s = (r - xi) / xi = eta . (2 xi_vec + eta) / (xi (r + xi)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "cpd_internal.cuh"

namespace cpd {
namespace {

constexpr int kBlock = 256;
inline int blocks_for(int64_t rows) { return (int)((rows + kBlock - 1) / kBlock); }

__device__ __noinline__ bool critical_exact64(const double* __restrict__ x,
                                              const double* __restrict__ u, int64_t np,
                                              int64_t i, int64_t j, double bbc)
{
    // CabanaPD_Force.hpp:74-93 + CabanaPD_ForceModels.hpp:123-128, every
    // operation separately rounded.
    const double xx = __dsub_rn(x[j], x[i]);
    const double xy = __dsub_rn(x[np + j], x[np + i]);
    const double xz = __dsub_rn(x[2 * np + j], x[2 * np + i]);
    const double rx = __dadd_rn(xx, __dsub_rn(u[j], u[i]));
    const double ry = __dadd_rn(xy, __dsub_rn(u[np + j], u[np + i]));
    const double rz = __dadd_rn(xz, __dsub_rn(u[2 * np + j], u[2 * np + i]));
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)),
                                __dmul_rn(rz, rz));
    const double x2 = __dadd_rn(__dadd_rn(__dmul_rn(xx, xx), __dmul_rn(xy, xy)),
                                __dmul_rn(xz, xz));
    const double r = __dsqrt_rn(r2);
    const double xi = __dsqrt_rn(x2);
    return __dmul_rn(r, r) >= __dmul_rn(__dmul_rn(bbc, xi), xi);
}

// ---------------------------------------------------------------------------
// Stencil coding.

// Smallest positive |x_j - x_i| per axis over all bonds (the lattice
// spacing on a lattice; tiny on an irregular cloud, which then codes every
// bond as generic). Positive doubles order like their bit patterns.
__global__ void __launch_bounds__(kBlock)
    k_min_spacing(ParticleView p, EllView nl, unsigned long long* out)
{
    __shared__ unsigned long long s[3][kBlock];
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double m[3] = {INFINITY, INFINITY, INFINITY};
    if (i < p.n) {
        const int64_t np = p.npad;
        const int cnt = nl.count[i];
        for (int k = 0; k < cnt; ++k) {
            const int64_t j = nl.idx[(int64_t)k * np + i];
            for (int d = 0; d < 3; ++d) {
                const double a = fabs(p.x[d * np + j] - p.x[d * np + i]);
                if (a > 0.0) m[d] = fmin(m[d], a);
            }
        }
    }
    for (int d = 0; d < 3; ++d) s[d][threadIdx.x] = __double_as_longlong(m[d]);
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int d = 0; d < 3; ++d)
                s[d][threadIdx.x] = min(s[d][threadIdx.x], s[d][threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) atomicMin(out + d, s[d][0]);
}

struct LatticeLut {
    double h[3];
    int32_t half[3];  // offsets -half..half per axis
    const int16_t* lut;  // [(2 half_x + 1)(2 half_y + 1)(2 half_z + 1)] -> code or -1
};

__global__ void __launch_bounds__(kBlock)
    k_code_bonds(ParticleView p, EllView nl, LatticeLut L, uint8_t* code,
                 unsigned long long* delta)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const int cnt = nl.count[i];
    const int nx = 2 * L.half[0] + 1, ny = 2 * L.half[1] + 1;
    for (int k = 0; k < cnt; ++k) {
        const int64_t j = nl.idx[(int64_t)k * np + i];
        int c = kMixedGeneric;
        int o[3];
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
            const double dd = p.x[d * np + j] - p.x[d * np + i];
            const double a = rint(dd / L.h[d]);
            if (fabs(dd - a * L.h[d]) > 1e-6 * L.h[d] || fabs(a) > L.half[d]) ok = false;
            o[d] = (int)a;
        }
        if (ok) {
            const int e = L.lut[(o[0] + L.half[0]) + nx * ((o[1] + L.half[1]) + ny * (o[2] + L.half[2]))];
            if (e >= 0) {
                c = e;
                // The code's index delta: the smallest j - i among its bonds
                // (deterministic; on an x-fastest lattice all are equal).
                // Stored biased by 2^62 so signed order survives the
                // unsigned atomic.
                atomicMin(delta + c, (unsigned long long)((long long)(j - i) + (1LL << 62)));
            }
        }
        code[(int64_t)k * np + i] = (uint8_t)c;
    }
}

__global__ void __launch_bounds__(kBlock)
    k_verify_delta(ParticleView p, EllView nl, const unsigned long long* delta, uint8_t* code)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const int cnt = nl.count[i];
    for (int k = 0; k < cnt; ++k) {
        const int64_t o = (int64_t)k * np + i;
        const int c = code[o];
        if (c == kMixedGeneric) continue;
        const int64_t j = nl.idx[o];
        if ((long long)delta[c] - (1LL << 62) != (long long)(j - i)) code[o] = (uint8_t)kMixedGeneric;
    }
}

// Per row: presence bits of the stencil entries it holds (its codes are a
// strictly increasing subset of the table); per warp: 2 if every row is the
// whole table, 1 if every row is a table subset, else 0.
__global__ void __launch_bounds__(kBlock)
    k_row_masks(ParticleView p, EllView nl, const uint8_t* code, int ntab, uint32_t* pmask,
                uint8_t* kind)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nmask = (ntab + 31) / 32;
    bool subset = i < p.n;
    bool full = subset;
    if (subset) {
        const int64_t np = p.npad;
        const int cnt = nl.count[i];
        full = cnt == ntab;
        uint32_t m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int prev = -1;
        for (int k = 0; k < cnt; ++k) {
            const int c = code[(int64_t)k * np + i];
            if (c >= ntab || c <= prev) {
                subset = false;
                break;
            }
            if (c != k) full = false;
            m[c >> 5] |= 1u << (c & 31);
            prev = c;
        }
        if (!subset) full = false;
        for (int w = 0; w < nmask; ++w) pmask[(int64_t)w * np + i] = subset ? m[w] : 0u;
    }
    full = __all_sync(0xffffffffu, full);
    subset = __all_sync(0xffffffffu, subset);
    if ((threadIdx.x & 31) == 0)
        kind[((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5] = full ? 2 : (subset ? 1 : 0);
}

// FP64 SoA -> FP32 hi/lo float4 (w carries an extra scalar per array).
__global__ void __launch_bounds__(kBlock)
    k_split(const double* __restrict__ src, int64_t n, int64_t np, const double* w_hi,
            const uint8_t* w_lo, float4* hi, float4* lo)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float h[3], l[3];
    for (int d = 0; d < 3; ++d) {
        const double v = src[d * np + i];
        h[d] = __double2float_rn(v);
        l[d] = __double2float_rn(v - (double)h[d]);
    }
    hi[i] = make_float4(h[0], h[1], h[2], w_hi ? __double2float_rn(w_hi[i]) : 0.f);
    lo[i] = make_float4(l[0], l[1], l[2], w_lo ? (float)w_lo[i] : 0.f);
}

// Velocity Verlet first half (CabanaPD_Integrate.hpp:89-116) that also
// refreshes the FP32 hi/lo copy of u with vol (w of hi) and nofail (w of lo).
__global__ void __launch_bounds__(kBlock)
    k_vv_initial_mixed(ParticleView p, double dt, double half_dt, float4* uh, float4* ul)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double half_dt_m = half_dt / p.rho[i];
    float h[3], l[3];
    for (int d = 0; d < 3; ++d) {
        const double v = p.v[d * np + i] + half_dt_m * p.f[d * np + i];
        p.v[d * np + i] = v;
        const double u = p.u[d * np + i] + dt * v;
        p.u[d * np + i] = u;
        h[d] = __double2float_rn(u);
        l[d] = __double2float_rn(u - (double)h[d]);
    }
    uh[i] = make_float4(h[0], h[1], h[2], __double2float_rn(p.vol[i]));
    ul[i] = make_float4(l[0], l[1], l[2], (float)p.nofail[i]);
}

struct MixedModel {
    float c, s0, guard;
    double bbc;
    int ntab;
};

// Kahan-compensated accumulation of one FP32 term.
__device__ __forceinline__ void kahan_add(float& sum, float& comp, float term)
{
    const float y = term - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// PMB force, mixed precision (force/CabanaPD_PMB.hpp:89-125, :222-287).
// Bonds are walked one 32-bond mask word at a time (the word is loaded,
// tested bit by bit and written back once); stencil codes stream two bonds
// ahead. MINB is the occupancy target passed to __launch_bounds__.
template <bool FRACTURE, int MINB, bool PIPE>
__global__ void __launch_bounds__(kBlock, MINB)
    k_pmb_force_mixed(ParticleView p, EllView nl, MixedView mv, MixedModel md)
{
    __shared__ MixedStencil tab[kMixedGeneric];
    for (int t = threadIdx.x; t < md.ntab; t += blockDim.x) tab[t] = mv.table[t];
    __syncthreads();
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const float4 uhi = mv.uh[i], uli = mv.ul[i];
    const bool nofail_i = FRACTURE ? (uli.w != 0.f) : false;
    const int cnt = nl.count[i];
    const uint8_t* __restrict__ code = mv.code + i;
    const float4* __restrict__ UH = mv.uh;
    const float4* __restrict__ UL = mv.ul;
    float sx = 0.f, sy = 0.f, sz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    const int kind = mv.warp_kind[((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5];
    if (kind == 2 && PIPE) {
        // Full-stencil warp, software-pipelined: the next entry's table row
        // and neighbour data are loaded before the current bond is computed.
        const float4* __restrict__ uh_i = UH + i;
        const float4* __restrict__ ul_i = UL + i;
        MixedStencil tn = tab[0];
        float4 uhn = uh_i[tn.delta], uln = ul_i[tn.delta];
        for (int base = 0; base < cnt; base += 32) {
            uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
            const uint32_t old = word;
            const int lim = min(32, cnt - base);
            for (int b = 0; b < lim; ++b) {
                const int k = base + b;
                const MixedStencil t = tn;
                const float4 uhj = uhn, ulj = uln;
                if (k + 1 < cnt) {
                    tn = tab[k + 1];
                    uhn = uh_i[tn.delta];
                    uln = ul_i[tn.delta];
                }
                const float nx = (uhj.x - uhi.x) + (ulj.x - uli.x);
                const float ny = (uhj.y - uhi.y) + (ulj.y - uli.y);
                const float nz = (uhj.z - uhi.z) + (ulj.z - uli.z);
                const float rx = t.x + nx, ry = t.y + ny, rz = t.z + nz;
                const float r2 = rx * rx + ry * ry + rz * rz;
                const float rinv = rsqrtf(r2);
                const float r = r2 * rinv;
                const float num = nx * (2.f * t.x + nx) + ny * (2.f * t.y + ny) + nz * (2.f * t.z + nz);
                const float s = __fdividef(num * t.xiinv, r + t.xi);
                bool intact = true;
                if (FRACTURE) {
                    bool crit = false;
                    if (!nofail_i && ulj.w == 0.f) {
                        if (fabsf(s - md.s0) <= md.guard)
                            crit = critical_exact64(p.x, p.u, np, i, i + t.delta, md.bbc);
                        else
                            crit = s >= md.s0;
                    }
                    if (crit) word &= ~(1u << b);
                    intact = (word >> b) & 1u;
                }
                if (intact) {
                    const float kf = md.c * uhj.w * s * rinv;
                    kahan_add(sx, cx, kf * rx);
                    kahan_add(sy, cy, kf * ry);
                    kahan_add(sz, cz, kf * rz);
                }
            }
            if (FRACTURE && word != old) nl.mu[(int64_t)(base >> 5) * np + i] = word;
        }
        p.f[i] = (double)sx - (double)cx;
        p.f[np + i] = (double)sy - (double)cy;
        p.f[2 * np + i] = (double)sz - (double)cz;
        return;
    }
    if (kind != 0) {
        // Stencil rows: bond slots are the row's table entries in table
        // order, so entry k is read at a warp-uniform address. Full rows
        // (kind 2) hold every entry; subset rows skip the absent ones.
        const float4* __restrict__ uh_i = UH + i;
        const float4* __restrict__ ul_i = UL + i;
        const int nmask = (md.ntab + 31) / 32;
        int slot = 0, cur_w = 0;
        uint32_t word = FRACTURE ? nl.mu[i] : 0xffffffffu;
        uint32_t old = word;
        for (int w = 0; w < nmask; ++w) {
            const uint32_t pm = kind == 2 ? 0xffffffffu : mv.pmask[(int64_t)w * np + i];
            const int kend = min(32, md.ntab - 32 * w);
            for (int b = 0; b < kend; ++b) {
                if (!((pm >> b) & 1u)) continue;
                if (FRACTURE && (slot >> 5) != cur_w) {
                    if (word != old) nl.mu[(int64_t)cur_w * np + i] = word;
                    cur_w = slot >> 5;
                    word = nl.mu[(int64_t)cur_w * np + i];
                    old = word;
                }
                const int sb = slot & 31;
                ++slot;
                const MixedStencil t = tab[32 * w + b];
                const float4 uhj = uh_i[t.delta], ulj = ul_i[t.delta];
                const float nx = (uhj.x - uhi.x) + (ulj.x - uli.x);
                const float ny = (uhj.y - uhi.y) + (ulj.y - uli.y);
                const float nz = (uhj.z - uhi.z) + (ulj.z - uli.z);
                const float rx = t.x + nx, ry = t.y + ny, rz = t.z + nz;
                const float r2 = rx * rx + ry * ry + rz * rz;
                const float rinv = rsqrtf(r2);
                const float r = r2 * rinv;
                const float num = nx * (2.f * t.x + nx) + ny * (2.f * t.y + ny) + nz * (2.f * t.z + nz);
                const float s = __fdividef(num * t.xiinv, r + t.xi);
                bool intact = true;
                if (FRACTURE) {
                    bool crit = false;
                    if (!nofail_i && ulj.w == 0.f) {
                        if (fabsf(s - md.s0) <= md.guard)
                            crit = critical_exact64(p.x, p.u, np, i, i + t.delta, md.bbc);
                        else
                            crit = s >= md.s0;
                    }
                    if (crit) word &= ~(1u << sb);
                    intact = (word >> sb) & 1u;
                }
                if (intact) {
                    const float kf = md.c * uhj.w * s * rinv;
                    kahan_add(sx, cx, kf * rx);
                    kahan_add(sy, cy, kf * ry);
                    kahan_add(sz, cz, kf * rz);
                }
            }
        }
        if (FRACTURE && word != old) nl.mu[(int64_t)cur_w * np + i] = word;
        p.f[i] = (double)sx - (double)cx;
        p.f[np + i] = (double)sy - (double)cy;
        p.f[2 * np + i] = (double)sz - (double)cz;
        return;
    }
    int c1 = cnt > 0 ? __ldg(code) : 0;
    int c2 = cnt > 1 ? __ldg(code + np) : 0;
    for (int base = 0; base < cnt; base += 32) {
        uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
        const uint32_t old = word;
        const int lim = min(32, cnt - base);
        for (int b = 0; b < lim; ++b) {
            const int k = base + b;
            const int c = c1;
            c1 = c2;
            c2 = (k + 2 < cnt) ? __ldg(code + (int64_t)(k + 2) * np) : 0;
            float ex, ey, ez, xi, xiinv;
            int64_t j;
            if (c != kMixedGeneric) {
                const MixedStencil t = tab[c];
                ex = t.x;
                ey = t.y;
                ez = t.z;
                xi = t.xi;
                xiinv = t.xiinv;
                j = i + t.delta;
            } else {
                j = __ldg(nl.idx + (int64_t)k * np + i);
                const float4 xhj = mv.xh[j], xlj = mv.xl[j];
                const float4 xhi = mv.xh[i], xli = mv.xl[i];
                ex = (xhj.x - xhi.x) + (xlj.x - xli.x);
                ey = (xhj.y - xhi.y) + (xlj.y - xli.y);
                ez = (xhj.z - xhi.z) + (xlj.z - xli.z);
                const float x2 = ex * ex + ey * ey + ez * ez;
                xiinv = rsqrtf(x2);
                xi = x2 * xiinv;
            }
            const float4 uhj = UH[j], ulj = UL[j];
            const float nx = (uhj.x - uhi.x) + (ulj.x - uli.x);
            const float ny = (uhj.y - uhi.y) + (ulj.y - uli.y);
            const float nz = (uhj.z - uhi.z) + (ulj.z - uli.z);
            const float rx = ex + nx, ry = ey + ny, rz = ez + nz;
            const float r2 = rx * rx + ry * ry + rz * rz;
            const float rinv = rsqrtf(r2);
            const float r = r2 * rinv;
            // eta . (2 xi_vec + eta) = r^2 - xi^2 without cancellation.
            const float num = nx * (2.f * ex + nx) + ny * (2.f * ey + ny) + nz * (2.f * ez + nz);
            const float s = __fdividef(num * xiinv, r + xi);
            bool intact = true;
            if (FRACTURE) {
                bool crit = false;
                if (!nofail_i && ulj.w == 0.f) {
                    if (fabsf(s - md.s0) <= md.guard)
                        crit = critical_exact64(p.x, p.u, np, i, j, md.bbc);
                    else
                        crit = s >= md.s0;
                }
                if (crit) word &= ~(1u << b);
                intact = (word >> b) & 1u;
            }
            if (intact) {
                const float kf = md.c * uhj.w * s * rinv;
                kahan_add(sx, cx, kf * rx);
                kahan_add(sy, cy, kf * ry);
                kahan_add(sz, cz, kf * rz);
            }
        }
        if (FRACTURE && word != old) nl.mu[(int64_t)(base >> 5) * np + i] = word;
    }
    p.f[i] = (double)sx - (double)cx;
    p.f[np + i] = (double)sy - (double)cy;
    p.f[2 * np + i] = (double)sz - (double)cz;
}

// Mixed-kernel variant, from CPD_MIXED_VARIANT: 0 -> 4 blocks of 256 per SM
// (64 registers), 1 -> 4 blocks with the full-stencil loop software
// pipelined, 2 -> pipelined with 3 blocks (more registers). Full plate on
// B200, ms per launch: 4.70 / 4.64 / 4.92; 0 is the default (no spills).
int mixed_variant()
{
    static int v = [] {
        const char* e = getenv("CPD_MIXED_VARIANT");
        int x = e ? atoi(e) : 0;
        return (x < 0 || x > 2) ? 0 : x;
    }();
    return v;
}

#define CPD_TRY(call)                                                     \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) {                                          \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
            return -1;                                                    \
        }                                                                 \
    } while (0)

}  // namespace

void free_mixed(MixedState& m, cudaStream_t st)
{
    void* ptrs[] = {m.xh, m.xl, m.uh, m.ul, m.code, m.table, m.warp_kind, m.pmask};
    for (void* q : ptrs)
        if (q) dev_free(q, st);
    m = MixedState{};
}

int prepare_mixed(const ParticleView& p, const NeighborList& pd, double cutoff,
                  MixedState& m, cudaStream_t st, std::string& err)
{
    int launches = 0;
    free_mixed(m, st);
    const int64_t np = p.npad;
    CPD_TRY(dev_alloc(&m.xh, sizeof(float4) * np, st));
    CPD_TRY(dev_alloc(&m.xl, sizeof(float4) * np, st));
    CPD_TRY(dev_alloc(&m.uh, sizeof(float4) * np, st));
    CPD_TRY(dev_alloc(&m.ul, sizeof(float4) * np, st));
    CPD_TRY(dev_alloc(&m.table, sizeof(MixedStencil) * kMixedGeneric, st));
    CPD_TRY(dev_alloc(&m.code, (size_t)std::max(pd.max_n, 1) * np, st));
    const int64_t nwarps = (np + 31) / 32 + 8;
    CPD_TRY(dev_alloc(&m.warp_kind, nwarps, st));
    m.bytes = 4 * sizeof(float4) * np + sizeof(MixedStencil) * kMixedGeneric +
              (size_t)std::max(pd.max_n, 1) * np + nwarps;
    CPD_TRY(cudaMemsetAsync(m.warp_kind, 0, nwarps, st));
    CPD_TRY(cudaMemsetAsync(m.code, kMixedGeneric, (size_t)std::max(pd.max_n, 1) * np, st));
    k_split<<<blocks_for(p.n), kBlock, 0, st>>>(p.x, p.n, np, nullptr, nullptr, m.xh, m.xl);
    launches++;
    m.ntab = 0;
    const int64_t rows = p.n - p.frozen;
    if (rows > 0 && pd.max_n > 0) {
        unsigned long long* d_min = nullptr;
        CPD_TRY(dev_alloc(&d_min, 3 * sizeof(unsigned long long), st));
        CPD_TRY(cudaMemsetAsync(d_min, 0x7f, 3 * sizeof(unsigned long long), st));
        k_min_spacing<<<blocks_for(rows), kBlock, 0, st>>>(p, pd.view(), d_min);
        launches++;
        unsigned long long hmin[3];
        CPD_TRY(cudaMemcpyAsync(hmin, d_min, sizeof(hmin), cudaMemcpyDeviceToHost, st));
        CPD_TRY(cudaStreamSynchronize(st));
        CPD_TRY(dev_free(d_min, st));
        double h[3];
        bool lattice = true;
        for (int d = 0; d < 3; ++d) {
            std::memcpy(&h[d], &hmin[d], sizeof(double));
            if (!(h[d] > 1e-6 * cutoff) || !std::isfinite(h[d])) lattice = false;
        }
        if (lattice) {
            // Table of lattice offsets within the cutoff (code order: z, y, x).
            int half[3];
            for (int d = 0; d < 3; ++d) half[d] = (int)std::floor(cutoff / h[d] + 1e-9);
            const int nx = 2 * half[0] + 1, ny = 2 * half[1] + 1, nz = 2 * half[2] + 1;
            std::vector<int16_t> lut((size_t)nx * ny * nz, -1);
            std::vector<MixedStencil> tab;
            for (int c = -half[2]; c <= half[2]; ++c)
                for (int b = -half[1]; b <= half[1]; ++b)
                    for (int a = -half[0]; a <= half[0]; ++a) {
                        if (a == 0 && b == 0 && c == 0) continue;
                        const double vx = a * h[0], vy = b * h[1], vz = c * h[2];
                        const double len = std::sqrt(vx * vx + vy * vy + vz * vz);
                        if (len > cutoff * (1.0 + 1e-9)) continue;
                        if ((int)tab.size() >= kMixedGeneric) {
                            lattice = false;
                            break;
                        }
                        lut[(a + half[0]) + nx * ((b + half[1]) + ny * (c + half[2]))] =
                            (int16_t)tab.size();
                        MixedStencil e;
                        e.x = (float)vx;
                        e.y = (float)vy;
                        e.z = (float)vz;
                        e.xi = (float)len;
                        e.xiinv = (float)(1.0 / len);
                        e.delta = 0;
                        tab.push_back(e);
                    }
            if (lattice && !tab.empty()) {
                int16_t* d_lut = nullptr;
                unsigned long long* d_delta = nullptr;
                CPD_TRY(dev_alloc(&d_lut, sizeof(int16_t) * lut.size(), st));
                CPD_TRY(dev_alloc(&d_delta, sizeof(unsigned long long) * kMixedGeneric, st));
                CPD_TRY(cudaMemcpyAsync(d_lut, lut.data(), sizeof(int16_t) * lut.size(),
                                        cudaMemcpyHostToDevice, st));
                CPD_TRY(cudaMemsetAsync(d_delta, 0xff, sizeof(unsigned long long) * kMixedGeneric, st));
                LatticeLut L;
                for (int d = 0; d < 3; ++d) {
                    L.h[d] = h[d];
                    L.half[d] = half[d];
                }
                L.lut = d_lut;
                k_code_bonds<<<blocks_for(rows), kBlock, 0, st>>>(p, pd.view(), L, m.code, d_delta);
                k_verify_delta<<<blocks_for(rows), kBlock, 0, st>>>(p, pd.view(), d_delta, m.code);
                launches += 2;
                std::vector<unsigned long long> delta(kMixedGeneric);
                CPD_TRY(cudaMemcpyAsync(delta.data(), d_delta,
                                        sizeof(unsigned long long) * kMixedGeneric,
                                        cudaMemcpyDeviceToHost, st));
                CPD_TRY(cudaStreamSynchronize(st));
                for (size_t t = 0; t < tab.size(); ++t)
                    tab[t].delta = (int32_t)((long long)delta[t] - (1LL << 62));
                CPD_TRY(cudaMemcpyAsync(m.table, tab.data(), sizeof(MixedStencil) * tab.size(),
                                        cudaMemcpyHostToDevice, st));
                CPD_TRY(cudaStreamSynchronize(st));
                CPD_TRY(dev_free(d_lut, st));
                CPD_TRY(dev_free(d_delta, st));
                m.ntab = (int)tab.size();
                for (int d = 0; d < 3; ++d) m.h[d] = h[d];
                const int nmask = (m.ntab + 31) / 32;
                CPD_TRY(dev_alloc(&m.pmask, sizeof(uint32_t) * nmask * np, st));
                m.bytes += sizeof(uint32_t) * nmask * np;
                k_row_masks<<<blocks_for(rows), kBlock, 0, st>>>(p, pd.view(), m.code, m.ntab,
                                                                 m.pmask, m.warp_kind);
                launches++;
            }
        }
    }
    CPD_TRY(cudaGetLastError());
    return launches;
}

int launch_split_u(const ParticleView& p, MixedState& m, cudaStream_t st)
{
    if (p.n <= 0) return 0;
    k_split<<<blocks_for(p.n), kBlock, 0, st>>>(p.u, p.n, p.npad, p.vol, p.nofail, m.uh, m.ul);
    return 1;
}

int launch_vv_initial_mixed(const ParticleView& p, double dt, MixedState& m, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    k_vv_initial_mixed<<<blocks_for(rows), kBlock, 0, st>>>(p, dt, 0.5 * dt, m.uh, m.ul);
    return 1;
}

int launch_pd_force_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                          const MixedState& m, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    MixedView mv{m.xh, m.xl, m.uh, m.ul, m.code, m.table, m.warp_kind, m.pmask};
    MixedModel mm;
    mm.c = (float)md.c;
    mm.s0 = (float)md.s0;
    mm.guard = (float)(1e-4 * md.s0);
    mm.bbc = md.bond_break_coeff;
    mm.ntab = m.ntab;
    const int g = blocks_for(rows);
    switch ((md.fracture ? 0 : 10) + mixed_variant()) {
    case 0: k_pmb_force_mixed<true, 4, false><<<g, kBlock, 0, st>>>(p, nl, mv, mm); break;
    case 1: k_pmb_force_mixed<true, 4, true><<<g, kBlock, 0, st>>>(p, nl, mv, mm); break;
    case 2: k_pmb_force_mixed<true, 3, true><<<g, kBlock, 0, st>>>(p, nl, mv, mm); break;
    case 10: k_pmb_force_mixed<false, 4, false><<<g, kBlock, 0, st>>>(p, nl, mv, mm); break;
    case 11: k_pmb_force_mixed<false, 4, true><<<g, kBlock, 0, st>>>(p, nl, mv, mm); break;
    default: k_pmb_force_mixed<false, 3, true><<<g, kBlock, 0, st>>>(p, nl, mv, mm); break;
    }
    return 1;
}

}  // namespace cpd
