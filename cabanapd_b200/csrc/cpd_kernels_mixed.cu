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

#include "cpd_epilogue.cuh"
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
// Sets *differs when some particle's volume differs from particle 0's.
__global__ void __launch_bounds__(kBlock)
    k_vol_uniform(const double* __restrict__ vol, int64_t n, unsigned long long* differs)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && vol[i] != vol[0]) atomicOr(differs, 1ull);
}

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

// Slots of the per-entry delta arrays (byte codes and the wide FP64 table).
constexpr int kDeltaSlots = kStencilMaxWide > kMixedGeneric ? kStencilMaxWide : kMixedGeneric;

struct LatticeLut {
    double h[3];
    double hinv[3];  // 1 / h
    int32_t half[3];  // offsets -half..half per axis
    const int16_t* lut;  // [(2 half_x + 1)(2 half_y + 1)(2 half_z + 1)] -> code or -1
};

// Codes every bond and records, per code, the smallest index delta j - i
// among its bonds (deterministic; on an x-fastest lattice all are equal),
// biased by 2^31 so signed order survives the unsigned minimum. The minimum
// is reduced in the warp (lanes holding the same code), then per block in
// shared memory, and a block updates the global value only to lower it.
__global__ void __launch_bounds__(kBlock)
    k_code_bonds(ParticleView p, EllView nl, LatticeLut L, uint8_t* code, unsigned int* delta)
{
    __shared__ unsigned int s_min[kMixedGeneric];
    for (int t = threadIdx.x; t < kMixedGeneric; t += blockDim.x) s_min[t] = 0xffffffffu;
    __syncthreads();
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool row = i < p.n;
    const int64_t np = p.npad;
    const int cnt = row ? nl.count[i] : 0;
    const int kmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    const int nx = 2 * L.half[0] + 1, ny = 2 * L.half[1] + 1;
    for (int k = 0; k < kmax; ++k) {
        int c = kMixedGeneric;
        unsigned int v = 0xffffffffu;
        if (k < cnt) {
            const int64_t j = nl.idx[(int64_t)k * np + i];
            int o[3];
            bool ok = true;
            for (int d = 0; d < 3; ++d) {
                const double dd = p.x[d * np + j] - p.x[d * np + i];
                const double a = rint(dd * L.hinv[d]);
                if (fabs(dd - a * L.h[d]) > 1e-6 * L.h[d] || fabs(a) > L.half[d]) ok = false;
                o[d] = (int)a;
            }
            if (ok) {
                const int e = L.lut[(o[0] + L.half[0]) +
                                    nx * ((o[1] + L.half[1]) + ny * (o[2] + L.half[2]))];
                if (e >= 0) {
                    c = e;
                    v = (unsigned int)((long long)(j - i) + (1LL << 31));
                }
            }
            code[(int64_t)k * np + i] = (uint8_t)c;
        }
        // Every lane of the warp takes part (inactive and generic lanes with
        // the generic code, which records nothing).
        const unsigned int grp = __match_any_sync(0xffffffffu, c);
        const unsigned int m = __reduce_min_sync(grp, v);
        if (c != kMixedGeneric && (int)(threadIdx.x & 31) == __ffs(grp) - 1) atomicMin(&s_min[c], m);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < kMixedGeneric; t += blockDim.x) {
        const unsigned int m = s_min[t];
        if (m != 0xffffffffu && m < *(volatile unsigned int*)(delta + t)) atomicMin(delta + t, m);
    }
}

// Sample rows for the index deltas: row r_s = lo + (2 s + 1) span / (2 S) of
// each block s writes its bonds' codes and index deltas (code kMixedGeneric
// past its count) at out[s][k], k < max_n.
__global__ void k_sample_rows(EllView nl, int64_t np, const uint8_t* __restrict__ code,
                              int64_t lo, int64_t span, int nsamples, int2* out)
{
    const int s = blockIdx.x;
    const int64_t r = lo + ((2 * (int64_t)s + 1) * span) / (2 * (int64_t)nsamples);
    const int cnt = nl.count[r];
    for (int k = threadIdx.x; k < nl.max_n; k += blockDim.x) {
        int2 v = make_int2(kMixedGeneric, 0);
        if (k < cnt) {
            v.x = code[(int64_t)k * np + r];
            v.y = (int)(nl.idx[(int64_t)k * np + r] - r);
        }
        out[(int64_t)s * nl.max_n + k] = v;
    }
}

// Order-preserving unsigned image of a double (for atomicMin / atomicMax).
__device__ __forceinline__ unsigned long long ordered_bits(double v)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// Per axis the smallest and largest position of rows [0, n) (ordered_bits:
// out[0..2] minima, out[3..5] maxima; grid-stride rows, one atomic per block
// and value).
__global__ void __launch_bounds__(kBlock)
    k_bounds(const double* __restrict__ x, int64_t n, int64_t np, unsigned long long* out)
{
    __shared__ unsigned long long s[6][kBlock];
    unsigned long long lo[3] = {~0ull, ~0ull, ~0ull}, hi[3] = {0ull, 0ull, 0ull};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        for (int d = 0; d < 3; ++d) {
            const unsigned long long b = ordered_bits(x[d * np + i]);
            lo[d] = b < lo[d] ? b : lo[d];
            hi[d] = b > hi[d] ? b : hi[d];
        }
    for (int d = 0; d < 3; ++d) {
        s[d][threadIdx.x] = lo[d];
        s[3 + d][threadIdx.x] = hi[d];
    }
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int d = 0; d < 3; ++d) {
                s[d][threadIdx.x] = min(s[d][threadIdx.x], s[d][threadIdx.x + w]);
                s[3 + d][threadIdx.x] = max(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) {
            atomicMin(out + d, s[d][0]);
            atomicMax(out + 3 + d, s[3 + d][0]);
        }
}

// Lattice cell of every row [0, n): cell = a + nc0 (b + nc1 c) from
// (x - x0) / h rounded per axis. flags[0] counts positions more than 1e-6
// spacings off the lattice, flags[1] cells taken twice; ext[0] / ext[1] are
// the smallest and largest cell - row (biased by 2^62).
__global__ void __launch_bounds__(kBlock)
    k_lattice_cells(const double* __restrict__ x, int64_t n, int64_t np, double3 x0,
                    double3 hinv, int3 nc, int32_t* __restrict__ cell,
                    uint32_t* __restrict__ occ, unsigned int* flags, unsigned long long* ext)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // Every lane reaches the warp's min / max below (one atomic per warp).
    unsigned long long lo = ~0ull, hi = 0ull;
    if (i < n) {
        const double t[3] = {(x[i] - x0.x) * hinv.x, (x[np + i] - x0.y) * hinv.y,
                             (x[2 * np + i] - x0.z) * hinv.z};
        const int ncs[3] = {nc.x, nc.y, nc.z};
        long long a[3];
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
            const double r = rint(t[d]);
            if (fabs(t[d] - r) > 1e-6 || r < 0.0 || r >= (double)ncs[d]) ok = false;
            a[d] = (long long)r;
        }
        if (!ok) {
            atomicAdd(flags, 1u);
            cell[i] = 0;
        } else {
            const long long g = a[0] + (long long)nc.x * (a[1] + (long long)nc.y * a[2]);
            cell[i] = (int32_t)g;
            if (atomicAdd(occ + g, 1u) != 0u) atomicAdd(flags + 1, 1u);
            lo = hi = (unsigned long long)(g - i + (1LL << 62));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long l2 = __shfl_xor_sync(0xffffffffu, lo, o);
        const unsigned long long h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    if ((threadIdx.x & 31) == 0 && lo != ~0ull) {
        atomicMin(ext, lo);
        atomicMax(ext + 1, hi);
    }
}

// Per row: first the delta check of every coded bond (a bond whose code's
// index delta is not its own j - i becomes generic), then the presence bits
// of the stencil entries the row holds (its codes are a strictly increasing
// subset of the table); per warp: 2 if every row is the whole table, 3 if
// every row is the same table subset (the subset is recorded for the warp),
// 1 if every row is a table subset, else 0.
// LUT: each bond's entry from the positions (L, as k_code_bonds does),
// written to code when it is given; else from the codes, which the delta
// check may rewrite.
template <bool LUT>
__global__ void __launch_bounds__(kBlock)
    k_row_masks(ParticleView p, EllView nl, const unsigned int* delta, uint8_t* code, int ntab,
                uint32_t* pmask, uint8_t* kind, uint32_t* warp_pmask,
                const int32_t* __restrict__ gcell, LatticeLut L)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int nmask = (ntab + 31) / 32;
    // Lanes past the last row do not vote against their warp.
    bool subset = true;
    bool full = true;
    uint32_t m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (i < p.n) {
        const int64_t np = p.npad;
        const int cnt = nl.count[i];
        full = cnt == ntab;
        int prev = -1;
        const int nx = 2 * L.half[0] + 1, ny = 2 * L.half[1] + 1;
        // No entry: the byte codes' generic code, or (positions, where the
        // table may hold up to kStencilMaxWide entries) a value past it.
        const int generic = LUT ? (1 << 20) : kMixedGeneric;
        for (int k = 0; k < cnt; ++k) {
            const int64_t o = (int64_t)k * np + i;
            const int64_t j = nl.idx[o];
            int c = generic;
            if (LUT) {
                int off[3];
                bool ok = true;
                for (int d = 0; d < 3; ++d) {
                    const double dd = p.x[d * np + j] - p.x[d * np + i];
                    const double a = rint(dd * L.hinv[d]);
                    if (fabs(dd - a * L.h[d]) > 1e-6 * L.h[d] || fabs(a) > L.half[d]) ok = false;
                    off[d] = (int)a;
                }
                if (ok) {
                    const int e = L.lut[(off[0] + L.half[0]) +
                                        nx * ((off[1] + L.half[1]) + ny * (off[2] + L.half[2]))];
                    if (e >= 0) c = e;
                }
            } else {
                c = code[o];
            }
            // The delta of the records' layout: lattice cells or rows.
            const long long dij = gcell ? (long long)gcell[j] - (long long)gcell[i]
                                        : (long long)(j - i);
            if (c != generic && (long long)delta[c] - (1LL << 31) != dij) c = generic;
            // The bond's code: rewritten when its delta fails, written in full
            // when the codes come from the positions (the mixed path).
            if (!LUT && c == generic) code[o] = (uint8_t)kMixedGeneric;
            if (LUT && code) code[o] = (uint8_t)(c < kMixedGeneric ? c : kMixedGeneric);
            if (!subset) continue;
            if (c >= ntab || c <= prev) {
                subset = false;
                continue;
            }
            if (c != k) full = false;
            m[c >> 5] |= 1u << (c & 31);
            prev = c;
        }
        if (!subset) full = false;
        for (int w = 0; w < nmask; ++w) pmask[(int64_t)w * np + i] = subset ? m[w] : 0u;
    }
    // Lane 0 holds a row whenever any lane of the warp does (rows are
    // contiguous from the warp's first lane).
    bool same = true;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const uint32_t lead = __shfl_sync(0xffffffffu, m[w], 0);
        if (i < p.n && m[w] != lead) same = false;
    }
    full = __all_sync(0xffffffffu, full);
    subset = __all_sync(0xffffffffu, subset);
    same = __all_sync(0xffffffffu, same);
    if ((threadIdx.x & 31) == 0) {
        const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int k = full ? 2 : (subset ? (same ? 3 : 1) : 0);
        kind[warp] = (uint8_t)k;
        if (k == 3)
            for (int w = 0; w < nmask; ++w) warp_pmask[warp * nmask + w] = m[w];
    }
}

// FP64 SoA positions -> FP32 hi/lo float4 (w = 0).
__global__ void __launch_bounds__(kBlock)
    k_split(const double* __restrict__ src, int64_t n, int64_t np, float4* hi, float4* lo)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float h[3], l[3];
    for (int d = 0; d < 3; ++d) {
        const double v = src[d * np + i];
        h[d] = __double2float_rn(v);
        l[d] = __double2float_rn(v - (double)h[d]);
    }
    hi[i] = make_float4(h[0], h[1], h[2], 0.f);
    lo[i] = make_float4(l[0], l[1], l[2], 0.f);
}

// FP64 displacement -> MixedU for every particle.
__global__ void __launch_bounds__(kBlock)
    k_split_u(ParticleView p, double c, MixedU* __restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    out[i] = split_u(p.u[i], p.u[np + i], p.u[2 * np + i], c * p.vol[i], p.nofail[i]);
}

// Velocity Verlet first half (CabanaPD_Integrate.hpp:89-116) that also
// refreshes the FP32 split of u; the new u goes to u_out (p.u: in place).
// Each operation is rounded separately, as in k_vv_initial.
__global__ void __launch_bounds__(kBlock)
    k_vv_initial_mixed(ParticleView p, double dt, double half_dt, double c,
                       double* __restrict__ u_out, MixedU* __restrict__ out)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double half_dt_m = __ddiv_rn(half_dt, p.rho[i]);
    double u[3];
    for (int d = 0; d < 3; ++d) {
        const double v = __dadd_rn(p.v[d * np + i], __dmul_rn(half_dt_m, p.f[d * np + i]));
        p.v[d * np + i] = v;
        u[d] = __dadd_rn(p.u[d * np + i], __dmul_rn(dt, v));
        u_out[d * np + i] = u[d];
    }
    out[i] = split_u(u[0], u[1], u[2], c * p.vol[i], p.nofail[i]);
}

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
// One bond of the mixed kernel: deformed bond vector r, FP32 stretch s and
// 1/|r| from the FP32 reference vector e (|e| = xi) and the split
// displacements of both ends.
struct MixedBond {
    float rx, ry, rz, s, rinv;
};

__device__ __forceinline__ void mixed_bond(float ex, float ey, float ez, float xi, float xiinv,
                                           const float4& uhj, const float4& ulj,
                                           const float4& uhi, const float4& uli, MixedBond& b)
{
    const float nx = (uhj.x - uhi.x) + (ulj.x - uli.x);
    const float ny = (uhj.y - uhi.y) + (ulj.y - uli.y);
    const float nz = (uhj.z - uhi.z) + (ulj.z - uli.z);
    b.rx = ex + nx;
    b.ry = ey + ny;
    b.rz = ez + nz;
    const float r2 = b.rx * b.rx + b.ry * b.ry + b.rz * b.rz;
    b.rinv = rsqrtf(r2);
    const float r = r2 * b.rinv;
    // eta . (2 xi_vec + eta) = r^2 - xi^2 without cancellation.
    const float num = nx * (2.f * ex + nx) + ny * (2.f * ey + ny) + nz * (2.f * ez + nz);
    b.s = __fdividef(num * xiinv, r + xi);
}

// The same bond with the x and y components carried as one float2 in the
// paired FP32 instructions of sm_100 (__fadd2_rn / __fmul2_rn / __ffma2_rn,
// each lane an IEEE round-to-nearest operation). eta and r are formed as in
// mixed_bond; the squared length and the stretch numerator group their
// terms differently, so results differ from mixed_bond by rounding only.
struct MixedBond2 {
    float2 rxy;
    float rz, s, rinv;
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ void mixed_bond2(float2 exy, float ez, float xi, float xiinv,
                                            const float4& uhj, const float4& ulj,
                                            float2 nuhi_xy, float nuhi_z, float2 nuli_xy,
                                            float nuli_z, MixedBond2& b)
{
    // u_j - u_i with the negated own displacement (hi and lo) held by the row.
    const float2 nxy = __fadd2_rn(__fadd2_rn(f2(uhj.x, uhj.y), nuhi_xy),
                                  __fadd2_rn(f2(ulj.x, ulj.y), nuli_xy));
    const float nz = (uhj.z + nuhi_z) + (ulj.z + nuli_z);
    b.rxy = __fadd2_rn(exy, nxy);
    b.rz = ez + nz;
    const float2 sq = __fmul2_rn(b.rxy, b.rxy);
    const float r2 = fmaf(b.rz, b.rz, sq.x + sq.y);
    b.rinv = rsqrtf(r2);
    const float r = r2 * b.rinv;
    const float2 a2 = __ffma2_rn(f2(2.f, 2.f), exy, nxy);
    const float2 pq = __fmul2_rn(nxy, a2);
    const float num = fmaf(nz, fmaf(2.f, ez, nz), pq.x + pq.y);
    b.s = __fdividef(num * xiinv, r + xi);
}

// Kahan-compensated accumulation of a pair of terms (x, y lanes).
__device__ __forceinline__ void kahan_add2(float2& sum, float2& comp, float2 term)
{
    const float2 m1 = f2(-1.f, -1.f);
    const float2 y = __ffma2_rn(comp, m1, term);   // term - comp
    const float2 t = __fadd2_rn(sum, y);
    const float2 z = __ffma2_rn(sum, m1, t);       // t - sum
    comp = __ffma2_rn(y, m1, z);                   // (t - sum) - y
    sum = t;
}

// The break test of one bond (CabanaPD_ForceModels.hpp:123-128 with the
// PMB no-fail rule, force/CabanaPD_PMB.hpp:260-261): FP32 stretch against
// s0, re-tested in FP64 inside the guard band.
__device__ __forceinline__ bool mixed_critical(float s, float nofail_j, bool nofail_i,
                                               const MixedModel& md, const ParticleView& p,
                                               int64_t i, int64_t j)
{
    if (nofail_i || nofail_j != 0.f) return false;
    if (fabsf(s - md.s0) <= md.guard) return critical_exact64(p.x, p.u, p.npad, i, j, md.bbc);
    return s >= md.s0;
}

// Full-stencil rows (every table entry present, bond slot k = entry k),
// x / y lanes in paired FP32 instructions: the table is walked in chunks of
// 8 bonds with the bond bits of a chunk tested at constant positions, broken
// bonds contribute a zero term instead of a branch, and the newly broken
// bits of a 32-bond word are cleared once.
template <bool FRACTURE>
__device__ __forceinline__ void mixed_full_rows2(const ParticleView& p, const EllView& nl,
                                                 const MixedU* __restrict__ u2_i,
                                                 const MixedStencil* tab,
                                                 const MixedModel& md, int64_t i,
                                                 const float4& uhi, const float4& uli,
                                                 bool nofail_i, float2& sxy, float2& cxy,
                                                 float& sz, float& cz)
{
    const int64_t np = p.npad;
    const float2 nuhi_xy = f2(-uhi.x, -uhi.y), nuli_xy = f2(-uli.x, -uli.y);
    const float nuhi_z = -uhi.z, nuli_z = -uli.z;
    for (int base = 0; base < md.ntab; base += 32) {
        const uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
        uint32_t clr = 0;
        const int lim = min(32, md.ntab - base);
        for (int b = 0; b < lim; b += 8) {
            const uint32_t w8 = word >> b;
            uint32_t c8 = 0;
            const int n8 = min(8, lim - b);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (u < n8) {
                    const MixedStencil t = tab[base + b + u];
                    const MixedU uj = u2_i[t.delta];
                    MixedBond2 bd;
                    mixed_bond2(f2(t.x, t.y), t.z, t.xi, t.xiinv, uj.hi, uj.lo, nuhi_xy, nuhi_z,
                                nuli_xy, nuli_z, bd);
                    float kf = uj.hi.w * bd.s * bd.rinv;
                    if (FRACTURE) {
                        const bool crit = mixed_critical(bd.s, uj.lo.w, nofail_i, md, p, i,
                                                         i + t.delta);
                        c8 |= (uint32_t)crit << u;
                        kf = (((w8 >> u) & 1u) && !crit) ? kf : 0.f;
                    }
                    kahan_add2(sxy, cxy, __fmul2_rn(f2(kf, kf), bd.rxy));
                    kahan_add(sz, cz, kf * bd.rz);
                }
            }
            clr |= c8 << b;
        }
        if (FRACTURE && (word & clr)) nl.mu[(int64_t)(base >> 5) * np + i] = word & ~clr;
    }
}

// Row i's own displacement split, negated, and its no-fail flag.
struct RowSplit {
    float2 nuh_xy, nul_xy;
    float nuh_z, nul_z;
    bool nofail;
};

// Bond geometry of the lean form: eta = u_j - u_i from the splits,
// num = eta . (2 xi_vec + eta) = r^2 - xi^2 without cancellation, r^2 =
// xi^2 + num, and s = (r - xi) / xi = num / (xi (r + xi)).
__device__ __forceinline__ void lean_geometry(const MixedStencil& t, const MixedU& uj,
                                              const RowSplit& ri, MixedBond2& b)
{
    const float2 exy = f2(t.x, t.y);
    const float2 nxy = __fadd2_rn(__fadd2_rn(f2(uj.hi.x, uj.hi.y), ri.nuh_xy),
                                  __fadd2_rn(f2(uj.lo.x, uj.lo.y), ri.nul_xy));
    const float nz = (uj.hi.z + ri.nuh_z) + (uj.lo.z + ri.nul_z);
    b.rxy = __fadd2_rn(exy, nxy);
    b.rz = t.z + nz;
    const float2 pq = __fmul2_rn(nxy, __ffma2_rn(f2(2.f, 2.f), exy, nxy));
    const float num = fmaf(nz, fmaf(2.f, t.z, nz), pq.x + pq.y);
    const float r2 = t.xi2 + num;
    b.rinv = rsqrtf(r2);
    const float r = r2 * b.rinv;
    b.s = __fdividef(num, fmaf(r, t.xi, t.xi2));
}

// Row i (of warp chunk `warp`) of the general mixed PMB kernel, with the
// stencil table staged at tab (the body of k_pmb_force_mixed and of the
// batch kernel's mixed PMB rows).
template <bool FRACTURE>
__device__ __forceinline__ void pmb_mixed_row(const ParticleView& p, const EllView& nl,
                                              const MixedView& mv, const MixedStencil* tab,
                                              const MixedModel& md, const StepEpilogue& ep,
                                              int64_t warp, int64_t i)
{
    const int kind = warp < ((p.n - p.frozen + 31) >> 5) ? mv.warp_kind[warp] : 0;
    const int64_t np = p.npad;
    const MixedU ui = mv.u2[i];
    const float4 uhi = ui.hi, uli = ui.lo;
    const bool nofail_i = FRACTURE ? (uli.w != 0.f) : false;
    const int cnt = nl.count[i];
    const uint8_t* __restrict__ code = mv.code + i;
    const MixedU* __restrict__ U2 = mv.u2;
    float sx = 0.f, sy = 0.f, sz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    if (kind == 2) {
        float2 sxy = f2(0.f, 0.f), cxy = f2(0.f, 0.f);
        float sz = 0.f, cz = 0.f;
        mixed_full_rows2<FRACTURE>(p, nl, U2 + i, tab, md, i, uhi, uli, nofail_i, sxy, cxy, sz,
                                   cz);
        step_epilogue<true>(p, ep, i, (double)sxy.x - (double)cxy.x,
                            (double)sxy.y - (double)cxy.y, (double)sz - (double)cz);
        return;
    }
    if (kind != 0) {
        // Stencil rows: bond slots are the row's table entries in table
        // order, so entry k is read at a warp-uniform address. Full rows
        // (kind 2) hold every entry; subset rows skip the absent ones.
        const MixedU* __restrict__ u2_i = U2 + i;
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
                const float4 uhj = u2_i[t.delta].hi, ulj = u2_i[t.delta].lo;
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
                    const float kf = uhj.w * s * rinv;
                    kahan_add(sx, cx, kf * rx);
                    kahan_add(sy, cy, kf * ry);
                    kahan_add(sz, cz, kf * rz);
                }
            }
        }
        if (FRACTURE && word != old) nl.mu[(int64_t)cur_w * np + i] = word;
        step_epilogue<true>(p, ep, i, (double)sx - (double)cx, (double)sy - (double)cy,
                            (double)sz - (double)cz);
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
            const float4 uhj = U2[j].hi, ulj = U2[j].lo;
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
                const float kf = uhj.w * s * rinv;
                kahan_add(sx, cx, kf * rx);
                kahan_add(sy, cy, kf * ry);
                kahan_add(sz, cz, kf * rz);
            }
        }
        if (FRACTURE && word != old) nl.mu[(int64_t)(base >> 5) * np + i] = word;
    }
    step_epilogue<true>(p, ep, i, (double)sx - (double)cx, (double)sy - (double)cy,
                        (double)sz - (double)cz);
}

// General mixed PMB kernel: rows that the stencil kernel does not take
// (irregular rows, tables over its size), one warp per chunk of 32 rows of
// the warp list, or every chunk in tile order without one. Dynamic shared
// memory: the stencil table.
template <bool FRACTURE>
__global__ void __launch_bounds__(kBlock, 4)
    k_pmb_force_mixed(ParticleView p, EllView nl, MixedView mv, MixedModel md, StepEpilogue ep,
                      const int32_t* __restrict__ wlist, int64_t wcount)
{
    extern __shared__ MixedStencil smem[];
    MixedStencil* tab = smem;
    for (int t = threadIdx.x; t < md.ntab; t += blockDim.x) tab[t] = mv.table[t];
    __syncthreads();
    int64_t warp;
    if (wlist) {
        const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        if (slot >= wcount) return;
        warp = wlist[slot];
    } else {
        warp = tile_chunk(nl);
    }
    const int64_t i = p.frozen + 32 * warp + (threadIdx.x & 31);
    if (i >= p.n) return;
    pmb_mixed_row<FRACTURE>(p, nl, mv, tab, md, ep, warp, i);
}

// Prologue of the lean kernels: stages the stencil table in shared memory
// and takes the calling warp's row chunk from the warp list; a warp whose
// rows share one stencil subset (kind 3) also stages its compacted table
// (entry k of the subset at slot "present entries before k"). Returns false
// for warps past the end of the list.
__device__ __forceinline__ bool lean_prologue(const MixedView& mv, int ntab,
                                              const int32_t* __restrict__ wlist, int64_t wcount,
                                              MixedStencil* smem, int64_t& warp,
                                              const MixedStencil*& wt, int& wcnt)
{
    for (int t = threadIdx.x; t < ntab; t += blockDim.x) smem[t] = mv.table[t];
    __syncthreads();
    const int64_t slot = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (slot >= wcount) return false;
    warp = wlist[slot];
    wt = smem;
    wcnt = ntab;
    if (mv.warp_kind[warp] == 3) {
        const int lane = threadIdx.x & 31;
        const int nmask = (ntab + 31) / 32;
        MixedStencil* mine = smem + ntab * (1 + (threadIdx.x >> 5));
        const uint32_t* wm = mv.warp_pmask + warp * nmask;
        int before = 0;
        for (int w = 0; w < nmask; ++w) {
            const uint32_t pm = wm[w];
            if ((pm >> lane) & 1u)
                mine[before + __popc(pm & ((1u << lane) - 1u))] = smem[32 * w + lane];
            before += __popc(pm);
        }
        __syncwarp();
        wt = mine;
        wcnt = before;
    }
    return true;
}

// ---------------------------------------------------------------------------
// LPS, mixed precision (force/CabanaPD_LPS.hpp:287-447 with the model of
// force_models/CabanaPD_LPS.hpp:85-134). Stencil rows only: jobs with an
// irregular row keep the FP64 LPS kernels. FP32 bond arithmetic as in the
// PMB kernel (split displacements, stretch without cancellation), Kahan-
// compensated FP32 sums; m, theta and the per-particle force factors
// a = theta_coeff theta / m and b = s_coeff / m are formed in FP64 from the
// sums and kept as FP32 pairs for the neighbours' force loop. The break test
// follows the LPS rule (no-fail of the row only, tested twice by the
// reference) with the FP64 re-test inside the guard band.

// omega xi^2 of a stencil entry (force_models/CabanaPD_LPS.hpp:85-106) and
// the omega xi factor of the force coefficient (:118-134).
template <int INFL>
__device__ __forceinline__ float lps_w(const MixedStencil& t)
{
    return INFL == 1 ? t.xi : t.xi * t.xi;
}
template <int INFL>
__device__ __forceinline__ float lps_oxi(const MixedStencil& t)
{
    return INFL == 1 ? 1.f : t.xi;
}

// Weighted volume (when WITH_M) and dilatation of one row, one pass.
template <bool FRACTURE, int INFL, bool WITH_M>
__device__ __forceinline__ void lps_mtheta_mixed_row(const ParticleView& p, const EllView& nl,
                                                     const MixedView& mv,
                                                     const MixedStencil* tab,
                                                     const MixedLps& md, float2* ab,
                                                     MixedU* pack, int64_t warp, int64_t i)
{
    const int64_t np = p.npad;
    const MixedU ui = mv.u2[i];
    const float4 uhi = ui.hi, uli = ui.lo;
    const float2 nuhi_xy = f2(-uhi.x, -uhi.y), nuli_xy = f2(-uli.x, -uli.y);
    const float nuhi_z = -uhi.z, nuli_z = -uli.z;
    const MixedU* __restrict__ u2_i = mv.u2 + i;
    const int kind = mv.warp_kind[warp];
    float ms = 0.f, mc = 0.f, ts = 0.f, tc = 0.f;
    if (kind == 2) {
        for (int base = 0; base < md.ntab; base += 32) {
            const uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
            const int lim = min(32, md.ntab - base);
            for (int b = 0; b < lim; b += 8) {
                const uint32_t w8 = word >> b;
                const int n8 = min(8, lim - b);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (u < n8) {
                        const MixedStencil t = tab[base + b + u];
                        const MixedU uj = u2_i[t.delta];
                        MixedBond2 bd;
                        mixed_bond2(f2(t.x, t.y), t.z, t.xi, t.xiinv, uj.hi, uj.lo, nuhi_xy,
                                    nuhi_z, nuli_xy, nuli_z, bd);
                        const float on = ((w8 >> u) & 1u) ? 1.f : 0.f;
                        const float wv = on * lps_w<INFL>(t) * uj.hi.w;
                        if (WITH_M) kahan_add(ms, mc, wv);
                        kahan_add(ts, tc, wv * bd.s);
                    }
                }
            }
        }
    } else {
        // Subset rows: bond slot = rank of the entry among the present ones.
        const int nmask = (md.ntab + 31) / 32;
        int slot = 0;
        uint32_t word = FRACTURE ? nl.mu[i] : 0xffffffffu;
        for (int w = 0; w < nmask; ++w) {
            const uint32_t pm = mv.pmask[(int64_t)w * np + i];
            const int kend = min(32, md.ntab - 32 * w);
            for (int b = 0; b < kend; ++b) {
                if (!((pm >> b) & 1u)) continue;
                if (FRACTURE && (slot & 31) == 0 && slot > 0)
                    word = nl.mu[(int64_t)(slot >> 5) * np + i];
                const bool on = (word >> (slot & 31)) & 1u;
                ++slot;
                if (!on) continue;
                const MixedStencil t = tab[32 * w + b];
                const MixedU uj = u2_i[t.delta];
                MixedBond2 bd;
                mixed_bond2(f2(t.x, t.y), t.z, t.xi, t.xiinv, uj.hi, uj.lo, nuhi_xy, nuhi_z,
                            nuli_xy, nuli_z, bd);
                const float wv = lps_w<INFL>(t) * uj.hi.w;
                if (WITH_M) kahan_add(ms, mc, wv);
                kahan_add(ts, tc, wv * bd.s);
            }
        }
    }
    const double m = WITH_M ? (double)ms - (double)mc : p.m[i];
    const double th = (!FRACTURE || m > 0) ? 3.0 * ((double)ts - (double)tc) / m : 0.0;
    if (WITH_M) p.m[i] = m;
    p.theta[i] = th;
    const double a = md.theta_coeff * th / m, b = md.s_coeff / m;
    p.lps_a[i] = a;
    p.lps_b[i] = b;
    ab[i] = make_float2((float)a, (float)b);
    if (pack)
        pack[i] = MixedU{make_float4(uhi.x, uhi.y, uhi.z, (float)a),
                         make_float4(uli.x, uli.y, uli.z, (float)b)};
}

template <bool FRACTURE, int INFL, bool WITH_M>
__global__ void __launch_bounds__(kBlock, 4)
    k_lps_mtheta_mixed(ParticleView p, EllView nl, MixedView mv, MixedLps md,
                       float2* __restrict__ ab, const int32_t* __restrict__ wlist,
                       int64_t wcount, MixedU* __restrict__ pack)
{
    __shared__ MixedStencil tab[kMixedGeneric];
    for (int t = threadIdx.x; t < md.ntab; t += blockDim.x) tab[t] = mv.table[t];
    __syncthreads();
    // Rows: the listed warps' chunks when a warp list is given.
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wlist) {
        const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        if (slot >= wcount) return;
        warp = wlist[slot];
    }
    const int64_t i = p.frozen + 32 * warp + (threadIdx.x & 31);
    if (i >= p.n) return;
    lps_mtheta_mixed_row<FRACTURE, INFL, WITH_M>(p, nl, mv, tab, md, ab, pack, warp, i);
}

__device__ __forceinline__ bool lps_critical(float s, bool nofail_i, const MixedLps& md,
                                             const ParticleView& p, int64_t i, int64_t j)
{
    // force/CabanaPD_LPS.hpp:417-418: only the row's no-fail flag counts.
    if (nofail_i) return false;
    if (fabsf(s - md.s0) <= md.guard) return critical_exact64(p.x, p.u, p.npad, i, j, md.bbc);
    return s >= md.s0;
}

template <bool FRACTURE, int INFL>
__device__ __forceinline__ void lps_force_mixed_row(const ParticleView& p, const EllView& nl,
                                                    const MixedView& mv,
                                                    const MixedStencil* tab,
                                                    const MixedLps& md, const float2* ab,
                                                    const StepEpilogue& ep, int64_t warp,
                                                    int64_t i)
{
    const int64_t np = p.npad;
    const MixedU ui = mv.u2[i];
    const float4 uhi = ui.hi, uli = ui.lo;
    const bool nofail_i = FRACTURE ? (uli.w != 0.f) : false;
    const float2 nuhi_xy = f2(-uhi.x, -uhi.y), nuli_xy = f2(-uli.x, -uli.y);
    const float nuhi_z = -uhi.z, nuli_z = -uli.z;
    const float2 abi = ab[i];
    const MixedU* __restrict__ u2_i = mv.u2 + i;
    const float2* __restrict__ ab_i = ab + i;
    const int kind = mv.warp_kind[warp];
    float2 sxy = f2(0.f, 0.f), cxy = f2(0.f, 0.f);
    float sz = 0.f, cz = 0.f;
    if (kind == 2) {
        for (int base = 0; base < md.ntab; base += 32) {
            const uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
            uint32_t clr = 0;
            const int lim = min(32, md.ntab - base);
            for (int b = 0; b < lim; b += 8) {
                const uint32_t w8 = word >> b;
                uint32_t c8 = 0;
                const int n8 = min(8, lim - b);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    if (u < n8) {
                        const MixedStencil t = tab[base + b + u];
                        const MixedU uj = u2_i[t.delta];
                        const float2 abj = ab_i[t.delta];
                        MixedBond2 bd;
                        mixed_bond2(f2(t.x, t.y), t.z, t.xi, t.xiinv, uj.hi, uj.lo, nuhi_xy,
                                    nuhi_z, nuli_xy, nuli_z, bd);
                        float kf = (abi.x + abj.x + bd.s * (abi.y + abj.y)) * lps_oxi<INFL>(t) *
                                   uj.hi.w * bd.rinv;
                        if (FRACTURE) {
                            const bool crit = lps_critical(bd.s, nofail_i, md, p, i, i + t.delta);
                            c8 |= (uint32_t)crit << u;
                            kf = (((w8 >> u) & 1u) && !crit) ? kf : 0.f;
                        }
                        kahan_add2(sxy, cxy, __fmul2_rn(f2(kf, kf), bd.rxy));
                        kahan_add(sz, cz, kf * bd.rz);
                    }
                }
                clr |= c8 << b;
            }
            if (FRACTURE && (word & clr)) nl.mu[(int64_t)(base >> 5) * np + i] = word & ~clr;
        }
    } else {
        const int nmask = (md.ntab + 31) / 32;
        int slot = 0, cur_w = 0;
        uint32_t word = FRACTURE ? nl.mu[i] : 0xffffffffu;
        uint32_t old = word;
        for (int w = 0; w < nmask; ++w) {
            const uint32_t pm = mv.pmask[(int64_t)w * np + i];
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
                const MixedU uj = u2_i[t.delta];
                const float2 abj = ab_i[t.delta];
                MixedBond2 bd;
                mixed_bond2(f2(t.x, t.y), t.z, t.xi, t.xiinv, uj.hi, uj.lo, nuhi_xy, nuhi_z,
                            nuli_xy, nuli_z, bd);
                float kf = (abi.x + abj.x + bd.s * (abi.y + abj.y)) * lps_oxi<INFL>(t) * uj.hi.w *
                           bd.rinv;
                if (FRACTURE) {
                    if (lps_critical(bd.s, nofail_i, md, p, i, i + t.delta)) word &= ~(1u << sb);
                    kf = ((word >> sb) & 1u) ? kf : 0.f;
                }
                kahan_add2(sxy, cxy, __fmul2_rn(f2(kf, kf), bd.rxy));
                kahan_add(sz, cz, kf * bd.rz);
            }
        }
        if (FRACTURE && word != old) nl.mu[(int64_t)cur_w * np + i] = word;
    }
    step_epilogue<true>(p, ep, i, (double)sxy.x - (double)cxy.x, (double)sxy.y - (double)cxy.y,
                        (double)sz - (double)cz);
}

template <bool FRACTURE, int INFL>
__global__ void __launch_bounds__(kBlock, 4)
    k_lps_force_mixed(ParticleView p, EllView nl, MixedView mv, MixedLps md,
                      const float2* __restrict__ ab, StepEpilogue ep,
                      const int32_t* __restrict__ wlist, int64_t wcount)
{
    __shared__ MixedStencil tab[kMixedGeneric];
    for (int t = threadIdx.x; t < md.ntab; t += blockDim.x) tab[t] = mv.table[t];
    __syncthreads();
    // Rows: the listed warps' chunks when a warp list is given.
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wlist) {
        const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        if (slot >= wcount) return;
        warp = wlist[slot];
    }
    const int64_t i = p.frozen + 32 * warp + (threadIdx.x & 31);
    if (i >= p.n) return;
    lps_force_mixed_row<FRACTURE, INFL>(p, nl, mv, tab, md, ab, ep, warp, i);
}

// LPS lean forms, over the warps of kinds 2 and 3 (warp list; the other
// warps run k_lps_mtheta_mixed / k_lps_force_mixed over theirs): as the PMB
// lean form, FP32 sums per chunk of 8 bonds added to FP64 row totals, and
// bonds near s0 deferred to the exact test after each 32-bond word.
template <int INFL, bool WITH_M>
__device__ __forceinline__ void lps_theta_bond(const MixedStencil& t,
                                               const MixedU* __restrict__ u2_i,
                                               const RowSplit& ri, bool on, float& cm, float& ct)
{
    const MixedU uj = u2_i[t.delta];
    MixedBond2 bd;
    lean_geometry(t, uj, ri, bd);
    const float wv = on ? (INFL == 1 ? t.xi : t.xi2) * uj.hi.w : 0.f;
    if (WITH_M) cm += wv;
    ct = fmaf(wv, bd.s, ct);
}

// 4-bond chunks at 3 blocks of 256 per SM: 72 registers, no spills. On the
// 8.0 M-particle LPS box (B200, ms per mixed step) this form runs 5.08;
// at 4 blocks (64 registers, spilling) 5.12, 8-bond chunks at 3 blocks
// 5.21, 2-bond chunks at 4 / 5 blocks 5.22 / 5.15.
constexpr int kThetaUnroll = 4;

template <bool FRACTURE, int INFL, bool WITH_M>
__global__ void __launch_bounds__(kBlock, 3)
    k_lps_mtheta_lean(ParticleView p, EllView nl, MixedView mv, MixedLps md,
                      float2* __restrict__ ab, const int32_t* __restrict__ wlist, int64_t wcount,
                      MixedU* __restrict__ pack)
{
    extern __shared__ MixedStencil smem[];
    int64_t warp;
    const MixedStencil* wt;
    int wcnt;
    if (!lean_prologue(mv, md.ntab, wlist, wcount, smem, warp, wt, wcnt)) return;
    const int64_t i = p.frozen + 32 * warp + (threadIdx.x & 31);
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const MixedU ui = mv.u2[i];
    const RowSplit ri{f2(-ui.hi.x, -ui.hi.y), f2(-ui.lo.x, -ui.lo.y), -ui.hi.z, -ui.lo.z, false};
    const MixedU* __restrict__ u2_i = mv.u2 + i;
    double msum = 0.0, tsum = 0.0;
    for (int base = 0; base < wcnt; base += 32) {
        const uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
        const int lim = min(32, wcnt - base);
        int b = 0;
        for (; b + kThetaUnroll <= lim; b += kThetaUnroll) {
            const uint32_t w8 = word >> b;
            float cm = 0.f, ct = 0.f;
#pragma unroll
            for (int u = 0; u < kThetaUnroll; ++u)
                lps_theta_bond<INFL, WITH_M>(wt[base + b + u], u2_i, ri, (w8 >> u) & 1u, cm, ct);
            msum += (double)cm;
            tsum += (double)ct;
        }
        if (b < lim) {
            float cm = 0.f, ct = 0.f;
            for (; b < lim; ++b)
                lps_theta_bond<INFL, WITH_M>(wt[base + b], u2_i, ri, (word >> b) & 1u, cm, ct);
            msum += (double)cm;
            tsum += (double)ct;
        }
    }
    const double m = WITH_M ? msum : p.m[i];
    const double th = (!FRACTURE || m > 0) ? 3.0 * tsum / m : 0.0;
    if (WITH_M) p.m[i] = m;
    p.theta[i] = th;
    const double a = md.theta_coeff * th / m, b = md.s_coeff / m;
    p.lps_a[i] = a;
    p.lps_b[i] = b;
    ab[i] = make_float2((float)a, (float)b);
    if (pack)
        pack[i] = MixedU{make_float4(ui.hi.x, ui.hi.y, ui.hi.z, (float)a),
                         make_float4(ui.lo.x, ui.lo.y, ui.lo.z, (float)b)};
}

// One LPS bond of the lean force (the break rule of lps_critical: only the
// row's no-fail flag counts).
// PACK: u2_i points into the packed records (a, b in the w lanes; the
// volume is md.vol), and ab_i is not read.
template <bool FRACTURE, int INFL, bool PACK = false>
__device__ __forceinline__ void lps_force_bond(const MixedStencil& t,
                                               const MixedU* __restrict__ u2_i,
                                               const float2* __restrict__ ab_i, float2 abi,
                                               const RowSplit& ri, bool on, uint32_t bit,
                                               const MixedLps& md, uint32_t& clr, uint32_t& pend,
                                               float2& cxy, float& cz)
{
    const MixedU uj = u2_i[t.delta];
    const float2 abj = PACK ? f2(uj.hi.w, uj.lo.w) : ab_i[t.delta];
    const float vol_j = PACK ? md.vol : uj.hi.w;
    MixedBond2 bd;
    lean_geometry(t, uj, ri, bd);
    if (FRACTURE && on && bd.s >= md.s_lo && !ri.nofail) {
        if (bd.s > md.s_hi)
            clr |= bit;
        else
            pend |= bit;
        on = false;
    }
    const float kf = (!FRACTURE || on)
                         ? (abi.x + abj.x + bd.s * (abi.y + abj.y)) * lps_oxi<INFL>(t) * vol_j *
                               bd.rinv
                         : 0.f;
    cxy = __ffma2_rn(f2(kf, kf), bd.rxy, cxy);
    cz = fmaf(kf, bd.rz, cz);
}

// 8-bond chunks at 4 blocks of 256 per SM (60 registers). Measured beside it
// on the 8.0 M-particle LPS box, no faster: 3 blocks, 4-bond chunks at 4 or
// 5 blocks.
// PACK: the neighbours' records come from pack (the m / theta pass's
// packed copy), one 32-byte load per bond instead of u2 and ab.
template <bool FRACTURE, int INFL, bool PACK = false>
__global__ void __launch_bounds__(kBlock, 4)
    k_lps_force_lean(ParticleView p, EllView nl, MixedView mv, MixedLps md,
                     const float2* __restrict__ ab, StepEpilogue ep,
                     const int32_t* __restrict__ wlist, int64_t wcount,
                     const MixedU* __restrict__ pack)
{
    extern __shared__ MixedStencil smem[];
    int64_t warp;
    const MixedStencil* wt;
    int wcnt;
    if (!lean_prologue(mv, md.ntab, wlist, wcount, smem, warp, wt, wcnt)) return;
    const int64_t i = p.frozen + 32 * warp + (threadIdx.x & 31);
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const MixedU ui = PACK ? pack[i] : mv.u2[i];
    const bool nofail_i = FRACTURE ? (PACK ? p.nofail[i] != 0 : ui.lo.w != 0.f) : false;
    const RowSplit ri{f2(-ui.hi.x, -ui.hi.y), f2(-ui.lo.x, -ui.lo.y), -ui.hi.z, -ui.lo.z,
                      nofail_i};
    const MixedU* __restrict__ u2_i = (PACK ? pack : mv.u2) + i;
    const float2* __restrict__ ab_i = ab + i;
    const float2 abi = PACK ? f2(ui.hi.w, ui.lo.w) : ab[i];
    double f[3] = {0.0, 0.0, 0.0};
    for (int base = 0; base < wcnt; base += 32) {
        const uint32_t word = FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
        uint32_t clr = 0, pend = 0;
        const int lim = min(32, wcnt - base);
        int b = 0;
        for (; b + 8 <= lim; b += 8) {
            const uint32_t w8 = word >> b;
            float2 cxy = f2(0.f, 0.f);
            float cz = 0.f;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                lps_force_bond<FRACTURE, INFL, PACK>(wt[base + b + u], u2_i, ab_i, abi, ri,
                                                     (w8 >> u) & 1u, 1u << (b + u), md, clr, pend,
                                                     cxy, cz);
            f[0] += (double)cxy.x;
            f[1] += (double)cxy.y;
            f[2] += (double)cz;
        }
        if (b < lim) {
            float2 cxy = f2(0.f, 0.f);
            float cz = 0.f;
            for (; b < lim; ++b)
                lps_force_bond<FRACTURE, INFL, PACK>(wt[base + b], u2_i, ab_i, abi, ri,
                                                     (word >> b) & 1u, 1u << b, md, clr, pend,
                                                     cxy, cz);
            f[0] += (double)cxy.x;
            f[1] += (double)cxy.y;
            f[2] += (double)cz;
        }
        if (FRACTURE) {
            while (pend) {
                const int k = __ffs(pend) - 1;
                pend &= pend - 1;
                const MixedStencil t = wt[base + k];
                if (critical_exact64(p.x, p.u, np, i, i + t.delta, md.bbc)) {
                    clr |= 1u << k;
                } else {
                    float2 cxy = f2(0.f, 0.f);
                    float cz = 0.f;
                    uint32_t none = 0;
                    lps_force_bond<false, INFL, PACK>(t, u2_i, ab_i, abi, ri, true, 0u, md, none,
                                                      none, cxy, cz);
                    f[0] += (double)cxy.x;
                    f[1] += (double)cxy.y;
                    f[2] += (double)cz;
                }
            }
            if (clr) nl.mu[(int64_t)(base >> 5) * np + i] = word & ~clr;
        }
    }
    step_epilogue<true>(p, ep, i, f[0], f[1], f[2]);
}

// The split forms (lean kernel, then the rest) pay only on large systems:
// below about a million rows the second launch's serial tail costs more than
// the lean kernel saves (B200: 69 K-row PMB wave 0.045 ms single vs 0.070 ms
// split, 125 K-row LPS box 0.123 vs 0.191 ms; 1.2 M-row plate 0.397 vs
// 0.376 ms).
// CPD_SPLIT_MIN_ROWS overrides the threshold (0: split forms at every size).
int64_t split_min_rows()
{
    static const int64_t v = [] {
        const char* e = getenv("CPD_SPLIT_MIN_ROWS");
        return e ? (int64_t)atoll(e) : (int64_t)(1 << 20);
    }();
    return v;
}

// ---------------------------------------------------------------------------
// Hertzian contact, mixed precision (force/CabanaPD_Contact.hpp:119-168 with
// force_models/CabanaPD_Hertzian.hpp:23-88 and per-pair radii). The overlap
// needs FP64: it is ~1e-7 of the centre distance, below FP32 resolution of
// the positions. So the deformed pair vector r = (x_j - x_i) + (u_j - u_i),
// |r| and the overlap delta = |r| - (R_i + R_j) stay FP64 (in the reference's
// operation order); the force law in the overlap (|delta|^(3/2), the contact
// stiffness, the damping sqrt(S_n m*) v_n and the normal projection) runs in
// FP32, and the row force is summed in FP64. Pairs without overlap add no
// force (the reference adds a zero).
struct HertzMixed {
    float Es43, Es2, coeff_h_d;  // 4/3 E*, 2 E*, the damping coefficient
    float Rs, coeff_h_n;         // single-radius model
    double sum_r;                // single-radius model: 2 R
};

// EPI: a contact-only fused step; the epilogue finishes the row (force BC,
// half steps, next displacement and velocity into the second buffers).
// 4 blocks of 256 per SM (64 registers, no spills): the fused DEM step's
// kernel 0.246 -> 0.202 ms against 3 blocks on the 4.0 M-sphere packing.
template <bool PER_PARTICLE, bool EPI = false>
__global__ void __launch_bounds__(kBlock, 4)
    k_hertz_force_mixed(ParticleView p, EllView nl, HertzMixed md, bool reset, StepEpilogue ep)
{
    const int64_t i = p.frozen + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int64_t np = p.npad;
    const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
    const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
    const double vi0 = p.v[i], vi1 = p.v[np + i], vi2 = p.v[2 * np + i];
    const double R_i = PER_PARTICLE ? p.radius[i] : 0.0;
    const float inv_vol_i = (float)(1.0 / p.vol[i]);
    const float m_i = (float)(p.rho[i] * p.vol[i]);
    double fx = reset ? 0.0 : p.f[i];
    double fy = reset ? 0.0 : p.f[np + i];
    double fz = reset ? 0.0 : p.f[2 * np + i];
    const int cnt = nl.count[i];
    for (int k = 0; k < cnt; ++k) {
        const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
        const double rx = (__ldg(p.x + j) - xi0) + (__ldg(p.u + j) - ui0);
        const double ry = (__ldg(p.x + np + j) - xi1) + (__ldg(p.u + np + j) - ui1);
        const double rz = (__ldg(p.x + 2 * np + j) - xi2) + (__ldg(p.u + 2 * np + j) - ui2);
        const double r = sqrt(rx * rx + ry * ry + rz * rz);
        const double R_j = PER_PARTICLE ? __ldg(p.radius + j) : 0.0;
        const double delta = r - (PER_PARTICLE ? R_i + R_j : md.sum_r);
        if (!(delta < 0.0)) continue;
        const float ad = (float)(-delta);
        const float rinv = (float)(1.0 / r);
        const float nx = (float)rx * rinv, ny = (float)ry * rinv, nz = (float)rz * rinv;
        const float vn = (float)(__ldg(p.v + j) - vi0) * nx + (float)(__ldg(p.v + np + j) - vi1) * ny +
                         (float)(__ldg(p.v + 2 * np + j) - vi2) * nz;
        float Rs, coeff_h_n, ms;
        if (PER_PARTICLE) {
            const float ri = (float)R_i, rj = (float)R_j;
            Rs = ri * (rj / (ri + rj));
            coeff_h_n = md.Es43 * sqrtf(Rs);
            const float m_j = (float)(__ldg(p.rho + j) * __ldg(p.vol + j));
            ms = m_i * (m_j / (m_i + m_j));
        } else {
            Rs = md.Rs;
            coeff_h_n = md.coeff_h_n;
            ms = 0.5f * m_i;
        }
        const float h = -coeff_h_n * ad * sqrtf(ad);
        const float Sn = md.Es2 * sqrtf(Rs * ad);
        const float coeff = (h - md.coeff_h_d * sqrtf(Sn * ms) * vn) * inv_vol_i;
        fx += (double)(coeff * nx);
        fy += (double)(coeff * ny);
        fz += (double)(coeff * nz);
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
// Strain energy density and damage on the mixed path (force/CabanaPD_PMB.hpp:
// 127-155, 289-339; force/CabanaPD_LPS.hpp:183-219, 449-504). One kernel over
// all rows in blocks of 256 consecutive rows (the exact kernel's blocks and
// partials). Warps of full-stencil or shared-subset rows walk the stencil
// table with the FP32 bond arithmetic of the force kernels, summing the bond
// terms in FP32 chunks of 8 into FP64; other warps walk their rows with FP64
// geometry. The damage sums FP64 volumes in row order, so phi_i is the
// exact kernel's. LPS: W_i = theta_coeff theta_i^2 / 6 (over the intact
// bonds' 1 / num_bonds shares) + (s_coeff / 2 m_i) sum omega xi^2 s^2 vol_j.
struct MixedEnergy {
    double c, theta_coeff, s_coeff;
    int ntab;
};

// UNI: every particle has one volume, so the damage sums of a stencil row
// are vol_sums[intact bonds] and vol_sums[bonds] (bit for bit the ordered
// FP64 sums), and the bond loop reads no FP64 volumes.
// LEAN: the listed warps are all of kinds 2 and 3 (the split form's first
// launch), so the per-bond-code branch is not compiled in.
// 4-bond chunks: on the full plate (B200, ms per energy read) 3.35 with UNI
// and 3.87 without, against 4.03 / 4.32 in 8-bond chunks (which spill at 64
// registers) and 3.53 / 4.03 in 4-bond chunks at 3 blocks per SM.
template <bool LPS, int INFL, bool FRACTURE, bool UNI = false, bool LEAN = false>
__global__ void __launch_bounds__(kBlock, 4)
    k_energy_mixed(ParticleView p, EllView nl, MixedView mv, MixedEnergy md, double* partials,
                   const int32_t* __restrict__ wlist, int64_t wcount,
                   const double* __restrict__ vol_sums)
{
    extern __shared__ MixedStencil smem[];
    __shared__ double s_phi[kBlock];
    __shared__ double s_dmg[kBlock];
    for (int t = threadIdx.x; t < md.ntab; t += blockDim.x) smem[t] = mv.table[t];
    __syncthreads();
    // Rows: the listed warps' chunks when a warp list is given (a slot past
    // its end holds no row), else consecutive rows.
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    bool listed = true;
    if (wlist) {
        const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
        listed = slot < wcount;
        warp = listed ? wlist[slot] : 0;
    }
    const int64_t i = listed ? p.frozen + 32 * warp + (threadIdx.x & 31) : p.n;
    const int kind =
        (listed && warp < ((p.n - p.frozen + 31) >> 5)) ? mv.warp_kind[warp] : 0;
    const MixedStencil* wt = smem;
    int wcnt = md.ntab;
    if (kind == 3) {
        const int lane = threadIdx.x & 31;
        const int nmask = (md.ntab + 31) / 32;
        MixedStencil* mine = smem + md.ntab * (1 + (threadIdx.x >> 5));
        const uint32_t* wm = mv.warp_pmask + warp * nmask;
        int before = 0;
        for (int w = 0; w < nmask; ++w) {
            const uint32_t pm = wm[w];
            if ((pm >> lane) & 1u)
                mine[before + __popc(pm & ((1u << lane) - 1u))] = smem[32 * w + lane];
            before += __popc(pm);
        }
        __syncwarp();
        wt = mine;
        wcnt = before;
    }
    double Phi_i = 0.0, dmg_i = 0.0;
    if (i < p.n) {
        const int64_t np = p.npad;
        const int cnt = nl.count[i];
        const double vol_i = p.vol[i];
        double bonds_part = 0.0, phi_sum = 0.0, vol_H = 0.0;
        int intact_n = 0;
        if (LEAN || kind >= 2) {
            const MixedU ui = mv.u2[i];
            const RowSplit ri{f2(-ui.hi.x, -ui.hi.y), f2(-ui.lo.x, -ui.lo.y), -ui.hi.z,
                              -ui.lo.z, false};
            const MixedU* __restrict__ u2_i = mv.u2 + i;
            // One bond: its energy term (zero when broken) into the FP32
            // chunk, and (fracture) its FP64 volume into the damage sums.
            auto bond = [&](const MixedStencil& t, bool on, float& chunk) {
                if (FRACTURE && !UNI) {
                    const double vol_j = __ldg(p.vol + i + t.delta);
                    phi_sum += on ? vol_j : 0.0;
                    vol_H += vol_j;
                }
                intact_n += on ? 1 : 0;
                const MixedU uj = u2_i[t.delta];
                MixedBond2 bd;
                lean_geometry(t, uj, ri, bd);
                // PMB: the w lane holds c vol_j; LPS: vol_j.
                const float term = LPS ? (INFL == 1 ? t.xi : t.xi2) * uj.hi.w * bd.s * bd.s
                                       : 0.25f * uj.hi.w * bd.s * bd.s * t.xi;
                chunk += on ? term : 0.f;
            };
            for (int base = 0; base < wcnt; base += 32) {
                const uint32_t word =
                    FRACTURE ? nl.mu[(int64_t)(base >> 5) * np + i] : 0xffffffffu;
                const int lim = min(32, wcnt - base);
                int b = 0;
                for (; b + 4 <= lim; b += 4) {
                    const uint32_t w4 = word >> b;
                    float chunk = 0.f;
#pragma unroll
                    for (int u = 0; u < 4; ++u) bond(wt[base + b + u], (w4 >> u) & 1u, chunk);
                    bonds_part += (double)chunk;
                }
                if (b < lim) {
                    float chunk = 0.f;
                    for (; b < lim; ++b) bond(wt[base + b], (word >> b) & 1u, chunk);
                    bonds_part += (double)chunk;
                }
            }
            if (FRACTURE && UNI) {
                phi_sum = vol_sums[intact_n];
                vol_H = vol_sums[wcnt];
            }
        } else if (!LEAN) {
            // Per-bond codes: a bond on a stencil entry takes the FP32 form
            // of the stencil rows (its term into 4-bond FP32 chunks), any
            // other bond the FP64 form. With one particle volume the damage
            // sums come from vol_sums, so no FP64 volume is read per bond.
            const double xi0 = p.x[i], xi1 = p.x[np + i], xi2 = p.x[2 * np + i];
            const double ui0 = p.u[i], ui1 = p.u[np + i], ui2 = p.u[2 * np + i];
            const MixedU ui = mv.u2[i];
            const RowSplit ri{f2(-ui.hi.x, -ui.hi.y), f2(-ui.lo.x, -ui.lo.y), -ui.hi.z,
                              -ui.lo.z, false};
            const MixedU* __restrict__ u2_i = mv.u2 + i;
            float chunk = 0.f;
            int in_chunk = 0;
            uint32_t word = 0xffffffffu;
            for (int k = 0; k < cnt; ++k) {
                if (FRACTURE && (k & 31) == 0) word = nl.mu[(int64_t)(k >> 5) * np + i];
                const bool on = (word >> (k & 31)) & 1u;
                if (FRACTURE && !UNI) {
                    const double vol_j = __ldg(p.vol + __ldg(nl.idx + (int64_t)k * np + i));
                    phi_sum += on ? vol_j : 0.0;
                    vol_H += vol_j;
                }
                if (!on) continue;
                ++intact_n;
                const uint8_t code = mv.code[(int64_t)k * np + i];
                if (code < md.ntab) {
                    const MixedStencil& t = smem[code];
                    const MixedU uj = u2_i[t.delta];
                    MixedBond2 bd;
                    lean_geometry(t, uj, ri, bd);
                    chunk += LPS ? (INFL == 1 ? t.xi : t.xi2) * uj.hi.w * bd.s * bd.s
                                 : 0.25f * uj.hi.w * bd.s * bd.s * t.xi;
                    if (++in_chunk == 4) {
                        bonds_part += (double)chunk;
                        chunk = 0.f;
                        in_chunk = 0;
                    }
                    continue;
                }
                const int64_t j = __ldg(nl.idx + (int64_t)k * np + i);
                const double vol_j = __ldg(p.vol + j);
                const double xx = __ldg(p.x + j) - xi0, xy = __ldg(p.x + np + j) - xi1,
                             xz = __ldg(p.x + 2 * np + j) - xi2;
                const double rx = xx + (__ldg(p.u + j) - ui0);
                const double ry = xy + (__ldg(p.u + np + j) - ui1);
                const double rz = xz + (__ldg(p.u + 2 * np + j) - ui2);
                const double r = sqrt(rx * rx + ry * ry + rz * rz);
                const double xi = sqrt(xx * xx + xy * xy + xz * xz);
                const double sv = (r - xi) / xi;
                bonds_part += LPS ? (INFL == 1 ? xi : xi * xi) * vol_j * sv * sv
                                  : 0.25 * md.c * vol_j * sv * sv * xi;
            }
            bonds_part += (double)chunk;
            if (FRACTURE && UNI) {
                phi_sum = vol_sums[intact_n];
                vol_H = vol_sums[cnt];
            }
        }
        double Wi;
        if (LPS) {
            const double th_i = p.theta[i];
            Wi = (intact_n > 0 ? 0.5 * md.theta_coeff / 3.0 * (th_i * th_i) : 0.0) +
                 0.5 * (md.s_coeff / p.m[i]) * bonds_part;
        } else {
            Wi = bonds_part;
        }
        p.W[i] = Wi;
        if (FRACTURE) {
            dmg_i = 1 - phi_sum / vol_H;
            p.phi[i] = dmg_i;
        }
        Phi_i = Wi * vol_i;
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

// Batched step over many systems (cpd_batch.cu), mixed bodies: as
// k_batch_fast, and the instance's stencil table is staged in shared memory
// with its table entry. Pass 0: LPS weighted volume (fracture) and
// dilatation; pass 1: bond force and step epilogue.
__global__ void __launch_bounds__(kBlock, 3)
    k_batch_mixed(const BatchInstance* __restrict__ insts, const int32_t* __restrict__ remaining,
                  const BatchTile* __restrict__ tiles, int32_t ntiles, int32_t K, int32_t s,
                  int32_t pass)
{
    static_assert(sizeof(BatchInstance) % 4 == 0 && sizeof(BatchInstance) <= 4 * kBlock,
                  "instance entry staged by one word per thread");
    __shared__ __align__(16) uint32_t dbuf[sizeof(BatchInstance) / 4];
    __shared__ MixedStencil tab[kMixedGeneric];
    BatchInstance& d = *reinterpret_cast<BatchInstance*>(dbuf);
    const int w = threadIdx.x >> 5;
    int32_t loaded = -1;
    for (int32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const BatchTile tl = tiles[t];
        if (pass == 0 && !tl.lps) continue;
        const BatchStep bs = batch_step(remaining[tl.inst], K, s);
        if (!bs.run) continue;
        if (tl.inst != loaded) {
            __syncthreads();
            const BatchInstance* src = insts + tl.inst;
            if (threadIdx.x < sizeof(BatchInstance) / 4)
                dbuf[threadIdx.x] = reinterpret_cast<const uint32_t*>(src)[threadIdx.x];
            const int ntab = src->pd == CPD_PD_PMB ? src->mm.ntab : src->ml.ntab;
            const MixedStencil* table = src->mv.table;
            for (int k = threadIdx.x; k < ntab; k += blockDim.x) tab[k] = table[k];
            __syncthreads();
            if (threadIdx.x == 0) {
                // This step's buffers (as k_batch_fast), and the split's.
                double* const u0 = d.p.u;
                MixedU* const s0 = const_cast<MixedU*>(d.mv.u2);
                d.p.u = bs.cur ? d.u_alt : u0;
                d.mv.u2 = bs.cur ? d.u2_alt : s0;
                d.ep.u_next = bs.cur ? u0 : d.u_alt;
                d.ep.u2_next = bs.cur ? s0 : d.u2_alt;
                d.ep.mode = bs.mode;
            }
            __syncthreads();
            loaded = tl.inst;
        }
        if (w >= tl.nwarps) continue;
        const int64_t warp = tl.warp0 + w;
        const int64_t i = d.p.frozen + 32 * warp + (threadIdx.x & 31);
        if (i >= d.p.n) continue;
        const bool infl = d.influence == 1;
        if (pass == 0) {
            if (d.fracture) {
                if (infl)
                    lps_mtheta_mixed_row<true, 1, true>(d.p, d.nl, d.mv, tab, d.ml, d.ab,
                                                        nullptr, warp, i);
                else
                    lps_mtheta_mixed_row<true, 0, true>(d.p, d.nl, d.mv, tab, d.ml, d.ab,
                                                        nullptr, warp, i);
            } else {
                if (infl)
                    lps_mtheta_mixed_row<false, 1, false>(d.p, d.nl, d.mv, tab, d.ml, d.ab,
                                                          nullptr, warp, i);
                else
                    lps_mtheta_mixed_row<false, 0, false>(d.p, d.nl, d.mv, tab, d.ml, d.ab,
                                                          nullptr, warp, i);
            }
            continue;
        }
        if (d.pd == CPD_PD_PMB) {
            if (d.fracture) pmb_mixed_row<true>(d.p, d.nl, d.mv, tab, d.mm, d.ep, warp, i);
            else pmb_mixed_row<false>(d.p, d.nl, d.mv, tab, d.mm, d.ep, warp, i);
        } else if (infl) {
            if (d.fracture)
                lps_force_mixed_row<true, 1>(d.p, d.nl, d.mv, tab, d.ml, d.ab, d.ep, warp, i);
            else
                lps_force_mixed_row<false, 1>(d.p, d.nl, d.mv, tab, d.ml, d.ab, d.ep, warp, i);
        } else {
            if (d.fracture)
                lps_force_mixed_row<true, 0>(d.p, d.nl, d.mv, tab, d.ml, d.ab, d.ep, warp, i);
            else
                lps_force_mixed_row<false, 0>(d.p, d.nl, d.mv, tab, d.ml, d.ab, d.ep, warp, i);
        }
    }
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
    free_stencil64(m, st);
    delete m.st32;
    m.st32 = nullptr;
    void* ptrs[] = {m.xh, m.xl, m.u2_base, m.code, m.table, m.warp_kind, m.pmask, m.warp_pmask,
                    m.ab, m.lean_list, m.rest_list, m.vol_sums, m.u2ab, m.stencil_list,
                    m.irregular_list, m.gcell};
    for (void* q : ptrs)
        if (q) dev_free(q, st);
    m = MixedState{};
}

namespace {

// The FP64 stencil records' layout. When every particle sits on its own
// lattice cell of the bounding box, each table entry's delta is its cell
// delta a + nc0 (b + nc1 c): layout 1 when the particle order is one box of
// lattice lines (cell - row constant: records by row, the index deltas being
// the cell deltas), layout 2 otherwise (a body with holes or a non-box
// outline: records by lattice cell, m.gcell), so that every lattice row keeps
// the stencil kernel. Layout 0 (not a lattice of distinct cells, or too
// sparse a bounding box): deltas from the bond codes.
#define CPD_RET(call)                   \
    do {                                \
        const cudaError_t e_ = (call);  \
        if (e_ != cudaSuccess) return e_; \
    } while (0)
cudaError_t lattice_cell_layout(const ParticleView& p, const double* h,
                                const std::vector<MixedStencil>& tab, int64_t rows,
                                MixedState& m, std::vector<unsigned int>& delta, int& launches,
                                int& layout, cudaStream_t st)
{
    layout = 0;
    if (p.n <= 0 || rows <= 0) return cudaSuccess;
    // Device buffers of this test, freed on every return but the cells kept.
    struct Buffers {
        cudaStream_t st;
        unsigned long long* bounds = nullptr;
        int32_t* cell = nullptr;
        uint32_t* occ = nullptr;
        unsigned int* flags = nullptr;
        ~Buffers()
        {
            if (bounds) dev_free(bounds, st);
            if (cell) dev_free(cell, st);
            if (occ) dev_free(occ, st);
            if (flags) dev_free(flags, st);
        }
    } buf{st};
    CPD_RET(dev_alloc(&buf.bounds, sizeof(unsigned long long) * 8, st));
    const unsigned long long init[8] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull, ~0ull, 0ull};
    CPD_RET(cudaMemcpyAsync(buf.bounds, init, sizeof init, cudaMemcpyHostToDevice, st));
    const int nb = (int)std::min<int64_t>(blocks_for(p.n), 148 * 8);
    k_bounds<<<nb, kBlock, 0, st>>>(p.x, p.n, p.npad, buf.bounds);
    launches++;
    unsigned long long hb[8];
    CPD_RET(cudaMemcpyAsync(hb, buf.bounds, sizeof hb, cudaMemcpyDeviceToHost, st));
    CPD_RET(cudaStreamSynchronize(st));
    auto from_bits = [](unsigned long long k) {
        const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double v;
        std::memcpy(&v, &b, sizeof v);
        return v;
    };
    double lo[3];
    int64_t nc[3];
    for (int d = 0; d < 3; ++d) {
        lo[d] = from_bits(hb[d]);
        nc[d] = (int64_t)std::llround((from_bits(hb[3 + d]) - lo[d]) / h[d]) + 1;
    }
    const int64_t cells = nc[0] * nc[1] * nc[2];
    // A sparse outline would need too many empty records.
    if (cells > 4 * p.n + 4096 || cells >= ((int64_t)1 << 31)) return cudaSuccess;
    CPD_RET(dev_alloc(&buf.cell, sizeof(int32_t) * (size_t)p.npad, st));
    CPD_RET(dev_alloc(&buf.occ, sizeof(uint32_t) * (size_t)cells, st));
    CPD_RET(dev_alloc(&buf.flags, sizeof(unsigned int) * 2, st));
    CPD_RET(cudaMemsetAsync(buf.occ, 0, sizeof(uint32_t) * (size_t)cells, st));
    CPD_RET(cudaMemsetAsync(buf.flags, 0, sizeof(unsigned int) * 2, st));
    k_lattice_cells<<<blocks_for(p.n), kBlock, 0, st>>>(
        p.x, p.n, p.npad, make_double3(lo[0], lo[1], lo[2]),
        make_double3(1.0 / h[0], 1.0 / h[1], 1.0 / h[2]),
        make_int3((int)nc[0], (int)nc[1], (int)nc[2]), buf.cell, buf.occ, buf.flags,
        buf.bounds + 6);
    launches++;
    unsigned int hf[2];
    CPD_RET(cudaMemcpyAsync(hf, buf.flags, sizeof hf, cudaMemcpyDeviceToHost, st));
    CPD_RET(cudaMemcpyAsync(hb + 6, buf.bounds + 6, sizeof(unsigned long long) * 2,
                            cudaMemcpyDeviceToHost, st));
    CPD_RET(cudaStreamSynchronize(st));
    // Off the lattice, or two particles in a cell.
    if (hf[0] != 0u || hf[1] != 0u) return cudaSuccess;
    if (hb[6] == hb[7]) {
        // One box in row order: records by row, whose index deltas are the
        // cell deltas.
        layout = 1;
    } else {
        m.gcell = buf.cell;
        buf.cell = nullptr;
        m.grid_cells = cells;
        m.bytes += sizeof(int32_t) * (size_t)p.npad;
        layout = 2;
    }
    for (size_t t = 0; t < tab.size(); ++t) {
        const long long a = std::llround(tab[t].x / h[0]);
        const long long b = std::llround(tab[t].y / h[1]);
        const long long c = std::llround(tab[t].z / h[2]);
        delta[t] = (unsigned int)(a + nc[0] * (b + nc[1] * c) + (1LL << 31));
    }
    return cudaSuccess;
}

#undef CPD_RET
}  // namespace

int lattice_layout_probe(const ParticleView& p, const double* h, cudaStream_t st)
{
    // The layout test alone: no table deltas are kept and the system's
    // state is left as it was.
    MixedState probe;
    std::vector<MixedStencil> none;
    std::vector<unsigned int> delta;
    int launches = 0, layout = 0;
    const cudaError_t e = lattice_cell_layout(p, h, none, p.n - p.frozen, probe, delta,
                                              launches, layout, st);
    if (probe.gcell) dev_free(probe.gcell, st);
    return e == cudaSuccess ? layout : 0;
}

int lattice_table_entries(const double* h, double cutoff)
{
    int half[3];
    for (int d = 0; d < 3; ++d) {
        if (!(h[d] > 1e-6 * cutoff) || !std::isfinite(h[d])) return 0;
        half[d] = (int)std::floor(cutoff / h[d] + 1e-9);
    }
    int n = 0;
    for (int c = -half[2]; c <= half[2]; ++c)
        for (int b = -half[1]; b <= half[1]; ++b)
            for (int a = -half[0]; a <= half[0]; ++a) {
                if (a == 0 && b == 0 && c == 0) continue;
                const double vx = a * h[0], vy = b * h[1], vz = c * h[2];
                if (std::sqrt(vx * vx + vy * vy + vz * vz) <= cutoff * (1.0 + 1e-9) &&
                    ++n > kStencilMaxWide)
                    return n;  // past every table: the count no longer matters
            }
    return n;
}

int prepare_mixed(const ParticleView& p, const NeighborList& pd, double cutoff, bool lps,
                  MixedState& m, cudaStream_t st, std::string& err, const Model* fp64_stencil,
                  const Model* md_pmb)
{
    int launches = 0;
    PhaseTrace tr("mixed");
    free_mixed(m, st);
    const int64_t np = p.npad;
    // The FP64 stencil path needs the table, masks and warp lists only.
    const bool fp32 = fp64_stencil == nullptr;
    if (fp32) {
        CPD_TRY(dev_alloc(&m.xh, sizeof(float4) * np, st));
        CPD_TRY(dev_alloc(&m.xl, sizeof(float4) * np, st));
        m.bytes = 2 * sizeof(float4) * np;
    }
    CPD_TRY(dev_alloc(&m.table, sizeof(MixedStencil) * kMixedGeneric, st));
    CPD_TRY(dev_alloc(&m.code, (size_t)std::max(pd.max_n, 1) * np, st));
    const int64_t nwarps = (np + 31) / 32 + 8;
    CPD_TRY(dev_alloc(&m.warp_kind, nwarps, st));
    m.bytes += sizeof(MixedStencil) * kMixedGeneric + (size_t)std::max(pd.max_n, 1) * np + nwarps;
    CPD_TRY(cudaMemsetAsync(m.warp_kind, 0, nwarps, st));
    CPD_TRY(cudaMemsetAsync(m.code, kMixedGeneric, (size_t)std::max(pd.max_n, 1) * np, st));
    if (fp32) {
        k_split<<<blocks_for(p.n), kBlock, 0, st>>>(p.x, p.n, np, m.xh, m.xl);
        launches++;
    }
    tr.mark("alloc+split", st);
    m.ntab = 0;
    const int64_t rows = p.n - p.frozen;
    if (rows > 0 && pd.max_n > 0) {
        unsigned long long* d_min = nullptr;
        CPD_TRY(dev_alloc(&d_min, 4 * sizeof(unsigned long long), st));
        CPD_TRY(cudaMemsetAsync(d_min, 0x7f, 3 * sizeof(unsigned long long), st));
        CPD_TRY(cudaMemsetAsync(d_min + 3, 0, sizeof(unsigned long long), st));
        // The neighbour build's count pass may have found the spacing already
        // (over the pairs it visited, which are the list's pairs). With
        // CPD_CHECK_SPACING=1 the list is walked anyway and the two must agree
        // bit for bit: a debug check that the list holds exactly those pairs.
        const char* chk = getenv("CPD_CHECK_SPACING");
        const bool check = pd.hmin_valid && chk && chk[0] == '1';
        if (!pd.hmin_valid || check) {
            k_min_spacing<<<blocks_for(rows), kBlock, 0, st>>>(p, pd.view(), d_min);
            launches++;
        }
        k_vol_uniform<<<blocks_for(p.n), kBlock, 0, st>>>(p.vol, p.n, d_min + 3);
        launches++;
        unsigned long long hmin[4];
        double v0 = 0.0;
        CPD_TRY(cudaMemcpyAsync(hmin, d_min, sizeof(hmin), cudaMemcpyDeviceToHost, st));
        CPD_TRY(cudaMemcpyAsync(&v0, p.vol, sizeof(double), cudaMemcpyDeviceToHost, st));
        CPD_TRY(cudaStreamSynchronize(st));
        CPD_TRY(dev_free(d_min, st));
        if (check) {
            for (int d = 0; d < 3; ++d) {
                if (std::memcmp(&hmin[d], &pd.hmin[d], sizeof(double)) != 0) {
                    err = "lattice spacing of the count pass differs from the list's on axis " +
                          std::to_string(d);
                    return -1;
                }
            }
        }
        if (pd.hmin_valid)
            for (int d = 0; d < 3; ++d) std::memcpy(&hmin[d], &pd.hmin[d], sizeof(double));
        if (hmin[3] == 0) {
            // The damage sums of the energy pass then depend only on how
            // many bonds are summed (in order, each adding v).
            std::vector<double> sums((size_t)pd.max_n + 1, 0.0);
            for (int k = 1; k <= pd.max_n; ++k) sums[k] = sums[k - 1] + v0;
            CPD_TRY(dev_alloc(&m.vol_sums, sizeof(double) * sums.size(), st));
            CPD_TRY(cudaMemcpyAsync(m.vol_sums, sums.data(), sizeof(double) * sums.size(),
                                    cudaMemcpyHostToDevice, st));
            m.bytes += sizeof(double) * sums.size();
            m.vol_uniform = v0;
        }
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
                        // Codes are bytes below kMixedGeneric; the FP64
                        // stencil path codes rows from the positions and
                        // takes up to kStencilMaxWide entries.
                        if ((int)tab.size() >= (fp32 ? kMixedGeneric : kStencilMaxWide)) {
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
                        e.xi2 = (float)(len * len);
                        e.delta = 0;
                        e.pad = 0;
                        tab.push_back(e);
                    }
            // FP64: when every particle sits on its own lattice cell, each
            // entry's delta comes from the geometry and rows are coded from
            // the positions (no per-bond codes); else the byte codes below.
            // The mixed path takes the geometric deltas of a box in row
            // order too (its FP32 records go by row), coding each bond in the
            // mask pass itself.
            int layout = 0;
            std::vector<unsigned int> delta(kDeltaSlots, 0xffffffffu);
            if (lattice && !tab.empty())
                CPD_TRY(lattice_cell_layout(p, h, tab, rows, m, delta, launches, layout, st));
            if (fp32 && layout == 2) {
                CPD_TRY(dev_free(m.gcell, st));
                m.gcell = nullptr;
                m.grid_cells = 0;
                m.bytes -= sizeof(int32_t) * (size_t)p.npad;
                layout = 0;
                std::fill(delta.begin(), delta.end(), 0xffffffffu);
            }
            const bool by_codes = layout == 0;
            if (by_codes && (int)tab.size() >= kMixedGeneric) lattice = false;
            if (lattice && !tab.empty()) {
                int16_t* d_lut = nullptr;
                unsigned int* d_delta = nullptr;
                CPD_TRY(dev_alloc(&d_lut, sizeof(int16_t) * lut.size(), st));
                CPD_TRY(dev_alloc(&d_delta, sizeof(unsigned int) * kDeltaSlots, st));
                CPD_TRY(cudaMemcpyAsync(d_lut, lut.data(), sizeof(int16_t) * lut.size(),
                                        cudaMemcpyHostToDevice, st));
                CPD_TRY(cudaMemcpyAsync(d_delta, delta.data(), sizeof(unsigned int) * kDeltaSlots,
                                        cudaMemcpyHostToDevice, st));
                LatticeLut L;
                for (int d = 0; d < 3; ++d) {
                    L.h[d] = h[d];
                    L.hinv[d] = 1.0 / h[d];
                    L.half[d] = half[d];
                }
                L.lut = d_lut;
                tr.mark("spacing+table", st);
                if (by_codes) {
                    k_code_bonds<<<blocks_for(rows), kBlock, 0, st>>>(p, pd.view(), L, m.code,
                                                                      d_delta);
                    launches++;
                    tr.mark("code", st);
                    CPD_TRY(cudaMemcpyAsync(delta.data(), d_delta,
                                            sizeof(unsigned int) * kMixedGeneric,
                                            cudaMemcpyDeviceToHost, st));
                    {
                        // Each code's index delta is the one most of 256 rows spread
                        // over the body hold (the minimum over all bonds where no
                        // sample holds the code). In a body with voids or holes the
                        // rows whose neighbours lie across one see shifted deltas;
                        // the minimum would take a shifted one and leave every other
                        // row irregular.
                        const int S = (int)std::min<int64_t>(256, rows);
                        const int mn = std::max(pd.max_n, 1);
                        if (S > 0) {
                            int2* d_samp = nullptr;
                            CPD_TRY(dev_alloc(&d_samp, sizeof(int2) * (size_t)S * mn, st));
                            k_sample_rows<<<S, kBlock, 0, st>>>(pd.view(), np, m.code, p.frozen,
                                                                rows, S, d_samp);
                            launches++;
                            std::vector<int2> samp((size_t)S * mn);
                            CPD_TRY(cudaMemcpyAsync(samp.data(), d_samp, sizeof(int2) * samp.size(),
                                                    cudaMemcpyDeviceToHost, st));
                            CPD_TRY(cudaStreamSynchronize(st));
                            CPD_TRY(dev_free(d_samp, st));
                            std::vector<std::vector<int>> seen(tab.size());
                            for (const int2& v : samp)
                                if (v.x < (int)tab.size()) seen[v.x].push_back(v.y);
                            for (size_t t = 0; t < tab.size(); ++t) {
                                std::vector<int>& d = seen[t];
                                if (d.empty()) continue;
                                std::sort(d.begin(), d.end());
                                int best = d[0], run = 0, best_run = 0;
                                for (size_t q = 0; q < d.size(); ++q) {
                                    run = (q > 0 && d[q] == d[q - 1]) ? run + 1 : 1;
                                    if (run > best_run) {
                                        best_run = run;
                                        best = d[q];
                                    }
                                }
                                delta[t] = (unsigned int)((long long)best + (1LL << 31));
                            }
                            CPD_TRY(cudaMemcpyAsync(d_delta, delta.data(),
                                                    sizeof(unsigned int) * kMixedGeneric,
                                                    cudaMemcpyHostToDevice, st));
                        }
                    }
                }
                CPD_TRY(cudaStreamSynchronize(st));
                for (size_t t = 0; t < tab.size(); ++t)
                    tab[t].delta = (int32_t)((long long)delta[t] - (1LL << 31));
                if (fp32)
                    CPD_TRY(cudaMemcpyAsync(m.table, tab.data(),
                                            sizeof(MixedStencil) * tab.size(),
                                            cudaMemcpyHostToDevice, st));
                CPD_TRY(cudaStreamSynchronize(st));
                m.ntab = (int)tab.size();
                for (int d = 0; d < 3; ++d) m.h[d] = h[d];
                const int nmask = (m.ntab + 31) / 32;
                CPD_TRY(dev_alloc(&m.pmask, sizeof(uint32_t) * nmask * np, st));
                m.bytes += sizeof(uint32_t) * nmask * np;
                CPD_TRY(dev_alloc(&m.warp_pmask, sizeof(uint32_t) * nmask * nwarps, st));
                m.bytes += sizeof(uint32_t) * nmask * nwarps;
                if (by_codes)
                    k_row_masks<false><<<blocks_for(rows), kBlock, 0, st>>>(
                        p, pd.view(), d_delta, m.code, m.ntab, m.pmask, m.warp_kind,
                        m.warp_pmask, m.gcell, L);
                else
                    k_row_masks<true><<<blocks_for(rows), kBlock, 0, st>>>(
                        p, pd.view(), d_delta, fp32 ? m.code : nullptr, m.ntab, m.pmask,
                        m.warp_kind, m.warp_pmask, m.gcell, L);
                launches++;
                CPD_TRY(dev_free(d_lut, st));
                CPD_TRY(dev_free(d_delta, st));
                tr.mark("masks", st);
                const int64_t nw = (rows + 31) / 32;
                std::vector<uint8_t> kinds(nw);
                CPD_TRY(cudaMemcpyAsync(kinds.data(), m.warp_kind, nw, cudaMemcpyDeviceToHost,
                                        st));
                CPD_TRY(cudaStreamSynchronize(st));
                if (lps) {
                    // The LPS kernels take stencil rows only: every warp of rows
                    // must be a stencil kind (1, 2 or 3).
                    m.lps_ok = std::all_of(kinds.begin(), kinds.end(),
                                           [](uint8_t k) { return k != 0; }) ? 1 : 0;
                    if (m.lps_ok) {
                        CPD_TRY(dev_alloc(&m.ab, sizeof(float2) * np, st));
                        m.bytes += sizeof(float2) * np;
                        if (m.vol_sums && p.frozen == 0) {
                            CPD_TRY(dev_alloc(&m.u2ab, sizeof(MixedU) * np, st));
                            m.bytes += sizeof(MixedU) * np;
                        }
                    }
                }
                {
                    // Warp lists, each in the tile order of tile_chunk: warps
                    // of kinds 2 and 3 and the rest (the split mixed forms);
                    // warps of kinds 1-3 and of kind 0 (the stencil kernels).
                    int g = 0;
                    const EllView tv = tile_view(pd.view(), rows, kBlock, &g);
                    const int64_t S = tv.stride, W = kBlock / 32;
                    std::vector<int32_t> lean, rest, sten, irr;
                    lean.reserve(nw);
                    sten.reserve(nw);
                    for (int64_t b = 0; b < g; ++b)
                        for (int64_t w = 0; w < W; ++w) {
                            const int64_t q = S > 1 ? (W * (b / S) + w) * S + b % S : W * b + w;
                            if (q >= nw) continue;
                            (kinds[q] >= 2 ? lean : rest).push_back((int32_t)q);
                            (kinds[q] >= 1 ? sten : irr).push_back((int32_t)q);
                        }
                    auto upload = [&](const std::vector<int32_t>& v, int32_t** dst,
                                      int64_t* count) -> bool {
                        *count = (int64_t)v.size();
                        if (v.empty()) return true;
                        if (dev_alloc(dst, sizeof(int32_t) * v.size(), st) != cudaSuccess)
                            return false;
                        m.bytes += sizeof(int32_t) * v.size();
                        return cudaMemcpyAsync(*dst, v.data(), sizeof(int32_t) * v.size(),
                                               cudaMemcpyHostToDevice, st) == cudaSuccess;
                    };
                    if (!upload(lean, &m.lean_list, &m.nlean) ||
                        !upload(rest, &m.rest_list, &m.nrest) ||
                        !upload(sten, &m.stencil_list, &m.nstencil) ||
                        !upload(irr, &m.irregular_list, &m.nirregular)) {
                        err = "warp lists: " + std::string(cudaGetErrorString(cudaGetLastError()));
                        return -1;
                    }
                    CPD_TRY(cudaStreamSynchronize(st));
                }
                if (fp32 && !lps && md_pmb)
                    prepare_stencil32(*md_pmb, h, tab.data(), m.ntab, m);
                if (!fp32) {
                    if (!prepare_stencil64(p, *fp64_stencil, h, tab.data(), m.ntab, m, st, err) &&
                        !err.empty())
                        return -1;
                    launches += m.u4 ? 1 : 0;
                    // The FP64 kernels read no bond codes.
                    CPD_TRY(dev_free(m.code, st));
                    m.code = nullptr;
                    m.bytes -= (size_t)std::max(pd.max_n, 1) * np;
                }
            }
        }
    }
    if (fp32) {
        // The split of u, with zero guard records on either side for the
        // stencil kernel's reads at i + delta of absent entries.
        if (!m.st32) m.guard = 0;
        const size_t recs = (size_t)(np + 2 * m.guard);
        CPD_TRY(dev_alloc(&m.u2_base, sizeof(MixedU) * recs, st));
        CPD_TRY(cudaMemsetAsync(m.u2_base, 0, sizeof(MixedU) * recs, st));
        m.u2 = m.u2_base + m.guard;
        m.bytes += sizeof(MixedU) * recs;
    }
    CPD_TRY(cudaGetLastError());
    tr.mark("lists", st);
    return launches;
}

// Scale of the volume in the w lane of the displacement split: the PMB
// micromodulus (its force is c s vol_j / r), 1 for LPS.
double mixed_wscale(const Model& md) { return md.pd == CPD_PD_PMB ? md.c : 1.0; }

int launch_split_u(const ParticleView& p, const Model& md, MixedState& m, cudaStream_t st)
{
    if (p.n <= 0) return 0;
    k_split_u<<<blocks_for(p.n), kBlock, 0, st>>>(p, mixed_wscale(md), m.u2);
    return 1;
}

int launch_vv_initial_mixed(const ParticleView& p, const Model& md, double dt, double* u_out,
                            MixedU* u2_out, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    k_vv_initial_mixed<<<blocks_for(rows), kBlock, 0, st>>>(p, dt, 0.5 * dt, mixed_wscale(md),
                                                            u_out, u2_out);
    return 1;
}

MixedModel to_mixed_model(const Model& md, const MixedState& m)
{
    MixedModel mm;
    mm.c = (float)md.c;
    mm.s0 = (float)md.s0;
    mm.guard = (float)(1e-4 * md.s0);
    mm.bbc = md.bond_break_coeff;
    mm.s_lo = mm.s0 - mm.guard;
    mm.s_hi = mm.s0 + mm.guard;
    mm.ntab = m.ntab;
    return mm;
}

int launch_batch_mixed(const BatchInstance* inst, const int32_t* remaining,
                       const BatchTile* tiles, int32_t ntiles, int32_t K, int32_t s,
                       int32_t pass, int grid, cudaStream_t st)
{
    if (ntiles <= 0 || grid <= 0) return 0;
    k_batch_mixed<<<grid, kBlock, 0, st>>>(inst, remaining, tiles, ntiles, K, s, pass);
    return 1;
}

int batch_mixed_blocks_per_sm()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_mixed, kBlock, 0) !=
        cudaSuccess)
        n = 1;
    return n > 0 ? n : 1;
}

MixedLps to_mixed_lps(const Model& md, const MixedState& m)
{
    MixedLps l;
    l.s0 = (float)md.s0;
    l.guard = (float)(1e-4 * md.s0);
    l.s_lo = l.s0 - l.guard;
    l.s_hi = l.s0 + l.guard;
    l.bbc = md.bond_break_coeff;
    l.theta_coeff = md.theta_coeff;
    l.s_coeff = md.s_coeff;
    l.ntab = m.ntab;
    l.vol = (float)(mixed_wscale(md) * m.vol_uniform);
    return l;
}

int launch_lps_mtheta_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                            const MixedState& m, bool with_m, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const MixedView mv{m.xh, m.xl, m.u2, m.code, m.table, m.warp_kind, m.pmask, m.warp_pmask};
    const MixedLps l = to_mixed_lps(md, m);
    const size_t lean_bytes = (1 + kBlock / 32) * sizeof(MixedStencil) * m.ntab;
    const bool split = m.lean_list && lean_bytes <= 48 * 1024 &&
                       rows >= split_min_rows();
    const int key = (md.fracture ? 4 : 0) + (md.influence == 1 ? 2 : 0) + (with_m ? 1 : 0);
    int n = 0;
    if (split) {
        const int gl = (int)((m.nlean + kBlock / 32 - 1) / (kBlock / 32));
#define CPD_MT_LEAN(F, I, W)                                                                \
    k_lps_mtheta_lean<F, I, W><<<gl, kBlock, lean_bytes, st>>>(p, nl, mv, l, m.ab, m.lean_list, \
                                                               m.nlean, m.u2ab)
        switch (key) {
        case 0: CPD_MT_LEAN(false, 0, false); break;
        case 1: CPD_MT_LEAN(false, 0, true); break;
        case 2: CPD_MT_LEAN(false, 1, false); break;
        case 3: CPD_MT_LEAN(false, 1, true); break;
        case 4: CPD_MT_LEAN(true, 0, false); break;
        case 5: CPD_MT_LEAN(true, 0, true); break;
        case 6: CPD_MT_LEAN(true, 1, false); break;
        default: CPD_MT_LEAN(true, 1, true); break;
        }
#undef CPD_MT_LEAN
        ++n;
        if (m.nrest == 0) return n;
    }
    const int32_t* list = split ? m.rest_list : nullptr;
    const int64_t count = split ? m.nrest : 0;
    const int g = split ? (int)((m.nrest + kBlock / 32 - 1) / (kBlock / 32)) : blocks_for(rows);
#define CPD_MT(F, I, W) \
    k_lps_mtheta_mixed<F, I, W><<<g, kBlock, 0, st>>>(p, nl, mv, l, m.ab, list, count, m.u2ab)
    switch (key) {
    case 0: CPD_MT(false, 0, false); break;
    case 1: CPD_MT(false, 0, true); break;
    case 2: CPD_MT(false, 1, false); break;
    case 3: CPD_MT(false, 1, true); break;
    case 4: CPD_MT(true, 0, false); break;
    case 5: CPD_MT(true, 0, true); break;
    case 6: CPD_MT(true, 1, false); break;
    default: CPD_MT(true, 1, true); break;
    }
#undef CPD_MT
    return n + 1;
}

int launch_lps_force_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                           const MixedState& m, const StepEpilogue& ep, cudaStream_t st)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    const MixedView mv{m.xh, m.xl, m.u2, m.code, m.table, m.warp_kind, m.pmask, m.warp_pmask};
    const MixedLps l = to_mixed_lps(md, m);
    const size_t lean_bytes = (1 + kBlock / 32) * sizeof(MixedStencil) * m.ntab;
    const bool split = m.lean_list && lean_bytes <= 48 * 1024 &&
                       rows >= split_min_rows();
    const int key = (md.fracture ? 2 : 0) + (md.influence == 1 ? 1 : 0);
    int n = 0;
    if (split) {
        const int gl = (int)((m.nlean + kBlock / 32 - 1) / (kBlock / 32));
#define CPD_F_LEAN(F, I)                                                                   \
    if (m.u2ab)                                                                            \
        k_lps_force_lean<F, I, true><<<gl, kBlock, lean_bytes, st>>>(                      \
            p, nl, mv, l, m.ab, ep, m.lean_list, m.nlean, m.u2ab);                         \
    else                                                                                   \
        k_lps_force_lean<F, I, false><<<gl, kBlock, lean_bytes, st>>>(                     \
            p, nl, mv, l, m.ab, ep, m.lean_list, m.nlean, m.u2ab)
        switch (key) {
        case 0: CPD_F_LEAN(false, 0); break;
        case 1: CPD_F_LEAN(false, 1); break;
        case 2: CPD_F_LEAN(true, 0); break;
        default: CPD_F_LEAN(true, 1); break;
        }
#undef CPD_F_LEAN
        ++n;
        if (m.nrest == 0) return n;
    }
    const int32_t* list = split ? m.rest_list : nullptr;
    const int64_t count = split ? m.nrest : 0;
    const int g = split ? (int)((m.nrest + kBlock / 32 - 1) / (kBlock / 32)) : blocks_for(rows);
#define CPD_F(F, I) k_lps_force_mixed<F, I><<<g, kBlock, 0, st>>>(p, nl, mv, l, m.ab, ep, list, count)
    switch (key) {
    case 0: CPD_F(false, 0); break;
    case 1: CPD_F(false, 1); break;
    case 2: CPD_F(true, 0); break;
    default: CPD_F(true, 1); break;
    }
#undef CPD_F
    return n + 1;
}

int launch_pd_force_mixed(const ParticleView& p, const EllView& list, const Model& md,
                          const MixedState& m, const StepEpilogue& ep, cudaStream_t st)
{
    if (md.pd == CPD_PD_LPS) return launch_lps_force_mixed(p, list, md, m, ep, st);
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    MixedView mv{m.xh, m.xl, m.u2, m.code, m.table, m.warp_kind, m.pmask, m.warp_pmask};
    const MixedModel mm = to_mixed_model(md, m);
    const size_t tab_bytes = sizeof(MixedStencil) * m.ntab;
    if (m.st32) {
        // Stencil warps on the unrolled table walk, irregular warps on the
        // general kernel.
        int n = launch_pd_force_stencil32(p, list, md, m, ep, st);
        if (m.nirregular > 0) {
            const int gr = (int)((m.nirregular + kBlock / 32 - 1) / (kBlock / 32));
            if (md.fracture)
                k_pmb_force_mixed<true><<<gr, kBlock, tab_bytes, st>>>(
                    p, list, mv, mm, ep, m.irregular_list, m.nirregular);
            else
                k_pmb_force_mixed<false><<<gr, kBlock, tab_bytes, st>>>(
                    p, list, mv, mm, ep, m.irregular_list, m.nirregular);
            ++n;
        }
        return n;
    }
    // No stencil kernel (a table over its size, or no lattice): the general
    // kernel over every row.
    const int g = blocks_for(rows);
    if (md.fracture)
        k_pmb_force_mixed<true><<<g, kBlock, tab_bytes, st>>>(p, list, mv, mm, ep, nullptr, 0);
    else
        k_pmb_force_mixed<false><<<g, kBlock, tab_bytes, st>>>(p, list, mv, mm, ep, nullptr, 0);
    return 1;
}

int launch_hertz_force_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                             bool reset, cudaStream_t st, const StepEpilogue* ep)
{
    const int64_t rows = p.n - p.frozen;
    if (rows <= 0) return 0;
    HertzMixed h;
    h.Es43 = (float)(4.0 / 3.0 * md.Es);
    h.Es2 = (float)(2.0 * md.Es);
    h.coeff_h_d = (float)md.coeff_h_d;
    h.Rs = (float)md.Rs;
    h.coeff_h_n = (float)md.coeff_h_n;
    h.sum_r = 2.0 * md.radius;
    const StepEpilogue e = ep ? *ep : StepEpilogue{};
    const int g = blocks_for(rows);
    if (ep) {
        if (md.per_particle_radius)
            k_hertz_force_mixed<true, true><<<g, kBlock, 0, st>>>(p, nl, h, true, e);
        else
            k_hertz_force_mixed<false, true><<<g, kBlock, 0, st>>>(p, nl, h, true, e);
    } else if (md.per_particle_radius) {
        k_hertz_force_mixed<true><<<g, kBlock, 0, st>>>(p, nl, h, reset, e);
    } else {
        k_hertz_force_mixed<false><<<g, kBlock, 0, st>>>(p, nl, h, reset, e);
    }
    return 1;
}

namespace {

// Energy kernel of the model over the listed warps (all rows: wlist null),
// grid blocks of 8 warps, partials per block.
void energy_mixed_launch(const ParticleView& p, const EllView& nl, const Model& md,
                         const MixedState& m, int grid, double* part, const int32_t* list,
                         int64_t count, bool lean, cudaStream_t st);

}  // namespace

int launch_energy_mixed_rows(const ParticleView& p, const EllView& nl, const Model& md,
                             const MixedState& m, const int32_t* wlist, int64_t wcount,
                             double* partials, int* launches, cudaStream_t st)
{
    *launches = 0;
    const size_t sb = (1 + kBlock / 32) * sizeof(MixedStencil) * m.ntab;
    if (m.ntab == 0 || sb > 48 * 1024 || !m.warp_kind) return -1;
    if (!(md.pd == CPD_PD_PMB || (md.pd == CPD_PD_LPS && m.lps_ok))) return -1;
    if (wcount <= 0) return 0;
    const int grid = (int)((wcount + kBlock / 32 - 1) / (kBlock / 32));
    energy_mixed_launch(p, nl, md, m, grid, partials, wlist, wcount, false, st);
    *launches = 1;
    return grid;
}

int launch_energy_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                        const MixedState& m, double* partials, int nblocks, int capacity,
                        int* launches, cudaStream_t st)
{
    *launches = 0;
    const size_t sb = (1 + kBlock / 32) * sizeof(MixedStencil) * m.ntab;
    if (m.ntab == 0 || sb > 48 * 1024 || !m.warp_kind) return -1;
    if (!(md.pd == CPD_PD_PMB || (md.pd == CPD_PD_LPS && m.lps_ok))) return -1;
    // Large systems: the lean warps in their tile order, then the others,
    // when the partials buffer holds both launches' blocks.
    const int64_t wpb = kBlock / 32;
    const int gl = (int)((m.nlean + wpb - 1) / wpb), gr = (int)((m.nrest + wpb - 1) / wpb);
    const bool split = m.lean_list && p.n - p.frozen >= split_min_rows() && gl + gr <= capacity;
    auto launch = [&](int grid, double* part, const int32_t* list, int64_t count, bool lean) {
        energy_mixed_launch(p, nl, md, m, grid, part, list, count, lean, st);
    };
    if (!split) {
        launch(nblocks, partials, nullptr, 0, false);
        *launches = 1;
        return nblocks;
    }
    launch(gl, partials, m.lean_list, m.nlean, true);
    if (gr > 0) launch(gr, partials + 2 * gl, m.rest_list, m.nrest, false);
    *launches = gr > 0 ? 2 : 1;
    return gl + gr;
}

namespace {

void energy_mixed_launch(const ParticleView& p, const EllView& nl, const Model& md,
                         const MixedState& m, int grid, double* part, const int32_t* list,
                         int64_t count, bool lean, cudaStream_t st)
{
    const size_t sb = (1 + kBlock / 32) * sizeof(MixedStencil) * m.ntab;
    const MixedView mv{m.xh, m.xl, m.u2, m.code, m.table, m.warp_kind, m.pmask, m.warp_pmask};
    const MixedEnergy e{md.c, md.theta_coeff, md.s_coeff, m.ntab};
    const int key = (md.pd == CPD_PD_LPS ? 4 : 0) + (md.influence == 1 ? 2 : 0) +
                    (md.fracture ? 1 : 0);
    const double* vs = md.fracture ? m.vol_sums : nullptr;
#define CPD_EN(L, I, F, U)                                                                   \
    if (lean)                                                                                \
        k_energy_mixed<L, I, F, U, true><<<grid, kBlock, sb, st>>>(p, nl, mv, e, part, list, \
                                                                   count, vs);               \
    else                                                                                     \
        k_energy_mixed<L, I, F, U, false><<<grid, kBlock, sb, st>>>(p, nl, mv, e, part, list, \
                                                                    count, vs)
    if (vs) {
        switch (key) {
        case 1: case 3: CPD_EN(false, 0, true, true); break;
        case 5: CPD_EN(true, 0, true, true); break;
        default: CPD_EN(true, 1, true, true); break;
        }
        return;
    }
    switch (key) {
    case 0: case 2: CPD_EN(false, 0, false, false); break;
    case 1: case 3: CPD_EN(false, 0, true, false); break;
    case 4: CPD_EN(true, 0, false, false); break;
    case 5: CPD_EN(true, 0, true, false); break;
    case 6: CPD_EN(true, 1, false, false); break;
    default: CPD_EN(true, 1, true, false); break;
    }
#undef CPD_EN
}

}  // namespace

}  // namespace cpd
