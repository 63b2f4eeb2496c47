// Plain-FP64 PMB bond kernel on the lattice stencil (CPD_FP64).
//
// On a lattice every bond of a stencil row is one entry of a table of at
// most kStencilMax lattice offsets, and the rows of a warp (kinds 1-3 of the
// stencil coding in cpd_kernels_mixed.cu) hold subsets of that table in table
// order. The kernel walks the table itself, fully unrolled, with the table in
// its parameter space: each entry's constants are immediate constant-bank
// operands, the neighbour of entry k is i + delta_k, and the displacement
// comes from 32-byte gather records (u_x, u_y, u_z, vol). No neighbour index,
// position or per-bond code is read, and no bond length is formed.
//
// Arithmetic (FP64 throughout). With eta = u_j - u_i and xi the entry's
// reference vector (the exact lattice offset),
//   num = eta . (2 xi + eta) = r^2 - xi^2            (no cancellation)
//   F   = (c vol_j / xi) (1 - xi / r) = (c vol_j / xi^3) num H(q)
// with q = num / xi^2: 1 - xi / r = 1 - (1 + q)^(-1/2) = q h(q), h(q) =
// 1 / (sqrt(1+q) (1 + sqrt(1+q))), and H interpolates h on |q| <= kStencilQ
// at Chebyshev nodes (degree kStencilPoly - 1, relative error ~2e-16 there;
// one set of coefficients for every entry). The pair force
// F r_vec, r_vec = xi + eta, equals the reference's c s vol_j r_vec / r
// (force/CabanaPD_PMB.hpp:242-279): s / r = (r - xi) / (xi r) = (1 - xi / r)
// / xi. The stretch comes without the cancellation of (r - xi) / xi, so a
// bond's force differs from the reference's by the reference's own rounding
// of r and xi (~1e-16 absolute in s); the offsets differ from x_j - x_i of
// the lattice positions by the positions' rounding (~1e-14 relative), which
// enters s only at second order.
//
// Bonds outside the polynomial's range or near the break (num within a
// band of the break stretch) are deferred: the loop only sets their bit, and
// after the table each of them takes the reference's exact FP64 expressions
// on positions and displacements (CabanaPD_ForceModels.hpp:123-128 break
// test, force/CabanaPD_PMB.hpp:259-279), so broken-bond sets equal the
// reference's for the same state. The band test compares the ordered high
// word of |num| with one integer per entry: a conservative, integer-pipe
// test that lets a bond within ~1e-6 relative of the edge take the exact
// path. The window is symmetric (|q| below the break band), so strongly
// compressed bonds take the exact path as well.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "cpd_epilogue.cuh"
#include "cpd_internal.cuh"

namespace cpd {
namespace {

constexpr int kBlock = 256;
inline int blocks_for(int64_t rows) { return (int)((rows + kBlock - 1) / kBlock); }

// High 32 bits of a double (host).
inline uint32_t hi_word(double v)
{
    uint64_t b;
    std::memcpy(&b, &v, sizeof b);
    return (uint32_t)(b >> 32);
}

// h(q) = 1 / (sqrt(1+q) (1 + sqrt(1+q))) as a polynomial of n coefficients
// on [-Q, Q] (monomial coefficients in q; long double Gaussian elimination on
// the Vandermonde system in t = q / Q at Chebyshev nodes, then scaled by
// Q^-k). Unanchored: h interpolated at n nodes. Anchored: the constant term
// is h(0) = 1/2 exactly and G(q) = (h(q) - 1/2) / q = -(s + 2) / (2 s (1 +
// s)^2), s = sqrt(1 + q), is interpolated at n - 1 nodes, so the relative
// error vanishes as q -> 0 instead of leaving a uniform bias of the size of
// the interpolation error (which the FP32 kernel's 4 coefficients would
// turn into a systematic stiffness error of ~5e-8).
// stretch: S(q) = 1 / (1 + sqrt(1+q)) instead (unanchored), so that the
// stretch is s = r / xi - 1 = q S(q).
void fit_stretch_poly(long double Q, int n, long double* out, bool anchored = false,
                      bool stretch = false)
{
    const int m = anchored ? n - 1 : n;
    long double A[kStencilPoly][kStencilPoly + 1];
    for (int r = 0; r < m; ++r) {
        const long double t = cosl(3.141592653589793238462643383279503L * (r + 0.5L) / m);
        const long double s = sqrtl(1.0L + t * Q);
        long double pw = 1.0L;
        for (int c = 0; c < m; ++c) {
            A[r][c] = pw;
            pw *= t;
        }
        A[r][m] = stretch    ? 1.0L / (1.0L + s)
                  : anchored ? -(s + 2.0L) / (2.0L * s * (1.0L + s) * (1.0L + s))
                             : 1.0L / (s * (1.0L + s));
    }
    for (int c = 0; c < m; ++c) {
        int piv = c;
        for (int r = c + 1; r < m; ++r)
            if (fabsl(A[r][c]) > fabsl(A[piv][c])) piv = r;
        for (int k = 0; k <= m; ++k) std::swap(A[c][k], A[piv][k]);
        const long double d = A[c][c];
        for (int k = 0; k <= m; ++k) A[c][k] /= d;
        for (int r = 0; r < m; ++r) {
            if (r == c) continue;
            const long double f = A[r][c];
            for (int k = 0; k <= m; ++k) A[r][k] -= f * A[c][k];
        }
    }
    const int o = anchored ? 1 : 0;
    if (anchored) out[0] = 0.5L;
    long double qk = 1.0L;
    for (int k = 0; k < m; ++k) {
        out[k + o] = A[k][m] / qk;
        qk *= Q;
    }
}

__global__ void __launch_bounds__(kBlock)
    k_pack_u4(const double* __restrict__ u, const double* __restrict__ vol, int64_t np,
              int64_t begin, int64_t end, double4* __restrict__ u4,
              const int32_t* __restrict__ cell)
{
    const int64_t i = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    u4[cell ? (int64_t)cell[i] : i] = make_double4(u[i], u[np + i], u[2 * np + i], vol[i]);
}

// The reference's exact break test and pair force of bond (i, j) from
// positions and displacements, every operation separately rounded
// (CabanaPD_Force.hpp:74-93 getDistance, CabanaPD_ForceModels.hpp:123-128,
// force/CabanaPD_PMB.hpp:259-279). Returns true when the bond breaks;
// otherwise adds its force to f.
// With w: the bond's strain energy c s^2 xi vol_j / 4 is added to *w when it
// stays intact (force/CabanaPD_PMB.hpp:127-155).
template <bool FRACTURE>
__device__ __forceinline__ bool exact_bond(const ParticleView& p, int64_t i, int64_t j, double c,
                                           double bbc, bool nofail_i, double (&f)[3],
                                           double* w)
{
    const int64_t np = p.npad;
    const double xx = __dsub_rn(p.x[j], p.x[i]);
    const double xy = __dsub_rn(p.x[np + j], p.x[np + i]);
    const double xz = __dsub_rn(p.x[2 * np + j], p.x[2 * np + i]);
    const double rx = __dadd_rn(xx, __dsub_rn(p.u[j], p.u[i]));
    const double ry = __dadd_rn(xy, __dsub_rn(p.u[np + j], p.u[np + i]));
    const double rz = __dadd_rn(xz, __dsub_rn(p.u[2 * np + j], p.u[2 * np + i]));
    const double r = __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz)));
    const double xi = __dsqrt_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(xx, xx), __dmul_rn(xy, xy)), __dmul_rn(xz, xz)));
    if (FRACTURE && __dmul_rn(r, r) >= __dmul_rn(__dmul_rn(bbc, xi), xi) && !nofail_i &&
        !p.nofail[j])
        return true;
    const double s = __ddiv_rn(__dsub_rn(r, xi), xi);
    const double coeff = __dmul_rn(__dmul_rn(c, s), p.vol[j]);
    if (w) *w += 0.25 * c * s * s * xi * p.vol[j];
    f[0] += __ddiv_rn(__dmul_rn(coeff, rx), r);
    f[1] += __ddiv_rn(__dmul_rn(coeff, ry), r);
    f[2] += __ddiv_rn(__dmul_rn(coeff, rz), r);
    return false;
}

// One bond of the unrolled table walk: entry e of row i, gather record uj.
// Adds F r_vec to f when the bond is present and intact (bit on) and num is
// inside the entry's window; a present bond outside it is deferred (pend).
// ENERGY: the bond's strain energy kw s^2 into w as well, s = q S(q).
template <bool UNIFORM, int NP, bool ENERGY = false>
__device__ __forceinline__ void stencil_bond64(const StencilEntry64& e, const double* h,
                                               const double4& uj, const double4& ui, bool on,
                                               uint32_t bit, uint32_t& pend, double& fx,
                                               double& fy, double& fz, const double* sh = nullptr,
                                               double kw = 0.0, double* w = nullptr)
{
    const double hx = uj.x - ui.x, hy = uj.y - ui.y, hz = uj.z - ui.z;
    const double num = fma(hz, hz + e.tz, fma(hy, hy + e.ty, hx * (hx + e.tx)));
    const double q = num * e.ixi2;
    double t = h[NP - 1];
#pragma unroll
    for (int k = NP - 2; k >= 0; --k) t = fma(t, q, h[k]);
    double F = (num * e.K) * t;
    if (!UNIFORM) F *= uj.w;
    const bool in = ((uint32_t)__double2hiint(num) & 0x7fffffffu) < e.khi;
    if (on && !in) pend |= bit;
    F = (on && in) ? F : 0.0;
    fx = fma(F, e.ex + hx, fx);
    fy = fma(F, e.ey + hy, fy);
    fz = fma(F, e.ez + hz, fz);
    if (ENERGY) {
        double sv = sh[NP - 1];
#pragma unroll
        for (int k = NP - 2; k >= 0; --k) sv = fma(sv, q, sh[k]);
        sv *= q;
        *w += (on && in) ? kw * sv * sv : 0.0;
    }
}

// Row i's present and intact table entries as entry-order bits (bit k of
// ew[w] = entry 32 w + k). Kind-2 rows hold the whole table, so bond slot k
// is entry k; other stencil rows hold the entries of their presence mask in
// table order, so their s-th present entry is bond slot s.
template <bool FRACTURE, int NW = 4>
__device__ __forceinline__ void row_entry_bits(const EllView& nl, const StencilRows& sr,
                                               int ntab, int nwords, int kind, int64_t i,
                                               int64_t np, uint32_t (&ew)[NW])
{
    uint32_t pm[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        uint32_t full = 0u;
        if (w < nwords) {
            const int rem = ntab - 32 * w;
            full = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
        }
        pm[w] = w < nwords ? (kind == 2 ? full : sr.pmask[(int64_t)w * np + i]) : 0u;
    }
    if (!FRACTURE) {
#pragma unroll
        for (int w = 0; w < NW; ++w) ew[w] = pm[w];
        return;
    }
    // The list holds ceil(max_n / 32) bond-state words per row, which can be
    // fewer than the table's words (a thin body holds only part of the
    // table): words past the list's are absent, not read.
    const int lwords = (nl.max_n + 31) >> 5;
    uint32_t mw[NW];
    int cnt = 0, intact = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        mw[w] = (w < nwords && w < lwords) ? nl.mu[(int64_t)w * np + i] : 0u;
        cnt += __popc(pm[w]);
        intact += __popc(mw[w]);
    }
    if (kind == 2) {
#pragma unroll
        for (int w = 0; w < NW; ++w) ew[w] = mw[w] & pm[w];
    } else if (intact == cnt) {
#pragma unroll
        for (int w = 0; w < NW; ++w) ew[w] = pm[w];
    } else {
        // Slot order -> entry order: the s-th present entry takes the s-th
        // bit of the slot-order words.
        int sw = 0, sb = 0;
        uint32_t src = mw[0];
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            uint32_t out = 0u, q = pm[w];
            while (q) {
                const int b = __ffs(q) - 1;
                q &= q - 1;
                out |= (src & 1u) << b;
                src >>= 1;
                if (++sb == 32) {
                    sb = 0;
                    ++sw;
                    src = 0u;
#pragma unroll
                    for (int v = 1; v < NW; ++v)
                        if (sw == v) src = mw[v];
                }
            }
            ew[w] = out;
        }
    }
}

// Bond slot of row i's table entry 32 w + b: the row's present entries
// before it (kind 2: the entry itself).
__device__ __forceinline__ int entry_slot(const StencilRows& sr, int kind, int64_t i,
                                          int64_t np, int w, int b)
{
    int s = 32 * w + b;
    if (kind != 2) {
        s = 0;
        for (int v = 0; v < w; ++v) s += __popc(sr.pmask[(int64_t)v * np + i]);
        s += __popc(sr.pmask[(int64_t)w * np + i] & ((1u << b) - 1u));
    }
    return s;
}

// Marks broken the bond of row i at table entry 32 w + b.
__device__ __forceinline__ void clear_bond_bit(const EllView& nl, const StencilRows& sr,
                                               int kind, int64_t i, int64_t np, int w, int b)
{
    const int s = entry_slot(sr, kind, i, np, w, b);
    nl.mu[(int64_t)(s >> 5) * np + i] &= ~(1u << (s & 31));
}

// One warp per chunk of 32 rows of the stencil warp list; each row walks
// table entries [K0, K1) (unrolled), and its own entries that are present
// and intact are the bits of ew. NP: coefficients of the stretch
// polynomial. The walk may be cut into parts launched one after the other
// (the whole table's code exceeds the instruction cache): a part that does
// not start at entry 0 continues from the partial force record FPART of the
// previous part, and a part that is not the last stores its sum there;
// the last part applies the step epilogue.
// ENERGY (output steps; one particle volume): the parts also sum the rows'
// strain energy density W_i (the first part's in FPART's w), and the last
// part writes W_i and phi_i = 1 - vol_sums[intact] / vol_sums[bonds] after
// the step's bond breaking, and per warp the sums of W_i vol_i and phi_i to
// ep.energy_part, as k_pmb_stencil32 does.
// TAB: the table's size (Stencil64 or Stencil64W); its bond-bit words NW.
template <bool FRACTURE, bool UNIFORM, int K0, int K1, int NP, bool LAST, bool ENERGY = false,
          class TAB = Stencil64>
__global__ void __launch_bounds__(kBlock, 4)
    k_pmb_stencil64(ParticleView p, EllView nl, StencilRows sr,
                    const double4* __restrict__ U4, double4* __restrict__ FPART,
                    StepEpilogue ep, const TAB st, const double* __restrict__ vol_sums,
                    const int32_t* __restrict__ CELL)
{
    constexpr int NW = (int)(sizeof(st.e) / sizeof(st.e[0])) / 32;
    constexpr bool SUMS = ENERGY && LAST;
    const int lane = threadIdx.x & 31;
    const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (slot >= sr.wcount) return;
    const int64_t warp = sr.wlist[slot];
    const int64_t i = p.frozen + 32 * warp + lane;
    // With the warp sums every lane of the warp reaches them.
    if (!SUMS && i >= p.n) return;
    double Phi_i = 0.0, dmg_i = 0.0;
    if (i < p.n) {
    const int64_t np = p.npad;
    const int kind = sr.warp_kind[warp];
    uint32_t ew[NW];
    row_entry_bits<FRACTURE, NW>(nl, sr, st.ntab, st.nwords, kind, i, np, ew);
    // Row i's gather record: by lattice cell, or by row.
    const int64_t rec = CELL ? (int64_t)CELL[i] : i;
    const double4 ui = U4[rec];
    const char* __restrict__ rb = reinterpret_cast<const char*>(U4 + rec);
    double fx = 0.0, fy = 0.0, fz = 0.0, wsum = 0.0;
    if (K0 > 0) {
        const double4 fp = FPART[i];
        fx = fp.x;
        fy = fp.y;
        fz = fp.z;
        if (ENERGY) wsum = fp.w;
    }
    uint32_t pend[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) pend[w] = 0u;
    // Fully unrolled, every entry of the range for every row: an absent entry
    // (no bit in ew) reads the record at i + delta_k (a neighbour, or a zero
    // guard record) and adds nothing, which costs less than a branch per
    // entry. Entries past ntab are zero-filled and add nothing either. (A
    // loop over chunks of 8 entries with the table in shared memory keeps
    // the code inside the instruction cache but waits on the shared-memory
    // loads: 4.75 vs 3.25 ms per step on the full plate; two rows per thread
    // halves the instruction fetch per bond but needs 128 registers, and
    // at 2 blocks per SM: 3.76 ms.)
#pragma unroll
    for (int k = K0; k < K1; ++k) {
        const int w = k >> 5;
        const uint32_t bit = 1u << (k & 31);
        const StencilEntry64& e = st.e[k];
        const double4 uj = *reinterpret_cast<const double4*>(rb + e.boff);
        stencil_bond64<UNIFORM, NP, ENERGY>(e, st.h, uj, ui, (ew[w] & bit) != 0u, bit, pend[w],
                                            fx, fy, fz, st.sh, ENERGY ? st.kw[k] : 0.0, &wsum);
    }
    int broken = 0;
    uint32_t anyp = 0u;
#pragma unroll
    for (int w = 0; w < NW; ++w) anyp |= pend[w];
    if (anyp) {
        // Deferred bonds: the reference's exact test and force.
        double f[3] = {fx, fy, fz};
        const bool nofail_i = FRACTURE ? (p.nofail[i] != 0) : false;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            uint32_t q = pend[w];
            while (q) {
                const int b = __ffs(q) - 1;
                q &= q - 1;
                const int k = 32 * w + b;
                // The neighbour: from the list when records are by lattice
                // cell (the table's deltas are then cell deltas).
                const int64_t j =
                    CELL ? (int64_t)nl.idx[(int64_t)entry_slot(sr, kind, i, np, w, b) * np + i]
                         : i + st.e[k].doff;
                if (exact_bond<FRACTURE>(p, i, j, st.c, st.bbc, nofail_i, f,
                                         ENERGY ? &wsum : nullptr)) {
                    clear_bond_bit(nl, sr, kind, i, np, w, b);
                    ++broken;
                }
            }
        }
        fx = f[0];
        fy = f[1];
        fz = f[2];
    }
    if (LAST) {
        step_epilogue<false>(p, ep, i, fx, fy, fz);
        if (ENERGY) {
            // ew covers every entry (the first part's breaking included).
            p.W[i] = wsum;
            Phi_i = wsum * p.vol[i];
            if (FRACTURE) {
                int intact = -broken;
#pragma unroll
                for (int w = 0; w < NW; ++w) intact += __popc(ew[w]);
                dmg_i = 1 - vol_sums[intact] / vol_sums[nl.count[i]];
                p.phi[i] = dmg_i;
            }
        }
    } else {
        FPART[i] = make_double4(fx, fy, fz, ENERGY ? wsum : 0.0);
    }
    }
    if (SUMS) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            Phi_i += __shfl_xor_sync(0xffffffffu, Phi_i, o);
            dmg_i += __shfl_xor_sync(0xffffffffu, dmg_i, o);
        }
        if (lane == 0) {
            ep.energy_part[2 * slot] = Phi_i;
            ep.energy_part[2 * slot + 1] = dmg_i;
        }
    }
}

// Mixed precision (CPD_MIXED, PMB): the same table walk in FP32 on the FP32
// split of u (MixedU: hi.xyz + lo.xyz, hi.w = c vol, lo.w = no-fail flag).
// eta = (hi_j - hi_i) + (lo_j - lo_i) keeps ~1e-7 relative accuracy under
// large rigid motion; num, q and the pair force as in the FP64 kernel, with
// an FP32 polynomial (kStencilPoly32 coefficients, anchored at h(0) = 1/2:
// error ~3e-8 relative at the plate's window edge, vanishing with q). Pair
// forces are summed in FP32 over chunks of 8 entries and each chunk sum is
// added to the FP64 row force. Bonds within 1e-4 s0 of the
// break (in q) or outside the polynomial's range take the FP64 exact path.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// x and y in paired FP32 operations (FADD2 / FMUL2 / FFMA2), z alone.
// ENERGY: the bond's strain energy kw s^2 into cw as well, with the stretch
// s = a / (1 - a) from a = q H(q) = 1 - xi / r.
template <bool UNIFORM, bool ENERGY = false>
__device__ __forceinline__ void stencil_bond32(const StencilEntry32& e, const float* h,
                                               const MixedU& uj, const float2& nh_xy,
                                               float nh_z, const float2& nl_xy, float nl_z,
                                               bool on, uint32_t bit, uint32_t& pend,
                                               float2& cxy, float& cz, float kw = 0.f,
                                               float* cw = nullptr)
{
    const float2 hxy = __fadd2_rn(__fadd2_rn(f2(uj.hi.x, uj.hi.y), nh_xy),
                                  __fadd2_rn(f2(uj.lo.x, uj.lo.y), nl_xy));
    const float hz = (uj.hi.z + nh_z) + (uj.lo.z + nl_z);
    const float2 pxy = __fmul2_rn(hxy, __fadd2_rn(hxy, e.txy));
    const float num = fmaf(hz, hz + e.tz, pxy.x + pxy.y);
    const float q = num * e.ixi2;
    const float t = fmaf(fmaf(fmaf(h[3], q, h[2]), q, h[1]), q, h[0]);
    float F = (num * e.K) * t;
    if (!UNIFORM) F *= uj.hi.w;
    // |num| below the window's bound T (khi holds T's bits): one compare
    // with the absolute-value operand; false for NaN, as the integer form.
    const bool in = fabsf(num) < __uint_as_float(e.khi);
    if (on && !in) pend |= bit;
    F = (on && in) ? F : 0.f;
    cxy = __ffma2_rn(f2(F, F), __fadd2_rn(e.exy, hxy), cxy);
    cz = fmaf(F, e.ez + hz, cz);
    if (ENERGY) {
        const float a = q * t;
        const float sv = __fdividef(a, 1.f - a);
        *cw += (on && in) ? kw * sv * sv : 0.f;
    }
}

// ENERGY (output steps; one particle volume): the rows' strain energy
// density W_i (the bond terms kw s^2 in the force's FP32 chunks of 8 into
// FP64, the deferred bonds' in FP64) and damage phi_i = 1 - vol_sums[intact]
// / vol_sums[bonds] (the ordered FP64 sums of the damage formula,
// force/CabanaPD_PMB.hpp:289-339), after this step's bond breaking; the
// warp's sums of W_i vol_i and phi_i go to ep.energy_part.
template <bool FRACTURE, bool UNIFORM, int NT, bool ENERGY = false>
__global__ void __launch_bounds__(kBlock, 3)
    k_pmb_stencil32(ParticleView p, EllView nl, StencilRows sr, const MixedU* __restrict__ U2,
                    StepEpilogue ep, const Stencil32 st, const double* __restrict__ vol_sums)
{
    const int lane = threadIdx.x & 31;
    const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (slot >= sr.wcount) return;
    const int64_t warp = sr.wlist[slot];
    const int64_t i = p.frozen + 32 * warp + lane;
    // Without ENERGY a lane past the last row leaves; with it every lane of
    // the warp reaches the warp's sums.
    if (!ENERGY && i >= p.n) return;
    double Phi_i = 0.0, dmg_i = 0.0;
    if (i < p.n) {
    const int64_t np = p.npad;
    const int kind = sr.warp_kind[warp];
    uint32_t ew[4];
    row_entry_bits<FRACTURE>(nl, sr, st.ntab, st.nwords, kind, i, np, ew);
    const MixedU ui = U2[i];
    const float2 nh_xy = f2(-ui.hi.x, -ui.hi.y), nl_xy = f2(-ui.lo.x, -ui.lo.y);
    const float nh_z = -ui.hi.z, nl_z = -ui.lo.z;
    const char* __restrict__ rb = reinterpret_cast<const char*>(U2 + i);
    double f[3] = {0.0, 0.0, 0.0};
    float2 cxy = f2(0.f, 0.f);
    float cz = 0.f;
    double wsum = 0.0;
    float cw = 0.f;
    uint32_t pend[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const int w = k >> 5;
        const uint32_t bit = 1u << (k & 31);
        const StencilEntry32& e = st.e[k];
        const MixedU uj = *reinterpret_cast<const MixedU*>(rb + e.boff);
        stencil_bond32<UNIFORM, ENERGY>(e, st.h, uj, nh_xy, nh_z, nl_xy, nl_z,
                                        (ew[w] & bit) != 0u, bit, pend[w], cxy, cz,
                                        ENERGY ? st.kw[k] : 0.f, &cw);
        if ((k & 7) == 7 || k == NT - 1) {
            f[0] += (double)cxy.x;
            f[1] += (double)cxy.y;
            f[2] += (double)cz;
            cxy = f2(0.f, 0.f);
            cz = 0.f;
            if (ENERGY) {
                wsum += (double)cw;
                cw = 0.f;
            }
        }
    }
    int broken = 0;
    if (pend[0] | pend[1] | pend[2] | pend[3]) {
        const bool nofail_i = FRACTURE ? (p.nofail[i] != 0) : false;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            uint32_t q = pend[w];
            while (q) {
                const int b = __ffs(q) - 1;
                q &= q - 1;
                const int k = 32 * w + b;
                if (exact_bond<FRACTURE>(p, i, i + st.e[k].doff, st.c, st.bbc, nofail_i, f,
                                         ENERGY ? &wsum : nullptr)) {
                    clear_bond_bit(nl, sr, kind, i, np, w, b);
                    ++broken;
                }
            }
        }
    }
    step_epilogue<true>(p, ep, i, f[0], f[1], f[2]);
    if (ENERGY) {
        p.W[i] = wsum;
        Phi_i = wsum * p.vol[i];
        if (FRACTURE) {
            const int intact =
                __popc(ew[0]) + __popc(ew[1]) + __popc(ew[2]) + __popc(ew[3]) - broken;
            dmg_i = 1 - vol_sums[intact] / vol_sums[nl.count[i]];
            p.phi[i] = dmg_i;
        }
    }
    }
    if (ENERGY) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            Phi_i += __shfl_xor_sync(0xffffffffu, Phi_i, o);
            dmg_i += __shfl_xor_sync(0xffffffffu, dmg_i, o);
        }
        if (lane == 0) {
            ep.energy_part[2 * slot] = Phi_i;
            ep.energy_part[2 * slot + 1] = dmg_i;
        }
    }
}

}  // namespace

void free_stencil64(MixedState& m, cudaStream_t st)
{
    delete m.st64;
    m.st64 = nullptr;
    delete m.st64w;
    m.st64w = nullptr;
    if (m.u4_base) dev_free(m.u4_base, st);
    if (m.u4_alt_base) dev_free(m.u4_alt_base, st);
    if (m.f64part) dev_free(m.f64part, st);
    m.f64part = nullptr;
    m.u4 = m.u4_base = m.u4_alt = m.u4_alt_base = nullptr;
    m.guard = 0;
}

bool stencil64_ready(const MixedState& m)
{
    return (m.st64 != nullptr || m.st64w != nullptr) && m.u4 && m.u4_alt;
}


namespace {

// Fills the FP64 table S from the lattice offsets; returns the largest
// |delta| of its entries.
template <int N>
int64_t fill_stencil64(const Model& md, const double* h, const MixedStencil* tab, int ntab,
                       const MixedState& m, Stencil64T<N>* S)
{
    S->ntab = ntab;
    S->nwords = (ntab + 31) / 32;
    S->bbc = md.bond_break_coeff;
    S->c = md.c;
    const bool uniform = m.vol_sums != nullptr;
    const long double scale = (long double)md.c * (uniform ? (long double)m.vol_uniform : 1.0L);
    // Window |q| < qwin per entry: inside the polynomial's range, and
    // (fracture) below the break by a margin far above the rounding of num
    // and of the lattice offsets (q units).
    const double qc = md.bond_break_coeff - 1.0;
    const double qwin = md.fracture ? std::min(kStencilQ, qc - 1e-9) : kStencilQ;
    // The polynomial interpolates on |q| <= qwin: 8 coefficients reach
    // ~2.5e-16 relative up to 0.0231 (the notched plate's window is 0.0228),
    // 9 up to kStencilQ.
    const long double qfit = qwin > 1e-6 ? (long double)qwin : 1e-6L;
    S->np = qfit <= 0.0231L ? 8 : 9;
    long double hc[kStencilPoly] = {}, sc[kStencilPoly] = {};
    fit_stretch_poly(qfit, S->np, hc);
    fit_stretch_poly(qfit, S->np, sc, false, true);
    for (int k = 0; k < kStencilPoly; ++k) {
        S->h[k] = (double)hc[k];
        S->sh[k] = (double)sc[k];
    }
    int64_t G = 0;
    for (int k = 0; k < ntab; ++k) {
        StencilEntry64& e = S->e[k];
        // The table stores the FP32 offsets of the lattice vectors (a hx,
        // b hy, c hz); the integers a, b, c give back the FP64 vectors.
        const double a = std::nearbyint((double)tab[k].x / h[0]);
        const double b = std::nearbyint((double)tab[k].y / h[1]);
        const double c = std::nearbyint((double)tab[k].z / h[2]);
        e.ex = a * h[0];
        e.ey = b * h[1];
        e.ez = c * h[2];
        e.tx = 2.0 * e.ex;
        e.ty = 2.0 * e.ey;
        e.tz = 2.0 * e.ez;
        const long double x2 = (long double)e.ex * e.ex + (long double)e.ey * e.ey +
                               (long double)e.ez * e.ez;
        const long double xi = sqrtl(x2);
        e.ixi2 = (double)(1.0L / x2);
        e.K = (double)(scale / (xi * x2));
        S->kw[k] = (double)(0.25L * scale * xi);
        // An entry that no row holds (a thin body) has no index delta: its
        // bonds are absent everywhere, and it reads the row's own record.
        e.doff = tab[k].delta == INT32_MAX ? 0 : tab[k].delta;
        e.boff = (int64_t)e.doff * (int64_t)sizeof(double4);
        // |num| below T = qwin xi^2 when the high word of |num| is below
        // T's: every such num is below T (conservative by < 2^-20 of T).
        e.khi = qwin > 0.0 ? hi_word(qwin * (double)x2) : 0u;
        G = std::max<int64_t>(G, std::abs((int64_t)e.doff));
    }
    return G;
}

}  // namespace

bool prepare_stencil64(const ParticleView& p, const Model& md, const double* h,
                       const MixedStencil* tab, int ntab, MixedState& m, cudaStream_t st,
                       std::string& err)
{
    free_stencil64(m, st);
    if (md.pd != CPD_PD_PMB || ntab <= 0 || ntab > kStencilMaxWide) return false;
    int64_t G = 0;
    if (ntab <= kStencilMax) {
        m.st64 = new Stencil64();
        G = fill_stencil64(md, h, tab, ntab, m, m.st64);
    } else {
        // The wide walk (three or four launches of 64 entries) takes one
        // particle volume only. On tables of 129-192 entries it is still
        // faster than the general FP64 kernel (200 x 100 x 12 cells of the
        // 0.2 x 0.1 x 0.009 m plate, 140 entries: 0.167 vs 0.214 ms per step;
        // 400 x 200 x 20, 130 entries: 0.776 vs 1.134 ms).
        if (m.vol_sums == nullptr) return false;
        m.st64w = new Stencil64W();
        G = fill_stencil64(md, h, tab, ntab, m, m.st64w);
    }
    m.guard = G + 32;
    // Records by lattice cell (m.gcell) or by row.
    const size_t recs = (size_t)((m.gcell ? m.grid_cells : p.npad) + 2 * m.guard);
    if (dev_alloc(&m.u4_base, sizeof(double4) * recs, st) != cudaSuccess ||
        dev_alloc(&m.u4_alt_base, sizeof(double4) * recs, st) != cudaSuccess ||
        dev_alloc(&m.f64part, sizeof(double4) * (size_t)p.npad, st) != cudaSuccess ||
        cudaMemsetAsync(m.u4_base, 0, sizeof(double4) * recs, st) != cudaSuccess ||
        cudaMemsetAsync(m.u4_alt_base, 0, sizeof(double4) * recs, st) != cudaSuccess) {
        err = std::string("stencil gather records: ") + cudaGetErrorString(cudaGetLastError());
        free_stencil64(m, st);
        return false;
    }
    m.u4 = m.u4_base + m.guard;
    m.u4_alt = m.u4_alt_base + m.guard;
    m.bytes += 2 * sizeof(double4) * recs + sizeof(double4) * (size_t)p.npad;
    return true;
}

bool prepare_stencil32(const Model& md, const double* h, const MixedStencil* tab, int ntab,
                       MixedState& m)
{
    delete m.st32;
    m.st32 = nullptr;
    if (md.pd != CPD_PD_PMB || ntab <= 0 || ntab > kStencilMax) return false;
    Stencil32* S = new Stencil32();
    S->ntab = ntab;
    S->nwords = (ntab + 31) / 32;
    S->bbc = md.bond_break_coeff;
    S->c = md.c;
    const bool uniform = m.vol_sums != nullptr;
    const long double scale = (long double)md.c * (uniform ? (long double)m.vol_uniform : 1.0L);
    // Window |q| < qwin: the break band of the FP32 kernels (stretch within
    // 1e-4 s0 of s0) and the polynomial's range.
    const double s_lo = md.s0 * (1.0 - 1e-4);
    const double qc_lo = (1.0 + s_lo) * (1.0 + s_lo) - 1.0;
    const double qwin = md.fracture ? std::min(kStencilQ, qc_lo) : kStencilQ;
    long double hc[kStencilPoly] = {};
    fit_stretch_poly(qwin > 1e-6 ? (long double)qwin : 1e-6L, kStencilPoly32, hc, true);
    for (int k = 0; k < kStencilPoly32; ++k) S->h[k] = (float)hc[k];
    int64_t G = 0;
    for (int k = 0; k < ntab; ++k) {
        StencilEntry32& e = S->e[k];
        const double a = std::nearbyint((double)tab[k].x / h[0]);
        const double b = std::nearbyint((double)tab[k].y / h[1]);
        const double c = std::nearbyint((double)tab[k].z / h[2]);
        const double vx = a * h[0], vy = b * h[1], vz = c * h[2];
        e.exy = make_float2((float)vx, (float)vy);
        e.ez = (float)vz;
        e.txy = make_float2(2.f * e.exy.x, 2.f * e.exy.y);
        e.tz = 2.f * e.ez;
        // Lengths of the FP32 vectors the kernel works with, so that the
        // force law is consistent with the geometry it sees: constants from
        // the FP64 lengths would give each bond length class a stiffness
        // error of ~1e-7 that accumulates over a run (measured: 1.2e-6 vs
        // 5e-7 in u after 100 steps of the 41^3 elastic wave).
        const long double fx = e.exy.x, fy = e.exy.y, fz = e.ez;
        const long double x2 = fx * fx + fy * fy + fz * fz;
        e.ixi2 = (float)(1.0L / x2);
        e.K = (float)(scale / (sqrtl(x2) * x2));
        S->kw[k] = (float)(0.25L * scale * sqrtl(x2));
        e.doff = tab[k].delta == INT32_MAX ? 0 : tab[k].delta;  // (as in the FP64 table)
        e.boff = (int64_t)e.doff * (int64_t)sizeof(MixedU);
        const float T = (float)(qwin * (double)x2);
        uint32_t tb;
        std::memcpy(&tb, &T, sizeof tb);
        e.khi = qwin > 0.0 ? tb : 0u;
        G = std::max<int64_t>(G, std::abs((int64_t)e.doff));
    }
    m.st32 = S;
    m.guard = G + 32;
    return true;
}

int launch_pd_force_stencil32(const ParticleView& p, const EllView& nl, const Model& md,
                              const MixedState& m, const StepEpilogue& ep, cudaStream_t st)
{
    if (p.n - p.frozen <= 0 || m.nstencil <= 0) return 0;
    const StencilRows sr{m.warp_kind, m.pmask, m.stencil_list, m.nstencil};
    const int g = (int)((m.nstencil + kBlock / 32 - 1) / (kBlock / 32));
    const bool uniform = m.vol_sums != nullptr;
    const Stencil32& S = *m.st32;
    const bool t122 = S.ntab == 122;
    if (ep.energy_part) {
        // Output step: the energy forms (one particle volume only).
        if (!uniform) return -1;
#define CPD_ST32E(F, NT) \
    k_pmb_stencil32<F, true, NT, true><<<g, kBlock, 0, st>>>(p, nl, sr, m.u2, ep, S, m.vol_sums)
        if (md.fracture) {
            if (t122) CPD_ST32E(true, 122); else CPD_ST32E(true, 128);
        } else {
            if (t122) CPD_ST32E(false, 122); else CPD_ST32E(false, 128);
        }
#undef CPD_ST32E
        return 1;
    }
#define CPD_ST32(F, U, NT) \
    k_pmb_stencil32<F, U, NT><<<g, kBlock, 0, st>>>(p, nl, sr, m.u2, ep, S, nullptr)
    if (!uniform) {
        if (md.fracture) CPD_ST32(true, false, 128); else CPD_ST32(false, false, 128);
    } else if (md.fracture) {
        if (t122) CPD_ST32(true, true, 122); else CPD_ST32(true, true, 128);
    } else {
        if (t122) CPD_ST32(false, true, 122); else CPD_ST32(false, true, 128);
    }
#undef CPD_ST32
    return 1;
}

int launch_pack_u4(const ParticleView& p, const double* u, int64_t begin, int64_t end,
                   double4* u4, cudaStream_t st, const int32_t* cell)
{
    if (end <= begin) return 0;
    k_pack_u4<<<blocks_for(end - begin), kBlock, 0, st>>>(u, p.vol, p.npad, begin, end, u4,
                                                          cell);
    return 1;
}

int launch_pd_force_stencil64(const ParticleView& p, const EllView& nl, const Model& md,
                              const MixedState& m, const StepEpilogue& ep, cudaStream_t st)
{
    if (p.n - p.frozen <= 0) return 0;
    int launched = 0;
    if (m.nstencil > 0) {
        const StencilRows sr{m.warp_kind, m.pmask, m.stencil_list, m.nstencil};
        const int g = (int)((m.nstencil + kBlock / 32 - 1) / (kBlock / 32));
        const bool uniform = m.vol_sums != nullptr;
        if (m.st64w) {
            // Tables past 128 entries (a horizon of 4 spacings: 256): four
            // launches of 64 entries, the partial force passed on between
            // them; one particle volume.
            const Stencil64W& W = *m.st64w;
            // Tables of up to 192 entries (unequal spacings at a 3-spacing
            // horizon) stop after the third launch.
            const bool t192 = W.ntab <= 192;
#define CPD_ST64W(F, NP, E)                                                                   \
    do {                                                                                      \
        k_pmb_stencil64<F, true, 0, 64, NP, false, E, Stencil64W>                             \
            <<<g, kBlock, 0, st>>>(p, nl, sr, m.u4, m.f64part, ep, W, m.vol_sums, m.gcell);   \
        k_pmb_stencil64<F, true, 64, 128, NP, false, E, Stencil64W>                           \
            <<<g, kBlock, 0, st>>>(p, nl, sr, m.u4, m.f64part, ep, W, m.vol_sums, m.gcell);   \
        if (t192) {                                                                           \
            k_pmb_stencil64<F, true, 128, 192, NP, true, E, Stencil64W>                       \
                <<<g, kBlock, 0, st>>>(p, nl, sr, m.u4, m.f64part, ep, W, m.vol_sums,         \
                                       m.gcell);                                              \
        } else {                                                                              \
            k_pmb_stencil64<F, true, 128, 192, NP, false, E, Stencil64W>                      \
                <<<g, kBlock, 0, st>>>(p, nl, sr, m.u4, m.f64part, ep, W, m.vol_sums,         \
                                       m.gcell);                                              \
            k_pmb_stencil64<F, true, 192, 256, NP, true, E, Stencil64W>                       \
                <<<g, kBlock, 0, st>>>(p, nl, sr, m.u4, m.f64part, ep, W, m.vol_sums,         \
                                       m.gcell);                                              \
        }                                                                                     \
    } while (0)
            // An output step (ep.energy_part): the energy forms.
            const bool en = ep.energy_part != nullptr;
            if (md.fracture) {
                if (W.np == 8) {
                    if (en) CPD_ST64W(true, 8, true); else CPD_ST64W(true, 8, false);
                } else {
                    if (en) CPD_ST64W(true, 9, true); else CPD_ST64W(true, 9, false);
                }
            } else {
                if (en) CPD_ST64W(false, 9, true); else CPD_ST64W(false, 9, false);
            }
#undef CPD_ST64W
            launched += t192 ? 3 : 4;
            if (m.nirregular > 0)
                launched += launch_pd_force_fast(p, nl, md, ep, st, m.irregular_list,
                                                 m.nirregular);
            return launched;
        }
        const Stencil64& S = *m.st64;
        // Two launches over the table's halves (entries 0-63, then 64 on):
        // the first stores its partial force and broken count per row, the
        // second adds its own and runs the epilogue. Each is a shorter
        // unrolled walk that stays in the instruction cache (B200, 11.52 M
        // row plate: 3.14 ms per step for the two, 3.30 ms for one walk).
#define CPD_ST64X(F, U, NT, NP, E)                                                           \
    do {                                                                                     \
        k_pmb_stencil64<F, U, 0, 64, NP, false, E><<<g, kBlock, 0, st>>>(                    \
            p, nl, sr, m.u4, m.f64part, ep, S, m.vol_sums, m.gcell);                         \
        k_pmb_stencil64<F, U, 64, NT, NP, true, E><<<g, kBlock, 0, st>>>(                    \
            p, nl, sr, m.u4, m.f64part, ep, S, m.vol_sums, m.gcell);                         \
    } while (0)
#define CPD_ST64(F, U, NT, NP) CPD_ST64X(F, U, NT, NP, false)
        // Unrolled forms: the 122-entry table of a cubic lattice at a
        // 3.01-spacing horizon, else 128 entries (zero past ntab).
        const bool t122 = S.ntab == 122;
        if (ep.energy_part && uniform) {
            // Output step: the energy forms.
            if (md.fracture) {
                if (S.np == 8) {
                    if (t122) CPD_ST64X(true, true, 122, 8, true);
                    else CPD_ST64X(true, true, 128, 8, true);
                } else {
                    CPD_ST64X(true, true, 128, 9, true);
                }
            } else {
                if (t122) CPD_ST64X(false, true, 122, 9, true);
                else CPD_ST64X(false, true, 128, 9, true);
            }
        } else if (!uniform) {
            if (md.fracture) CPD_ST64(true, false, 128, 9); else CPD_ST64(false, false, 128, 9);
        } else if (md.fracture) {
            if (S.np == 8) {
                if (t122) CPD_ST64(true, true, 122, 8); else CPD_ST64(true, true, 128, 8);
            } else {
                CPD_ST64(true, true, 128, 9);
            }
        } else {
            if (t122) CPD_ST64(false, true, 122, 9); else CPD_ST64(false, true, 128, 9);
        }
#undef CPD_ST64
#undef CPD_ST64X
        launched += 2;
    }
    if (m.nirregular > 0)
        launched += launch_pd_force_fast(p, nl, md, ep, st, m.irregular_list, m.nirregular);
    return launched;
}

}  // namespace cpd
