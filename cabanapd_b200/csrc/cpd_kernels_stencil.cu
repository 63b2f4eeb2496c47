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

// h(q) = 1 / (sqrt(1+q) (1 + sqrt(1+q))) interpolated at n Chebyshev nodes
// of [-Q, Q]; monomial coefficients in q (long double Gaussian elimination
// on the Vandermonde system in t = q / Q, then scaled by Q^-k).
void fit_stretch_poly(long double Q, int n, long double* out)
{
    long double A[kStencilPoly][kStencilPoly + 1];
    for (int r = 0; r < n; ++r) {
        const long double t = cosl(3.141592653589793238462643383279503L * (r + 0.5L) / n);
        const long double s = sqrtl(1.0L + t * Q);
        long double pw = 1.0L;
        for (int c = 0; c < n; ++c) {
            A[r][c] = pw;
            pw *= t;
        }
        A[r][n] = 1.0L / (s * (1.0L + s));
    }
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (fabsl(A[r][c]) > fabsl(A[piv][c])) piv = r;
        for (int k = 0; k <= n; ++k) std::swap(A[c][k], A[piv][k]);
        const long double d = A[c][c];
        for (int k = 0; k <= n; ++k) A[c][k] /= d;
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const long double f = A[r][c];
            for (int k = 0; k <= n; ++k) A[r][k] -= f * A[c][k];
        }
    }
    long double qk = 1.0L;
    for (int k = 0; k < n; ++k) {
        out[k] = A[k][n] / qk;
        qk *= Q;
    }
}

__global__ void __launch_bounds__(kBlock)
    k_pack_u4(const double* __restrict__ u, const double* __restrict__ vol, int64_t np,
              int64_t begin, int64_t end, double4* __restrict__ u4)
{
    const int64_t i = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    u4[i] = make_double4(u[i], u[np + i], u[2 * np + i], vol[i]);
}

// The reference's exact break test and pair force of bond (i, j) from
// positions and displacements, every operation separately rounded
// (CabanaPD_Force.hpp:74-93 getDistance, CabanaPD_ForceModels.hpp:123-128,
// force/CabanaPD_PMB.hpp:259-279). Returns true when the bond breaks;
// otherwise adds its force to f.
template <bool FRACTURE>
__device__ __forceinline__ bool exact_bond(const ParticleView& p, int64_t i, int64_t j, double c,
                                           double bbc, bool nofail_i, double (&f)[3])
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
    f[0] += __ddiv_rn(__dmul_rn(coeff, rx), r);
    f[1] += __ddiv_rn(__dmul_rn(coeff, ry), r);
    f[2] += __ddiv_rn(__dmul_rn(coeff, rz), r);
    return false;
}

// One bond of the unrolled table walk: entry e of row i, gather record uj.
// Adds F r_vec to f when the bond is present and intact (bit on) and num is
// inside the entry's window; a present bond outside it is deferred (pend).
template <bool UNIFORM, int NP>
__device__ __forceinline__ void stencil_bond64(const StencilEntry64& e, const double* h,
                                               const double4& uj, const double4& ui, bool on,
                                               uint32_t bit, uint32_t& pend, double& fx,
                                               double& fy, double& fz)
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
}

// One warp per chunk of 32 rows of the stencil warp list; each row walks the
// whole table (NT >= ntab entries, unrolled), and its own entries that are
// present and intact are the bits of ew (entry order: bit k of word w =
// entry 32 w + k). NP: coefficients of the stretch polynomial.
template <bool FRACTURE, bool UNIFORM, int NT, int NP>
__global__ void __launch_bounds__(kBlock, 4)
    k_pmb_stencil64(ParticleView p, EllView nl, StencilRows sr,
                    const double4* __restrict__ U4, StepEpilogue ep, const Stencil64 st)
{
    const int lane = threadIdx.x & 31;
    const int64_t slot = (int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (slot >= sr.wcount) return;
    const int64_t warp = sr.wlist[slot];
    const int64_t i = p.frozen + 32 * warp + lane;
    const bool live = i < p.n;
    const int64_t np = p.npad;
    const int kind = sr.warp_kind[warp];
    uint32_t pm[4], ew[4];
#pragma unroll
    for (int w = 0; w < 4; ++w) {
        uint32_t full = 0u;
        if (w < st.nwords) {
            const int rem = st.ntab - 32 * w;
            full = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
        }
        pm[w] = (w < st.nwords && live) ? (kind == 2 ? full : sr.pmask[(int64_t)w * np + i]) : 0u;
    }
    if (!live) return;
    if (FRACTURE) {
        uint32_t mw[4];
        int cnt = 0, intact = 0;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            mw[w] = w < st.nwords ? nl.mu[(int64_t)w * np + i] : 0u;
            cnt += __popc(pm[w]);
            intact += __popc(mw[w]);
        }
        if (kind == 2) {
#pragma unroll
            for (int w = 0; w < 4; ++w) ew[w] = mw[w] & pm[w];
        } else if (intact == cnt) {
#pragma unroll
            for (int w = 0; w < 4; ++w) ew[w] = pm[w];
        } else {
            // Slot order -> entry order: the row's s-th present entry holds
            // slot s; its bit is the s-th bit of the slot-order words.
            int sw = 0, sb = 0;
            uint32_t src = mw[0];
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                uint32_t out = 0u, q = pm[w];
                while (q) {
                    const int b = __ffs(q) - 1;
                    q &= q - 1;
                    out |= (src & 1u) << b;
                    src >>= 1;
                    if (++sb == 32) {
                        sb = 0;
                        ++sw;
                        src = sw == 1 ? mw[1] : (sw == 2 ? mw[2] : mw[3]);
                    }
                }
                ew[w] = out;
            }
        }
    } else {
#pragma unroll
        for (int w = 0; w < 4; ++w) ew[w] = pm[w];
    }
    const double4 ui = U4[i];
    const char* __restrict__ rb = reinterpret_cast<const char*>(U4 + i);
    double fx = 0.0, fy = 0.0, fz = 0.0;
    uint32_t pend[4] = {0u, 0u, 0u, 0u};
    // Fully unrolled, every entry of the table for every row: an absent entry
    // (no bit in ew) reads the record at i + delta_k (a neighbour, or a zero
    // guard record) and adds nothing, which costs less than a branch per
    // entry. Entries past ntab are zero-filled and add nothing either.
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const int w = k >> 5;
        const uint32_t bit = 1u << (k & 31);
        const StencilEntry64& e = st.e[k];
        const double4 uj = *reinterpret_cast<const double4*>(rb + e.boff);
        stencil_bond64<UNIFORM, NP>(e, st.h, uj, ui, (ew[w] & bit) != 0u, bit, pend[w], fx, fy,
                                    fz);
    }
    if (pend[0] | pend[1] | pend[2] | pend[3]) {
        // Deferred bonds: the reference's exact test and force.
        double f[3] = {fx, fy, fz};
        const bool nofail_i = FRACTURE ? (p.nofail[i] != 0) : false;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            uint32_t q = pend[w];
            while (q) {
                const int b = __ffs(q) - 1;
                q &= q - 1;
                const int k = 32 * w + b;
                if (!exact_bond<FRACTURE>(p, i, i + st.e[k].doff, st.c, st.bbc, nofail_i, f))
                    continue;
                // Broken: clear its slot's bit (slot = present entries before k).
                int s = k;
                if (kind != 2) {
                    s = 0;
                    for (int v = 0; v < w; ++v) s += __popc(sr.pmask[(int64_t)v * np + i]);
                    s += __popc(sr.pmask[(int64_t)w * np + i] & ((1u << b) - 1u));
                }
                nl.mu[(int64_t)(s >> 5) * np + i] &= ~(1u << (s & 31));
            }
        }
        fx = f[0];
        fy = f[1];
        fz = f[2];
    }
    step_epilogue<false>(p, ep, i, fx, fy, fz);
}

}  // namespace

void free_stencil64(MixedState& m, cudaStream_t st)
{
    delete m.st64;
    m.st64 = nullptr;
    if (m.u4_base) dev_free(m.u4_base, st);
    if (m.u4_alt_base) dev_free(m.u4_alt_base, st);
    m.u4 = m.u4_base = m.u4_alt = m.u4_alt_base = nullptr;
    m.guard = 0;
}

bool stencil64_ready(const MixedState& m) { return m.st64 != nullptr && m.u4 && m.u4_alt; }

bool prepare_stencil64(const ParticleView& p, const Model& md, const double* h,
                       const MixedStencil* tab, int ntab, MixedState& m, cudaStream_t st,
                       std::string& err)
{
    free_stencil64(m, st);
    if (md.pd != CPD_PD_PMB || ntab <= 0 || ntab > kStencilMax) return false;
    Stencil64* S = new Stencil64();
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
    long double hc[kStencilPoly] = {};
    fit_stretch_poly(qfit, S->np, hc);
    for (int k = 0; k < kStencilPoly; ++k) S->h[k] = (double)hc[k];
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
        e.doff = tab[k].delta;
        e.boff = (int64_t)e.doff * (int64_t)sizeof(double4);
        // |num| below T = qwin xi^2 when the high word of |num| is below
        // T's: every such num is below T (conservative by < 2^-20 of T).
        e.khi = qwin > 0.0 ? hi_word(qwin * (double)x2) : 0u;
        G = std::max<int64_t>(G, std::abs((int64_t)e.doff));
    }
    m.st64 = S;
    m.guard = G + 32;
    const size_t recs = (size_t)(p.npad + 2 * m.guard);
    if (dev_alloc(&m.u4_base, sizeof(double4) * recs, st) != cudaSuccess ||
        dev_alloc(&m.u4_alt_base, sizeof(double4) * recs, st) != cudaSuccess ||
        cudaMemsetAsync(m.u4_base, 0, sizeof(double4) * recs, st) != cudaSuccess ||
        cudaMemsetAsync(m.u4_alt_base, 0, sizeof(double4) * recs, st) != cudaSuccess) {
        err = std::string("stencil gather records: ") + cudaGetErrorString(cudaGetLastError());
        free_stencil64(m, st);
        return false;
    }
    m.u4 = m.u4_base + m.guard;
    m.u4_alt = m.u4_alt_base + m.guard;
    m.bytes += 2 * sizeof(double4) * recs;
    return true;
}

int launch_pack_u4(const ParticleView& p, const double* u, int64_t begin, int64_t end,
                   double4* u4, cudaStream_t st)
{
    if (end <= begin) return 0;
    k_pack_u4<<<blocks_for(end - begin), kBlock, 0, st>>>(u, p.vol, p.npad, begin, end, u4);
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
        const Stencil64& S = *m.st64;
#define CPD_ST64(F, U, NT, NP) \
    k_pmb_stencil64<F, U, NT, NP><<<g, kBlock, 0, st>>>(p, nl, sr, m.u4, ep, S)
        // Unrolled forms: the 122-entry table of a cubic lattice at a
        // 3.01-spacing horizon, else 128 entries (zero past ntab).
        const bool t122 = S.ntab == 122;
        if (!uniform) {
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
        ++launched;
    }
    if (m.nirregular > 0)
        launched += launch_pd_force_fast(p, nl, md, ep, st, m.irregular_list, m.nirregular);
    return launched;
}

}  // namespace cpd
