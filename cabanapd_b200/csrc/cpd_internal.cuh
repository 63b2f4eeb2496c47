// Internal data structures of the cabanapd_b200 library.
//
// HBM layout (one cpd_system):
//   particle fields   structure-of-arrays, component-major: a vector field is
//                     three contiguous double arrays of `npad` entries
//                     (x0[0..npad), x1[...], x2[...]); scalars are [npad].
//   PD neighbour list padded ELL, column-major: idx[k * npad + i] is the k-th
//                     neighbour of particle i (internal index), k < count[i].
//                     Row order is ascending caller index of the neighbour.
//   broken bonds      one bit per bond: mu[w * npad + i] bit b covers bond
//                     k = 32 w + b of particle i (1 = intact).
// Column-major ELL makes the k-th loads of a warp's 32 consecutive particles
// contiguous, and for particles on a lattice stored x-fastest the k-th
// neighbours of consecutive particles are consecutive too, so neighbour
// gathers coalesce.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>

#include <string>
#include <vector>

#include "../../include/cabanapd_b200.h"

namespace cpd {

constexpr double kPi = 3.14159265358979323846;

// Device memory of the library comes from one stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the owning system's stream),
// so setting up or releasing a system never synchronises the device: a job
// admitted or retired while others run does not stall them. Freed blocks
// stay in the pool for the next system and are returned to the driver when
// the last live system on the device is destroyed.
// Message returned by cpd_last_error() on the calling thread.
void set_last_error(const std::string& msg);

cudaError_t dev_alloc(void** ptr, size_t bytes, cudaStream_t st);
cudaError_t dev_free(void* ptr, cudaStream_t st);
template <class T>
inline cudaError_t dev_alloc(T** ptr, size_t bytes, cudaStream_t st)
{
    return dev_alloc(reinterpret_cast<void**>(ptr), bytes, st);
}

// Model constants, derived on the host with the reference constructors'
// expressions (force_models/CabanaPD_PMB.hpp:41-47, CabanaPD_LPS.hpp:64-75,
// CabanaPD_ForceModels.hpp:93-102, CabanaPD_Hertzian.hpp:40-56).
struct Model {
    int pd = CPD_PD_NONE;
    int fracture = 0;
    int influence = 1;
    int contact = CPD_CONTACT_NONE;
    int per_particle_radius = 0;
    double horizon = 0, K = 0, G = 0, G0 = 0;
    double c = 0;
    double theta_coeff = 0, s_coeff = 0;
    double s0 = 0, bond_break_coeff = 0;
    double radius = 0, radius_extend = 0, nu = 0, E = 0, e = 0;
    double Rs = 0, Es = 0, beta = 0, coeff_h_n = 0, coeff_h_d = 0;
    // Normal repulsion: its own delta and stiffness constant c.
    double contact_horizon = 0, c_contact = 0;
};

// Device view of one neighbour list.
struct EllView {
    const int32_t* count;
    const int32_t* idx;
    uint32_t* mu;  // nullptr for lists without bond state
    int32_t max_n;
    // Rows per block of a bond kernel (tile_chunk): warps take chunks of 32
    // rows; with stride > 1 the warps of a block take chunks stride apart.
    int32_t stride = 1;
    int64_t pitch = 0;  // index delta to the next lattice line (0: unknown)
};

// Row chunk of the calling warp. stride 1: consecutive chunks per block.
// stride S > 1: block b holds chunks (W g + w) S + c for its warps w < W,
// with g = b / S and c = b % S, so that on an x-fastest lattice (S = pitch /
// 32) the block's warps hold neighbouring lattice lines and the neighbour
// lines one warp brings into L1 serve the next. Both map launched warps one
// to one onto row chunks (tile_view sizes the grid).
__device__ __forceinline__ int64_t tile_chunk(const EllView& nl)
{
    if (nl.stride > 1) {
        const int64_t g = blockIdx.x / nl.stride, c = blockIdx.x % nl.stride;
        return ((int64_t)(blockDim.x >> 5) * g + (threadIdx.x >> 5)) * nl.stride + c;
    }
    return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ int64_t tile_row(const EllView& nl, int64_t first)
{
    return first + 32 * tile_chunk(nl) + (threadIdx.x & 31);
}

// Host-side trace of set-up phases (CPD_TRACE=1): each mark waits for the
// stream and prints the wall time since the previous mark to stderr.
// Without the variable a mark does nothing.
inline bool trace_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("CPD_TRACE");
        return e && std::atoi(e) != 0;
    }();
    return on;
}
struct PhaseTrace {
    const char* scope;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    explicit PhaseTrace(const char* s) : scope(s) {}
    void mark(const char* phase, cudaStream_t st)
    {
        if (!trace_enabled()) return;
        cudaStreamSynchronize(st);
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[cpd trace] %s/%s %.3f ms\n", scope, phase,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

// Tiled view of a list for `rows` rows and its grid (blocks of `block`
// threads): with a lattice line pitch of 64 rows or more, a block's warps
// take chunks one lattice line apart.
inline EllView tile_view(EllView v, int64_t rows, int block, int* grid)
{
    const int64_t chunks = (rows + 31) / 32, wpb = block / 32;
    v.stride = 1;
    if (v.pitch >= 64) {
        v.stride = (int32_t)((v.pitch + 16) / 32);
        const int64_t per = wpb * v.stride;
        *grid = (int)(((chunks + per - 1) / per) * v.stride);
    } else {
        *grid = (int)((chunks + wpb - 1) / wpb);
    }
    return v;
}

// Model constants of the throughput kernels, as the kernels take them:
// the FP64 form (cpd_kernels_fast.cu) and the FP32 forms of the mixed PMB
// and LPS kernels (cpd_kernels_mixed.cu), with the guard band of the FP64
// re-test around s0.
struct FastModel {
    double c, theta_coeff, s_coeff, bond_break_coeff;
};
struct MixedModel {
    float c, s0, guard;
    float s_lo, s_hi;  // s0 - guard, s0 + guard
    double bbc;
    int ntab;
};
struct MixedLps {
    float s0, guard;
    float s_lo, s_hi;  // s0 - guard, s0 + guard
    double bbc;
    double theta_coeff, s_coeff;
    int ntab;
    float vol;  // the particle volume when the packed records are used
};

// Everything a particle kernel needs, passed by value.
struct ParticleView {
    int64_t n, frozen, npad;
    const double* x;  // [3][npad]
    double* u;        // [3][npad]
    double* v;
    double* f;
    const double* vol;
    const double* rho;
    const uint8_t* nofail;
    double* m;
    double* theta;
    double* lps_a;  // theta_coeff * theta / m per particle
    double* lps_b;  // s_coeff / m per particle
    double* W;
    double* phi;
    const double* radius;
    double* u_neigh;
};

struct NeighborList {
    int32_t max_n = 0;
    int32_t cap = 0;      // allocated row capacity (>= max_n)
    size_t bytes = 0;     // device bytes held
    int64_t total = 0;
    int32_t nwords = 0;
    int32_t* count = nullptr;
    int32_t* idx = nullptr;
    uint32_t* mu = nullptr;
    int64_t pitch = 0;  // index delta to the next lattice line of a middle row (0: none)
    // Per axis the smallest nonzero pair separation, from the count pass
    // when requested (hmin_valid).
    double hmin[3] = {0, 0, 0};
    bool hmin_valid = false;
    EllView view() const { return EllView{count, idx, mu, max_n, 1, pitch}; }
};

struct BoundaryCondition {
    int kind = 0;
    int component = 0;
    int64_t count = 0;
    int32_t* idx = nullptr;      // internal indices
    double* values = nullptr;    // device, [count] for FORCE_ADD
    double value = 0;            // scalar kinds
};

struct StepEpilogue;

// ---------------------------------------------------------------------------
// Kernel launchers (definitions in cpd_kernels_exact.cu / cpd_neighbor.cu).
// Each returns the number of kernels it launched.
// u_out: where the new displacement goes (p.u for in place).
int launch_vv_initial(const ParticleView& p, double dt, bool track_max,
                      double* block_max, int max_blocks, double* u_out, cudaStream_t st);
int launch_vv_final(const ParticleView& p, double dt, cudaStream_t st);
int launch_lps_weighted_volume(const ParticleView& p, const EllView& nl,
                               const Model& md, cudaStream_t st);
int launch_lps_dilatation(const ParticleView& p, const EllView& nl,
                          const Model& md, cudaStream_t st);
int launch_pd_force(const ParticleView& p, const EllView& nl, const Model& md,
                    cudaStream_t st);
int launch_pd_energy(const ParticleView& p, const EllView& nl, const Model& md,
                     double* partials, int nblocks, cudaStream_t st);
// Throughput-form FP64 kernels (cpd_kernels_fast.cu): PMB and LPS.
bool fast_supported(const Model& md);
// wlist: only the listed warps of 32 rows (wcount of them).
int launch_pd_force_fast(const ParticleView& p, const EllView& nl, const Model& md,
                         const StepEpilogue& ep, cudaStream_t st,
                         const int32_t* wlist = nullptr, int64_t wcount = 0);
// Energy / damage of the FP64 and mixed paths (PMB, LPS): -1 for other
// models (the exact kernel serves those).
int launch_pd_energy_fast(const ParticleView& p, const EllView& nl, const Model& md,
                          double* partials, int nblocks, cudaStream_t st);
int launch_lps_m_theta_fast(const ParticleView& p, const EllView& nl, const Model& md,
                            bool with_m, cudaStream_t st);
// ep (optional): the contact-only fused step's epilogue instead of storing f.
int launch_hertz_force(const ParticleView& p, const EllView& nl,
                       const Model& md, bool reset, cudaStream_t st,
                       const StepEpilogue* ep = nullptr);
// Mixed precision (cpd_kernels_mixed.cu): FP64 overlap, FP32 force law.
int launch_hertz_force_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                             bool reset, cudaStream_t st, const StepEpilogue* ep = nullptr);
// Normal repulsion over the contact list (exact FP64).
int launch_repulsion_force(const ParticleView& p, const EllView& nl, const Model& md,
                           bool reset, cudaStream_t st);
int launch_force_bc(const ParticleView& p, const BoundaryCondition& bc,
                    cudaStream_t st);
int launch_prenotch(const ParticleView& p, const EllView& nl, const double* v1,
                    const double* v2, const double* p0, double margin,
                    cudaStream_t st);
int launch_pd_stress(const ParticleView& p, const EllView& nl, const Model& md, double* sigma,
                     cudaStream_t st);
int launch_sum_partials(const double* partials, int nblocks, int ncols,
                        double* out, cudaStream_t st);
int launch_max_partials(const double* partials, int nblocks, double* out,
                        cudaStream_t st);
int energy_blocks(int64_t nrows);
int vv_blocks(int64_t nrows);

// Mixed-precision PMB path (cpd_kernels_mixed.cu).
constexpr int kMixedGeneric = 254;  // bond code: no lattice stencil entry
struct __align__(16) MixedStencil {
    float x, y, z, xi;  // FP32 bond reference vector and its length
    float xiinv;        // 1 / length
    int32_t delta;      // neighbour index - particle index
    float xi2;          // squared length
    int32_t pad;
};
// FP32 split of one particle's displacement, hi and lo together so one
// address serves both loads: u = hi.xyz + lo.xyz; hi.w = c vol (the PMB
// micromodulus times the particle volume), lo.w = no-fail flag.
struct __align__(32) MixedU {
    float4 hi, lo;
};
struct MixedView {
    const float4* xh;  // positions, FP32 hi part
    const float4* xl;  // positions, FP32 lo part (x - hi)
    const MixedU* u2;  // displacement split
    const uint8_t* code;  // [max_n][npad] stencil code per bond slot
    const MixedStencil* table;
    const uint8_t* warp_kind;  // per warp of rows: 2 all rows full stencil, 3 all rows
                               // the same stencil subset, 1 all rows stencil subsets,
                               // 0 otherwise (per-bond codes)
    const uint32_t* pmask;     // [ceil(ntab/32)][npad] stencil entries present per row
    const uint32_t* warp_pmask;  // [warp][ceil(ntab/32)] the common subset of a kind-3 warp
};
// Lattice-stencil bond kernels (cpd_kernels_stencil.cu). On a lattice the
// rows of stencil warps (warp kinds 1-3) hold subsets of one table of bond
// offsets in table order, so bond slot k of a full row is entry k and its
// neighbour is i + delta_k. The table rides in the kernel's parameter space:
// the bond loop is unrolled over the entries, every entry constant is an
// immediate constant-bank operand, and no index or per-bond code is read.
constexpr int kStencilMax = 128;  // entries of the unrolled kernels
constexpr int kStencilPoly = 9;   // coefficients of the FP64 stretch polynomial
// Half-width of the range of q = (r^2 - xi^2) / xi^2 the stretch polynomial
// covers; bonds outside it take the exact formula.
constexpr double kStencilQ = 0.03;
struct __align__(16) StencilEntry64 {
    double ex, ey, ez;        // bond reference vector xi (FP64 lattice offset)
    double tx, ty, tz;        // 2 xi
    double ixi2;              // 1 / xi^2
    // Pair force factor F = (c vol / xi) (1 - xi / r) = K num H(num / xi^2)
    // with K = c vol / xi^3 and the stretch polynomial H (Stencil64::h), so
    // that the pair force is F r_vec (= c s vol r_vec / r,
    // force/CabanaPD_PMB.hpp:266-270).
    double K;
    int64_t boff;             // (neighbour index - particle index) * 32: record bytes
    int32_t doff;             // neighbour index - particle index
    // num lies in the polynomial's range and below the break band when the
    // high word of |num| is below khi.
    uint32_t khi;
};
// The FP64 table in two sizes: up to kStencilMax entries (horizons to ~3.5
// spacings; one struct per launch keeps the parameters small) and up to
// kStencilMaxWide (a horizon of 4 spacings: 256 entries).
constexpr int kStencilMaxWide = 256;
template <int N>
struct Stencil64T {
    int32_t ntab = 0, nwords = 0;
    int32_t np = 0;        // coefficients of h in use (8 or 9)
    double bbc = 0;        // bond_break_coeff (the exact re-test)
    double c = 0;          // micromodulus (the exact formula)
    // H(q) = sum_k h[k] q^k ~ 1 / (sqrt(1+q) (1 + sqrt(1+q))) on |q| <= kStencilQ,
    // so that 1 - xi / r = q H(q) with q = (r^2 - xi^2) / xi^2.
    double h[kStencilPoly];
    // S(q) = sum_k sh[k] q^k ~ 1 / (1 + sqrt(1+q)), the stretch s = q S(q)
    // (output steps' energy).
    double sh[kStencilPoly];
    StencilEntry64 e[N];  // past ntab: zero (no force, never deferred)
    // Energy factor of each entry, c vol xi / 4 (one particle volume).
    double kw[N];
};
using Stencil64 = Stencil64T<kStencilMax>;
using Stencil64W = Stencil64T<kStencilMaxWide>;
// The mixed-precision form (FP32 bond arithmetic on the FP32 split of u).
constexpr int kStencilPoly32 = 4;  // coefficients of the FP32 stretch polynomial
struct __align__(16) StencilEntry32 {
    float2 exy;               // bond reference vector xi (FP32 of the lattice
    float ez;                 // offset), x and y paired for the FP32x2 operations
    float tz;                 // 2 xi (z)
    float2 txy;               // 2 xi (x, y)
    float ixi2;               // 1 / xi^2
    float K;                  // c vol / xi^3 (c / xi^3 with per-particle volumes)
    int64_t boff;             // (neighbour index - particle index) * 32: record bytes
    int32_t doff;             // neighbour index - particle index
    uint32_t khi;             // |num| inside the window: its bits below khi
};
struct Stencil32 {
    int32_t ntab = 0, nwords = 0;
    double bbc = 0, c = 0;
    float h[kStencilPoly32];  // H(q) ~ 1 / (sqrt(1+q) (1 + sqrt(1+q))), FP32
    StencilEntry32 e[kStencilMax];  // past ntab: zero (no force, never deferred)
    // Energy factor of each entry, c vol xi / 4 (one particle volume; the
    // bond's strain energy is kw s^2, force/CabanaPD_PMB.hpp:127-155).
    float kw[kStencilMax];
};

// Where the stencil kernels find their rows: the warp list (kinds 1-3, tile
// order), the kinds, and the per-row presence masks over the table.
struct StencilRows {
    const uint8_t* warp_kind;
    const uint32_t* pmask;  // [ceil(ntab / 32)][npad]
    const int32_t* wlist;
    int64_t wcount;
};

// What a throughput bond kernel does after summing row i's force
// (cpd_epilogue.cuh): mode 0 stores f; mode 1 applies the row's force
// boundary condition and the second half step (v); mode 2 also applies the
// next step's first half step, writing the new displacement to u_next (and
// its FP32 split to u2_next on the mixed path) instead of storing f.
struct StepEpilogue {
    int mode = 0;
    double dt = 0, half_dt = 0;
    double* u_next = nullptr;
    MixedU* u2_next = nullptr;
    double c = 0;                      // PMB micromodulus, for the mixed split
    const uint32_t* bc_bits = nullptr; // [ceil(npad / 32)] rows with a condition
    const int32_t* bc_row = nullptr;   // [nbc] their internal indices, ascending
    const uint8_t* bc_keep = nullptr;  // [nbc] bit 4+d: component d touched;
                                       // bit d: then f_d + add_d, else add_d
    const double* bc_add = nullptr;    // [3][nbc]
    int32_t nbc = 0;
    // Contact steps: neighbours read this row's velocity during the pass
    // (Hertz damping), so the new velocity goes to this second buffer.
    double* v_next = nullptr;
    // FP64 stencil path: the next displacement's gather records as well, at
    // record u4_cell[i] of row i (the lattice-cell layout) or at i (null).
    double4* u4_next = nullptr;
    const int32_t* u4_cell = nullptr;
    // Mixed stencil kernel on an output step: also the rows' strain energy
    // density and damage (W, phi), and per stencil warp the partial sums
    // (sum W_i vol_i, sum phi_i) at energy_part[2 slot], [2 slot + 1].
    double* energy_part = nullptr;
};

struct MixedState {
    float4* xh = nullptr;
    float4* xl = nullptr;
    MixedU* u2 = nullptr;
    uint8_t* code = nullptr;
    MixedStencil* table = nullptr;
    uint8_t* warp_kind = nullptr;
    uint32_t* pmask = nullptr;
    uint32_t* warp_pmask = nullptr;
    int ntab = 0;
    double h[3] = {0, 0, 0};
    size_t bytes = 0;     // device bytes held
    float2* ab = nullptr; // LPS: per-particle FP32 (theta_coeff theta / m, s_coeff / m)
    // PMB split form: warps of kinds 2 / 3 (lean kernel) and the others.
    int32_t* lean_list = nullptr;
    int32_t* rest_list = nullptr;
    int64_t nlean = 0, nrest = 0;
    int lps_ok = 0;       // LPS: every row is a stencil row (the mixed LPS kernels apply)
    // All particles of one volume v: vol_sums[k] = v + v + ... (k terms,
    // summed in order), the FP64 volume sum of any k bonds; else nullptr.
    double* vol_sums = nullptr;
    double vol_uniform = 0;
    // LPS with one particle volume and no frozen particles: per particle the
    // FP32 split of u with the force factors a, b in the w lanes (written by
    // the m / theta pass, read by the lean force kernel in place of u2 and
    // ab), so a neighbour is one 32-byte record.
    MixedU* u2ab = nullptr;
    // FP64 stencil path (CPD_FP64, PMB): the table in kernel-parameter form
    // (host memory, built at set-up), and the displacement as 32-byte gather
    // records (u_x, u_y, u_z, vol) with `guard` zero records on either side,
    // so i + delta of an absent stencil entry stays inside the allocation.
    Stencil64* st64 = nullptr;
    Stencil64W* st64w = nullptr;  // tables past kStencilMax entries
    // The FP64 stencil walk runs in two launches: the first one's force sum
    // per row (x, y, z; w unused), which the second one continues.
    double4* f64part = nullptr;
    // Lattice-cell layout of the FP64 gather records (a lattice body whose
    // particle order is not one box of lattice lines, e.g. with holes): row
    // i's record is u4[gcell[i]], gcell[i] = a + nx (b + ny c) from its
    // lattice coordinates, so that entry k is always record gcell[i] +
    // delta_k; cells without a particle hold zero records. Null: records by
    // row (u4[i]), the table's deltas then being index deltas.
    int32_t* gcell = nullptr;
    int64_t grid_cells = 0;
    // Mixed PMB stencil kernel: its table, and the allocation behind u2
    // (u2 = u2_base + guard; `guard` zero records on either side).
    Stencil32* st32 = nullptr;
    MixedU* u2_base = nullptr;
    double4* u4 = nullptr;       // record of particle 0
    double4* u4_base = nullptr;  // allocation
    double4* u4_alt = nullptr;   // the fused step's second buffer, same form
    double4* u4_alt_base = nullptr;
    int64_t guard = 0;
    int64_t nstencil = 0;        // warps of kinds 1-3 (stencil_list)
    int32_t* stencil_list = nullptr;
    int64_t nirregular = 0;      // warps of kind 0 (irregular_list)
    int32_t* irregular_list = nullptr;
};
// lps: set up the LPS mixed kernels too (lps_ok, ab). fp64_stencil: set up
// the stencil data for the FP64 stencil kernel only (no FP32 copies).
// md_pmb (mixed PMB): also the table of the mixed stencil kernel.
int prepare_mixed(const ParticleView& p, const NeighborList& pd, double cutoff, bool lps,
                  MixedState& m, cudaStream_t st, std::string& err,
                  const Model* fp64_stencil = nullptr, const Model* md_pmb = nullptr);
// FP64 stencil path (cpd_kernels_stencil.cu).
// Builds m.st64 and the gather records (false: the stencil does not apply).
// Entries of the lattice table for per-axis spacings h within cutoff (the
// offsets prepare_mixed tabulates).
int lattice_table_entries(const double* h, double cutoff);
// The FP64 stencil records' layout a body would take (0: not a lattice of
// distinct cells; 1: one box of lattice lines in row order; 2: by lattice
// cell), from its positions and spacings h; synchronises the stream.
int lattice_layout_probe(const ParticleView& p, const double* h, cudaStream_t st);
bool prepare_stencil64(const ParticleView& p, const Model& md, const double* h,
                       const MixedStencil* tab, int ntab, MixedState& m, cudaStream_t st,
                       std::string& err);
void free_stencil64(MixedState& m, cudaStream_t st);
bool stencil64_ready(const MixedState& m);
// Mixed PMB: builds m.st32 (false: the stencil kernel does not apply).
bool prepare_stencil32(const Model& md, const double* h, const MixedStencil* tab, int ntab,
                       MixedState& m);
int launch_pd_force_stencil32(const ParticleView& p, const EllView& nl, const Model& md,
                              const MixedState& m, const StepEpilogue& ep, cudaStream_t st);
// Gather records of rows [begin, end) from the displacement u (SoA).
// Rows [begin, end) of u (and vol) as gather records: u4[cell[i]], or u4[i]
// when cell is null.
int launch_pack_u4(const ParticleView& p, const double* u, int64_t begin, int64_t end,
                   double4* u4, cudaStream_t st, const int32_t* cell = nullptr);
int launch_pd_force_stencil64(const ParticleView& p, const EllView& nl, const Model& md,
                              const MixedState& m, const StepEpilogue& ep, cudaStream_t st);
// Energy and damage of the listed warps' rows on the mixed path (the rows
// the mixed stencil kernel does not hold, after its output step): block
// partials at partials; returns the partial rows written, -1 when the
// mixed energy kernels do not serve the model.
int launch_energy_mixed_rows(const ParticleView& p, const EllView& nl, const Model& md,
                             const MixedState& m, const int32_t* wlist, int64_t wcount,
                             double* partials, int* launches, cudaStream_t st);
int launch_lps_mtheta_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                            const MixedState& m, bool with_m, cudaStream_t st);
double mixed_wscale(const Model& md);
void free_mixed(MixedState& m, cudaStream_t st);
int launch_split_u(const ParticleView& p, const Model& md, MixedState& m, cudaStream_t st);
int launch_vv_initial_mixed(const ParticleView& p, const Model& md, double dt, double* u_out,
                            MixedU* u2_out, cudaStream_t st);
// Energy / damage on the mixed path into [.][2] block partials: returns the
// number of partial rows written (nblocks, or more when the split form fits
// in capacity rows), -1 when the mixed data does not apply.
int launch_energy_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                        const MixedState& m, double* partials, int nblocks, int capacity,
                        int* launches, cudaStream_t st);
int launch_pd_force_mixed(const ParticleView& p, const EllView& nl, const Model& md,
                          const MixedState& m, const StepEpilogue& ep, cudaStream_t st);
// Neighbour build (cpd_neighbor.cu). Builds rows for [begin, n) from
// positions pos (+ optional displacement disp) with squared distance
// <= cutoff^2; rows sorted by ascending user_id of the neighbour.
struct BuildScratch;
int build_neighbor_list(const double* pos, const double* disp, int64_t n,
                        int64_t npad, int64_t begin, double cutoff,
                        const int32_t* user_id, bool with_mu,
                        NeighborList& out, cudaStream_t st, std::string& err,
                        double* min_spacing = nullptr);
void free_neighbor_list(NeighborList& nl, cudaStream_t st);

// Layout kernels.
int launch_aos_to_soa(const double* aos, double* soa, int64_t n, int64_t npad,
                      int comps, const int32_t* perm, cudaStream_t st);
int launch_fill_value(double* a, int64_t n, double v, cudaStream_t st);
int launch_nofail_to_u8(const int32_t* src, uint8_t* dst, int64_t n, const int32_t* perm,
                        cudaStream_t st);
int launch_soa_to_aos(const double* soa, double* aos, int64_t n, int64_t npad,
                      int comps, const int32_t* perm, cudaStream_t st);
int launch_ell_to_rows(const NeighborList& nl, int64_t n, int64_t npad,
                       const int32_t* perm, const int32_t* user_id,
                       int32_t* counts, int32_t* indices, int32_t* mu,
                       cudaStream_t st);

// ---------------------------------------------------------------------------
// Batched step of many systems (cpd_batch.cu). Each instance is a set-up
// system; the batch kernels read its device views from a table
// (BatchInstance, one per instance) and take their rows in tiles of up to
// kBatchTileWarps chunks of 32 rows of one instance. Per chunk of K steps an
// instance advances r = min(K, remaining) steps: the first half step into
// buffer (r - 1) & 1 (0: the system's own arrays, 1: its second buffers), then
// per step s < r one bond pass whose epilogue writes the other buffer, so
// that the last step ends in the system's arrays, as cpd_step's fused step.
constexpr int kBatchTileWarps = 8;
// Step s of a K-step chunk for an instance with `remaining` steps left:
// r = min(K, remaining); the step runs when s < r, reads buffer cur =
// ((r - 1) ^ s) & 1 and writes the other, and its epilogue takes the next
// first half step (mode 2) but on the last step (mode 1).
struct BatchStep {
    int run, cur, mode;
};
__host__ __device__ inline BatchStep batch_step(int32_t remaining, int32_t K, int32_t s)
{
    const int32_t r = remaining < K ? remaining : K;
    BatchStep b;
    b.run = s < r;
    b.cur = ((r - 1) ^ s) & 1;
    b.mode = s + 1 < r ? 2 : 1;
    return b;
}
enum BatchBody : int32_t { kBatchFast = 0, kBatchMixed = 1 };
struct BatchInstance {
    ParticleView p;      // p.u: buffer 0 (the system's displacement)
    EllView nl;          // PD list (mu null without fracture)
    StepEpilogue ep;     // dt, boundary-condition row program, split factor
    MixedView mv;        // mixed body: mv.u2 = buffer 0's FP32 split
    double* u_alt;       // buffer 1
    MixedU* u2_alt;      // buffer 1's split (mixed body)
    float2* ab;          // mixed LPS: FP32 force factors per particle
    FastModel fm;
    MixedModel mm;
    MixedLps ml;
    double wscale;       // the mixed split's factor (c for PMB, 1 for LPS)
    int32_t body;        // BatchBody
    int32_t pd;          // CPD_PD_PMB or CPD_PD_LPS
    int32_t fracture, influence;
};
struct BatchTile {
    int32_t inst;        // instance
    int32_t warp0;       // first chunk of 32 rows (counted from the first movable row)
    int32_t nwarps;      // chunks in the tile (<= kBatchTileWarps)
    int32_t lps;         // 1: the instance is an LPS instance
};
// One pass of step s of a K-step chunk over the tiles of one body: pass 0
// the LPS weighted volume / dilatation of LPS tiles, pass 1 the bond force
// and step epilogue. Persistent blocks: grid blocks take tiles grid apart.
int launch_batch_fast(const BatchInstance* inst, const int32_t* remaining,
                      const BatchTile* tiles, int32_t ntiles, int32_t K, int32_t s,
                      int32_t pass, int grid, cudaStream_t st);
int launch_batch_mixed(const BatchInstance* inst, const int32_t* remaining,
                       const BatchTile* tiles, int32_t ntiles, int32_t K, int32_t s,
                       int32_t pass, int grid, cudaStream_t st);
// Resident blocks per SM of the batch kernels (occupancy at their launch
// bounds), for the persistent grid.
int batch_fast_blocks_per_sm();
int batch_mixed_blocks_per_sm();
// System side of a batch (cpd_api.cu): batch_attach validates system s
// (set up, initialised, PD without contact, CPD_FP64 or CPD_MIXED, fused step
// prepared), fills its table entry and directed-bond count, and marks it as
// advanced by `batch` (state-changing calls are then refused until
// batch_detach).
cpd_status batch_attach(cpd_system* s, const void* batch, BatchInstance* out, int64_t* bonds);
void batch_detach(cpd_system* s);
cudaStream_t system_stream(const cpd_system* s);
int system_device(const cpd_system* s);
int64_t system_rows(const cpd_system* s);
// The stream a batch issues its chunks on (cpd_batch.cu).
cudaStream_t batch_stream(const cpd_batch* b);
// Model constant forms of the throughput kernels.
FastModel to_fast(const Model& m);
MixedModel to_mixed_model(const Model& md, const MixedState& m);
MixedLps to_mixed_lps(const Model& md, const MixedState& m);

}  // namespace cpd
