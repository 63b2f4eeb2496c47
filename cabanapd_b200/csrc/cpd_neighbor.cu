// Linked-cell full neighbour list build and layout kernels.
//
// Restates what the reference's Neighbor constructor obtains from
// Cabana::VerletList<FullNeighborTag, VerletLayout2D>
// (CabanaPD_Neighbor.hpp:44-66, 107-132): every particle is a candidate
// neighbour, rows exist for particles [begin, n), and j is a neighbour of i
// when |pos_j - pos_i|^2 <= cutoff^2. Compiled with --fmad=false so the
// squared distance rounds as a scalar evaluation does; the neighbour SET is
// therefore identical to the CPU oracle's.
//
// Steps: bounding box -> cell size (>= cutoff) -> cell index per particle ->
// counting sort into cells -> per-row count over the 27 surrounding cells ->
// max / total -> per-row fill, rows sorted by ascending caller index (the
// order the oracle sums in) -> intact-bond bits.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>

#include "cpd_internal.cuh"

namespace cpd {
namespace {

constexpr int kBlock = 256;
constexpr int kLocalRow = 256;  // rows up to this length are sorted in registers/local memory

inline int blocks_for(int64_t rows) { return (int)((rows + kBlock - 1) / kBlock); }

struct Grid {
    double lo[3];
    double cell;
    int32_t nc[3];
    int32_t R;  // visit radius in cells: every pair within the cutoff is at most R cells apart
};

__global__ void k_positions(const double* x, const double* disp, double* y, int64_t n,
                            int64_t npad)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int d = 0; d < 3; d++) y[d * npad + i] = x[d * npad + i] + disp[d * npad + i];
}

__global__ void k_bbox(const double* pos, int64_t n, int64_t npad, double* partial)
{
    __shared__ double s[6][kBlock];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int d = 0; d < 3; d++) {
        double v = i < n ? pos[d * npad + i] : pos[d * npad];
        s[d][threadIdx.x] = v;
        s[3 + d][threadIdx.x] = v;
    }
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int d = 0; d < 3; d++) {
                s[d][threadIdx.x] = fmin(s[d][threadIdx.x], s[d][threadIdx.x + w]);
                s[3 + d][threadIdx.x] = fmax(s[3 + d][threadIdx.x], s[3 + d][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 6; c++) partial[6 * blockIdx.x + c] = s[c][0];
}

__device__ __forceinline__ void cell_coords(const Grid& g, double px, double py, double pz,
                                            int32_t c[3])
{
    const double p[3] = {px, py, pz};
    for (int d = 0; d < 3; d++) {
        double k = floor((p[d] - g.lo[d]) / g.cell);
        int32_t kk = (int32_t)fmax(0.0, fmin(k, (double)(g.nc[d] - 1)));
        c[d] = kk;
    }
}

__global__ void k_cell_index(const double* pos, int64_t n, int64_t npad, Grid g,
                             int32_t* cell, int32_t* cell_count)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int32_t c[3];
    cell_coords(g, pos[i], pos[npad + i], pos[2 * npad + i], c);
    const int32_t id = c[0] + g.nc[0] * (c[1] + g.nc[1] * c[2]);
    cell[i] = id;
    atomicAdd(cell_count + id, 1);
}

__global__ void k_cell_fill(const int32_t* cell, int64_t n, const int32_t* cell_start,
                            int32_t* cursor, int32_t* order)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t c = cell[i];
    const int32_t slot = atomicAdd(cursor + c, 1);
    order[cell_start[c] + slot] = (int32_t)i;
}

// Calls emit(j) for every j != i within the cutoff: walks the (2R + 1)^2
// lines of cells around particle i in increasing (z, y); the cells of one
// line are consecutive cell ids, so their particles are one contiguous run
// of the cell-sorted order. With cells about cutoff / 3 wide, a lattice
// holds about one particle per cell and an x-fastest lattice row is emitted
// in nearly ascending index order (the row sort then moves little).
template <typename Emit>
__device__ __forceinline__ void visit_neighbors(const double* __restrict__ pos, int64_t npad,
                                                const Grid& g, const int32_t* __restrict__ cell_start,
                                                const int32_t* __restrict__ order, int64_t i,
                                                double rsqr, Emit&& emit)
{
    const double px = pos[i], py = pos[npad + i], pz = pos[2 * npad + i];
    int32_t c[3];
    cell_coords(g, px, py, pz, c);
    const int32_t cx0 = max(c[0] - g.R, 0), cx1 = min(c[0] + g.R, g.nc[0] - 1);
    for (int dz = -g.R; dz <= g.R; dz++) {
        const int32_t cz = c[2] + dz;
        if (cz < 0 || cz >= g.nc[2]) continue;
        for (int dy = -g.R; dy <= g.R; dy++) {
            const int32_t cy = c[1] + dy;
            if (cy < 0 || cy >= g.nc[1]) continue;
            const int64_t line = (int64_t)g.nc[0] * (cy + (int64_t)g.nc[1] * cz);
            const int32_t q1 = cell_start[line + cx1 + 1];
            for (int32_t q = cell_start[line + cx0]; q < q1; q++) {
                const int64_t j = order[q];
                if (j == i) continue;
                const double ddx = pos[j] - px;
                const double ddy = pos[npad + j] - py;
                const double ddz = pos[2 * npad + j] - pz;
                const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                if (d2 <= rsqr) emit(j);
            }
        }
    }
}

// min_out (optional, 3 slots): per axis the smallest nonzero |x_j - x_i|
// over the accepted pairs (the bit patterns of non-negative doubles order
// like the values), the lattice spacing the mixed path's stencil needs.
__global__ void __launch_bounds__(kBlock)
    k_count(const double* pos, int64_t n, int64_t npad, int64_t begin, Grid g,
            const int32_t* cell_start, const int32_t* order, double rsqr, int32_t* count,
            unsigned long long* min_out)
{
    __shared__ unsigned long long s_min[3][kBlock];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double m[3] = {INFINITY, INFINITY, INFINITY};
    if (i < npad) {
        if (i < begin || i >= n) {
            count[i] = 0;
        } else {
            int32_t cnt = 0;
            const double xi0 = pos[i], xi1 = pos[npad + i], xi2 = pos[2 * npad + i];
            visit_neighbors(pos, npad, g, cell_start, order, i, rsqr, [&](int64_t j) {
                cnt++;
                if (min_out) {
                    const double a0 = fabs(pos[j] - xi0), a1 = fabs(pos[npad + j] - xi1),
                                 a2 = fabs(pos[2 * npad + j] - xi2);
                    if (a0 > 0.0) m[0] = fmin(m[0], a0);
                    if (a1 > 0.0) m[1] = fmin(m[1], a1);
                    if (a2 > 0.0) m[2] = fmin(m[2], a2);
                }
            });
            count[i] = cnt;
        }
    }
    if (!min_out) return;  // uniform across the grid
    for (int d = 0; d < 3; ++d) s_min[d][threadIdx.x] = __double_as_longlong(m[d]);
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int d = 0; d < 3; ++d)
                s_min[d][threadIdx.x] = min(s_min[d][threadIdx.x], s_min[d][threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < 3; ++d) atomicMin(min_out + d, s_min[d][0]);
}

__global__ void k_count_stats(const int32_t* count, int64_t npad, int32_t* block_max,
                              long long* block_sum)
{
    __shared__ int32_t smax[kBlock];
    __shared__ long long ssum[kBlock];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t c = i < npad ? count[i] : 0;
    smax[threadIdx.x] = c;
    ssum[threadIdx.x] = c;
    __syncthreads();
    for (int w = kBlock / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            smax[threadIdx.x] = max(smax[threadIdx.x], smax[threadIdx.x + w]);
            ssum[threadIdx.x] += ssum[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        block_max[blockIdx.x] = smax[0];
        block_sum[blockIdx.x] = ssum[0];
    }
}

// Fill row i and sort it by the caller index of the neighbour. Rows that fit
// kLocalRow are sorted in a thread-local array; longer rows are sorted in
// place in the column-major list.
__global__ void __launch_bounds__(kBlock)
    k_fill(const double* pos, int64_t n, int64_t npad, int64_t begin, Grid g,
           const int32_t* cell_start, const int32_t* order, double rsqr,
           const int32_t* count, const int32_t* user_id, int32_t max_n, int32_t* idx)
{
    const int64_t i = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t cnt = count[i];
    auto key = [&](int32_t j) -> int32_t { return user_id ? user_id[j] : j; };
    if (cnt <= kLocalRow) {
        int32_t row[kLocalRow];
        int32_t k = 0;
        visit_neighbors(pos, npad, g, cell_start, order, i, rsqr, [&](int64_t j) {
            if (k < kLocalRow) row[k] = (int32_t)j;
            k++;
        });
        for (int32_t a = 1; a < cnt; a++) {
            const int32_t v = row[a];
            const int32_t kv = key(v);
            int32_t b = a - 1;
            while (b >= 0 && key(row[b]) > kv) {
                row[b + 1] = row[b];
                b--;
            }
            row[b + 1] = v;
        }
        for (int32_t a = 0; a < cnt; a++) idx[(int64_t)a * npad + i] = row[a];
    } else {
        int32_t k = 0;
        visit_neighbors(pos, npad, g, cell_start, order, i, rsqr, [&](int64_t j) {
            if (k < max_n) idx[(int64_t)k * npad + i] = (int32_t)j;
            k++;
        });
        for (int32_t a = 1; a < cnt; a++) {
            const int32_t v = idx[(int64_t)a * npad + i];
            const int32_t kv = key(v);
            int32_t b = a - 1;
            while (b >= 0 && key(idx[(int64_t)b * npad + i]) > kv) {
                idx[(int64_t)(b + 1) * npad + i] = idx[(int64_t)b * npad + i];
                b--;
            }
            idx[(int64_t)(b + 1) * npad + i] = v;
        }
    }
    for (int32_t a = cnt; a < max_n; a++) idx[(int64_t)a * npad + i] = (int32_t)i;
}

__global__ void k_init_mu(const int32_t* count, int64_t npad, int32_t nwords, uint32_t* mu)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npad) return;
    const int32_t cnt = count[i];
    for (int32_t w = 0; w < nwords; w++) {
        const int32_t left = cnt - 32 * w;
        uint32_t word = left >= 32 ? 0xffffffffu : (left <= 0 ? 0u : ((1u << left) - 1u));
        mu[(int64_t)w * npad + i] = word;
    }
}

__global__ void k_aos_to_soa(const double* aos, double* soa, int64_t n, int64_t npad,
                             int comps, const int32_t* perm)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t src = perm ? perm[k] : k;
    for (int d = 0; d < comps; d++) soa[d * npad + k] = aos[src * comps + d];
}

__global__ void k_fill_value(double* a, int64_t n, double v)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) a[k] = v;
}

// Caller-order int32 no-fail flags -> internal-order bytes.
__global__ void k_nofail_to_u8(const int32_t* src, uint8_t* dst, int64_t n, const int32_t* perm)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    dst[k] = src[perm ? perm[k] : k] != 0;
}

__global__ void k_soa_to_aos(const double* soa, double* aos, int64_t n, int64_t npad,
                             int comps, const int32_t* perm)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t dst = perm ? perm[k] : k;
    for (int d = 0; d < comps; d++) aos[dst * comps + d] = soa[d * npad + k];
}

// Row k of the internal list -> caller row perm[k], neighbour indices
// translated to caller indices (already in ascending caller order).
__global__ void k_ell_to_rows(const int32_t* count, const int32_t* idx, const uint32_t* mu,
                              int64_t n, int64_t npad, int32_t max_n, const int32_t* perm,
                              const int32_t* user_id, int32_t* out_counts, int32_t* out_idx,
                              int32_t* out_mu)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int64_t row = perm ? perm[k] : k;
    const int32_t cnt = count[k];
    if (out_counts) out_counts[row] = cnt;
    for (int32_t a = 0; a < max_n; a++) {
        const bool valid = a < cnt;
        if (out_idx) {
            int32_t j = idx[(int64_t)a * npad + k];
            out_idx[row * max_n + a] = valid ? (user_id ? user_id[j] : j) : -1;
        }
        if (out_mu) {
            int32_t bit = 0;
            if (valid && mu) bit = (mu[(int64_t)(a >> 5) * npad + k] >> (a & 31)) & 1u;
            out_mu[row * max_n + a] = bit;
        }
    }
}

#define CPD_TRY(call)                                                           \
    do {                                                                        \
        cudaError_t e_ = (call);                                                \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);           \
            return -1;                                                          \
        }                                                                       \
    } while (0)

}  // namespace

void free_neighbor_list(NeighborList& nl, cudaStream_t st)
{
    if (nl.count) dev_free(nl.count, st);
    if (nl.idx) dev_free(nl.idx, st);
    if (nl.mu) dev_free(nl.mu, st);
    nl = NeighborList{};
}

// Index delta from a row to its nearest neighbour straight along +y (same x
// and z within tol): the line pitch of an x-fastest lattice, used only to
// group bond-kernel warps (tile_view).
__global__ void k_row_pitch(const double* __restrict__ pos, int64_t npad, int64_t row,
                            const int32_t* __restrict__ count, const int32_t* __restrict__ idx,
                            double tol, long long* out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int cnt = count[row];
    double best = INFINITY;
    long long d = 0;
    for (int k = 0; k < cnt; ++k) {
        const int64_t j = idx[(int64_t)k * npad + row];
        const double dx = pos[j] - pos[row];
        const double dy = pos[npad + j] - pos[npad + row];
        const double dz = pos[2 * npad + j] - pos[2 * npad + row];
        if (fabs(dx) <= tol && fabs(dz) <= tol && dy > tol && dy < best) {
            best = dy;
            d = (long long)(j - row);
        }
    }
    *out = d < 0 ? -d : d;
}

int build_neighbor_list(const double* x, const double* disp, int64_t n, int64_t npad,
                        int64_t begin, double cutoff, const int32_t* user_id,
                        bool with_mu, NeighborList& out, cudaStream_t st,
                        std::string& err, double* min_spacing)
{
    int launches = 0;
    PhaseTrace tr("list");
    const double* pos = x;
    double* y = nullptr;
    if (disp) {
        CPD_TRY(dev_alloc(&y, sizeof(double) * 3 * npad, st));
        k_positions<<<blocks_for(n), kBlock, 0, st>>>(x, disp, y, n, npad);
        launches++;
        pos = y;
    }
    // Bounding box.
    const int nb = blocks_for(n);
    double* d_part = nullptr;
    CPD_TRY(dev_alloc(&d_part, sizeof(double) * 6 * nb, st));
    k_bbox<<<nb, kBlock, 0, st>>>(pos, n, npad, d_part);
    launches++;
    std::vector<double> part(6 * (size_t)nb);
    CPD_TRY(cudaMemcpyAsync(part.data(), d_part, sizeof(double) * 6 * nb,
                            cudaMemcpyDeviceToHost, st));
    CPD_TRY(cudaStreamSynchronize(st));
    CPD_TRY(dev_free(d_part, st));
    double lo[3], hi[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = part[d];
        hi[d] = part[3 + d];
    }
    for (int b = 1; b < nb; b++)
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], part[6 * b + d]);
            hi[d] = std::max(hi[d], part[6 * b + 3 + d]);
        }
    // Cells a little over a third of the cutoff wide (visit radius 3), grown
    // by doubling while the grid would hold far more cells than particles
    // (visit radius 2, then 1). The 1e-9 margin keeps cutoff / cell below the
    // radius, so pairs within the cutoff are at most R cells apart.
    Grid g;
    double cell = cutoff / 3.0 * (1.0 + 1e-9);
    for (;;) {
        for (int d = 0; d < 3; d++) {
            double span = (hi[d] - lo[d]) / cell;
            g.nc[d] = (int32_t)std::max<int64_t>(1, std::min<int64_t>((int64_t)span + 1, 1 << 20));
        }
        if ((double)g.nc[0] * g.nc[1] * g.nc[2] <= 4.0 * (double)n + 4096.0) break;
        cell *= 2.0;
    }
    for (int d = 0; d < 3; d++) g.lo[d] = lo[d];
    g.cell = cell;
    g.R = std::max(1, (int32_t)std::ceil(cutoff / cell - 1e-9));
    const int64_t ncell = (int64_t)g.nc[0] * g.nc[1] * g.nc[2];

    int32_t *cellid = nullptr, *cell_count = nullptr, *cell_start = nullptr, *order = nullptr;
    CPD_TRY(dev_alloc(&cellid, sizeof(int32_t) * n, st));
    CPD_TRY(dev_alloc(&cell_count, sizeof(int32_t) * (ncell + 1), st));
    CPD_TRY(dev_alloc(&cell_start, sizeof(int32_t) * (ncell + 1), st));
    CPD_TRY(dev_alloc(&order, sizeof(int32_t) * n, st));
    CPD_TRY(cudaMemsetAsync(cell_count, 0, sizeof(int32_t) * (ncell + 1), st));
    k_cell_index<<<blocks_for(n), kBlock, 0, st>>>(pos, n, npad, g, cellid, cell_count);
    launches++;
    size_t tmp_bytes = 0;
    CPD_TRY(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, cell_count, cell_start,
                                          (int)(ncell + 1), st));
    void* tmp = nullptr;
    CPD_TRY(dev_alloc(&tmp, tmp_bytes, st));
    CPD_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, cell_count, cell_start,
                                          (int)(ncell + 1), st));
    launches++;
    CPD_TRY(cudaMemsetAsync(cell_count, 0, sizeof(int32_t) * (ncell + 1), st));
    k_cell_fill<<<blocks_for(n), kBlock, 0, st>>>(cellid, n, cell_start, cell_count, order);
    launches++;

    tr.mark("cells", st);
    // Row counts.
    if (!out.count) CPD_TRY(dev_alloc(&out.count, sizeof(int32_t) * npad, st));
    const double rsqr = cutoff * cutoff;
    unsigned long long* d_min = nullptr;
    if (min_spacing) {
        CPD_TRY(dev_alloc(&d_min, 3 * sizeof(unsigned long long), st));
        CPD_TRY(cudaMemsetAsync(d_min, 0x7f, 3 * sizeof(unsigned long long), st));
    }
    k_count<<<blocks_for(npad), kBlock, 0, st>>>(pos, n, npad, begin, g, cell_start, order,
                                                 rsqr, out.count, d_min);
    launches++;
    unsigned long long hmin[3] = {0, 0, 0};
    if (d_min)
        CPD_TRY(cudaMemcpyAsync(hmin, d_min, sizeof(hmin), cudaMemcpyDeviceToHost, st));
    const int nbc = blocks_for(npad);
    int32_t* d_bmax = nullptr;
    long long* d_bsum = nullptr;
    CPD_TRY(dev_alloc(&d_bmax, sizeof(int32_t) * nbc, st));
    CPD_TRY(dev_alloc(&d_bsum, sizeof(long long) * nbc, st));
    k_count_stats<<<nbc, kBlock, 0, st>>>(out.count, npad, d_bmax, d_bsum);
    launches++;
    std::vector<int32_t> bmax(nbc);
    std::vector<long long> bsum(nbc);
    CPD_TRY(cudaMemcpyAsync(bmax.data(), d_bmax, sizeof(int32_t) * nbc,
                            cudaMemcpyDeviceToHost, st));
    CPD_TRY(cudaMemcpyAsync(bsum.data(), d_bsum, sizeof(long long) * nbc,
                            cudaMemcpyDeviceToHost, st));
    CPD_TRY(cudaStreamSynchronize(st));
    CPD_TRY(dev_free(d_bmax, st));
    CPD_TRY(dev_free(d_bsum, st));
    if (d_min) {
        CPD_TRY(dev_free(d_min, st));
        for (int d = 0; d < 3; ++d) std::memcpy(&min_spacing[d], &hmin[d], sizeof(double));
    }
    int32_t max_n = 0;
    long long total = 0;
    for (int b = 0; b < nbc; b++) {
        max_n = std::max(max_n, bmax[b]);
        total += bsum[b];
    }
    tr.mark("count", st);
    // (Re)allocate the padded list when it grows.
    const int32_t cap = std::max(max_n, 1);
    if (!out.idx || cap > out.cap) {
        if (out.idx) CPD_TRY(dev_free(out.idx, st));
        out.idx = nullptr;
        CPD_TRY(dev_alloc(&out.idx, sizeof(int32_t) * (size_t)cap * npad, st));
        out.cap = cap;
        out.bytes = sizeof(int32_t) * (size_t)npad * (1 + (size_t)cap);
        if (with_mu) {
            if (out.mu) CPD_TRY(dev_free(out.mu, st));
            out.mu = nullptr;
            const int32_t nw = (cap + 31) / 32;
            CPD_TRY(dev_alloc(&out.mu, sizeof(uint32_t) * (size_t)nw * npad, st));
            out.bytes += sizeof(uint32_t) * (size_t)nw * npad;
        }
    }
    out.max_n = max_n;
    out.total = total;
    out.nwords = (max_n + 31) / 32;
    tr.mark("alloc", st);
    if (n > begin) {
        k_fill<<<blocks_for(n - begin), kBlock, 0, st>>>(pos, n, npad, begin, g, cell_start,
                                                        order, rsqr, out.count, user_id,
                                                        max_n, out.idx);
        launches++;
    }
    if (with_mu && out.nwords > 0) {
        k_init_mu<<<blocks_for(npad), kBlock, 0, st>>>(out.count, npad, out.nwords, out.mu);
        launches++;
    }
    tr.mark("fill", st);
    // Lists on reference positions (PD bonds): the lattice line pitch at a
    // middle row.
    out.pitch = 0;
    if (!disp && n > begin && max_n > 0) {
        long long* d_pitch = nullptr;
        CPD_TRY(dev_alloc(&d_pitch, sizeof(long long), st));
        k_row_pitch<<<1, 32, 0, st>>>(pos, npad, begin + (n - begin) / 2, out.count, out.idx,
                                      1e-6 * cutoff, d_pitch);
        launches++;
        long long pitch = 0;
        CPD_TRY(cudaMemcpyAsync(&pitch, d_pitch, sizeof(pitch), cudaMemcpyDeviceToHost, st));
        CPD_TRY(cudaStreamSynchronize(st));
        CPD_TRY(dev_free(d_pitch, st));
        out.pitch = pitch;
    }
    CPD_TRY(cudaGetLastError());
    CPD_TRY(dev_free(tmp, st));
    CPD_TRY(dev_free(cellid, st));
    CPD_TRY(dev_free(cell_count, st));
    CPD_TRY(dev_free(cell_start, st));
    CPD_TRY(dev_free(order, st));
    if (y) CPD_TRY(dev_free(y, st));
    return launches;
}

int launch_aos_to_soa(const double* aos, double* soa, int64_t n, int64_t npad, int comps,
                      const int32_t* perm, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_aos_to_soa<<<blocks_for(n), kBlock, 0, st>>>(aos, soa, n, npad, comps, perm);
    return 1;
}

int launch_fill_value(double* a, int64_t n, double v, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_fill_value<<<blocks_for(n), kBlock, 0, st>>>(a, n, v);
    return 1;
}

int launch_nofail_to_u8(const int32_t* src, uint8_t* dst, int64_t n, const int32_t* perm,
                        cudaStream_t st)
{
    if (n <= 0) return 0;
    k_nofail_to_u8<<<blocks_for(n), kBlock, 0, st>>>(src, dst, n, perm);
    return 1;
}

int launch_soa_to_aos(const double* soa, double* aos, int64_t n, int64_t npad, int comps,
                      const int32_t* perm, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_soa_to_aos<<<blocks_for(n), kBlock, 0, st>>>(soa, aos, n, npad, comps, perm);
    return 1;
}

int launch_ell_to_rows(const NeighborList& nl, int64_t n, int64_t npad, const int32_t* perm,
                       const int32_t* user_id, int32_t* counts, int32_t* indices,
                       int32_t* mu, cudaStream_t st)
{
    if (n <= 0) return 0;
    k_ell_to_rows<<<blocks_for(n), kBlock, 0, st>>>(nl.count, nl.idx, nl.mu, n, npad,
                                                     nl.max_n, perm, user_id, counts,
                                                     indices, mu);
    return 1;
}

}  // namespace cpd
