// Batched step of many systems (cpd_batch_*). No counterpart in the
// reference, which advances one specimen per process with one kernel per
// phase and a fence after each (CabanaPD_Solver.hpp:332-404,
// CabanaPD_Force.hpp:176-198).
//
// A batch holds a device table of per-instance views (BatchInstance: the
// instance's particle, neighbour-list, boundary-condition and mixed-precision
// arrays, at their offsets in the device pool) and a tile list over all
// instances' movable rows (up to kBatchTileWarps chunks of 32 rows of one
// instance per tile). A chunk of K steps is:
//   k_batch_vv_initial             first half step of every instance that
//                                  still has steps, into buffer (r - 1) & 1
//   per step s < K: [LPS pass]     k_batch_fast / k_batch_mixed pass 0
//                   bond pass      pass 1: force, breaking, BC, second half
//                                  step and the next first half step
//   k_batch_advance                remaining -= min(K, remaining)
// with r = min(K, remaining) per instance (batch_step), captured once per
// (K, launch shape) as a CUDA graph and replayed. The persistent blocks of
// the pass kernels take tiles grid apart, so one launch covers every
// instance whatever their sizes.
//
// Launch shapes (autotuner candidates): persistent grid of 1, 2 or the
// occupancy limit of blocks per SM, tiles by instance or interleaved across
// instances. A row's arithmetic does not depend on which block runs it, so
// every candidate gives identical results; the first chunks run one
// candidate each, timed with CUDA events, and the fastest (bond-updates per
// second over the chunk's work) is kept.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "cpd_epilogue.cuh"
#include "cpd_internal.cuh"

using namespace cpd;

namespace {

constexpr int kBlock = 256;

cpd_status fail(cpd_status code, const std::string& msg)
{
    set_last_error(msg);
    return code;
}

// First half step (CabanaPD_Integrate.hpp:89-116) of every movable row of
// every instance that still has steps, into buffer (r - 1) & 1 (and the FP32
// split for mixed instances); each operation separately rounded, as
// k_vv_initial / k_vv_initial_mixed.
__global__ void __launch_bounds__(kBlock)
    k_batch_vv_initial(const BatchInstance* __restrict__ insts,
                       const int32_t* __restrict__ remaining, const BatchTile* __restrict__ tiles,
                       int32_t ntiles, int32_t K)
{
    const int w = threadIdx.x >> 5;
    for (int32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const BatchTile tl = tiles[t];
        if (w >= tl.nwarps) continue;
        const BatchStep bs = batch_step(remaining[tl.inst], K, 0);
        if (!bs.run) continue;
        const BatchInstance& d = insts[tl.inst];
        const int64_t i = d.p.frozen + 32 * (int64_t)(tl.warp0 + w) + (threadIdx.x & 31);
        if (i >= d.p.n) continue;
        const int64_t np = d.p.npad;
        double* const u_out = bs.cur ? d.u_alt : d.p.u;
        const double half_dt_m = __ddiv_rn(d.ep.half_dt, d.p.rho[i]);
        double u[3];
        for (int c = 0; c < 3; ++c) {
            const double v = __dadd_rn(d.p.v[c * np + i], __dmul_rn(half_dt_m, d.p.f[c * np + i]));
            d.p.v[c * np + i] = v;
            u[c] = __dadd_rn(d.p.u[c * np + i], __dmul_rn(d.ep.dt, v));
            u_out[c * np + i] = u[c];
        }
        if (d.body == kBatchMixed) {
            MixedU* const s_out = bs.cur ? d.u2_alt : const_cast<MixedU*>(d.mv.u2);
            s_out[i] = split_u(u[0], u[1], u[2], __dmul_rn(d.wscale, d.p.vol[i]), d.p.nofail[i]);
        }
    }
}

__global__ void k_batch_advance(int32_t* remaining, int32_t count, int32_t K)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < count) remaining[b] -= min(K, remaining[b]);
}

struct Candidate {
    int blocks_per_sm;
    int order;  // 0: tiles by instance, 1: interleaved across instances
    double throughput = 0.0;
};

}  // namespace

struct cpd_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cpd_system*> sys;
    std::vector<int64_t> bonds;
    std::vector<int32_t> remaining;   // host mirror, as of the chunks issued
    std::vector<char> released;       // instance handed back (cpd_batch_release)
    BatchInstance* d_inst = nullptr;
    int32_t* d_remaining = nullptr;
    // Tiles per body (fast, mixed) and order (by instance, interleaved).
    BatchTile* d_tiles[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int32_t ntiles[2] = {0, 0};
    bool lps[2] = {false, false};
    int sms = 0;
    int occupancy[2] = {1, 1};
    std::vector<Candidate> cands;
    int forced = -1, chosen = -1;
    size_t next_trial = 0;
    // Chunk being timed: candidate, work (bond-updates) and events.
    int timing_cand = -1;
    double timing_work = 0.0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, done = nullptr;
    std::map<std::pair<int, int>, std::pair<cudaGraphExec_t, int64_t>> graphs;
    int64_t launches = 0;
};

namespace {

cpd_status check_cuda(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return CPD_OK;
    return fail(e == cudaErrorMemoryAllocation ? CPD_ERR_OUT_OF_MEMORY : CPD_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
}
#define CPD_BATCH_CUDA(call)                                  \
    do {                                                      \
        cpd_status st_ = check_cuda((call), #call);           \
        if (st_ != CPD_OK) return st_;                        \
    } while (0)

// Tiles of the instances of one body, by instance or round-robin across them.
std::vector<BatchTile> make_tiles(const std::vector<std::vector<BatchTile>>& per, int order)
{
    std::vector<BatchTile> out;
    if (order == 0) {
        for (const auto& v : per) out.insert(out.end(), v.begin(), v.end());
        return out;
    }
    size_t most = 0;
    for (const auto& v : per) most = std::max(most, v.size());
    for (size_t k = 0; k < most; ++k)
        for (const auto& v : per)
            if (k < v.size()) out.push_back(v[k]);
    return out;
}

// Kernels of one chunk of K steps in launch shape c, issued on the batch
// stream (captured into a graph by the caller). Returns the launch count.
int issue_chunk(cpd_batch* b, int K, const Candidate& c)
{
    int n = 0;
    const int o = c.order;
    const int32_t tiles_all = b->ntiles[0] + b->ntiles[1];
    const int gv = std::max(1, std::min<int>(tiles_all, b->sms * 4));
    if (tiles_all > 0) {
        // First half step over both bodies' tiles (two launches share the kernel).
        for (int body = 0; body < 2; ++body) {
            if (b->ntiles[body] == 0) continue;
            k_batch_vv_initial<<<std::min<int>(gv, b->ntiles[body]), kBlock, 0, b->stream>>>(
                b->d_inst, b->d_remaining, b->d_tiles[body][o], b->ntiles[body], K);
            ++n;
        }
    }
    const int grid[2] = {std::min<int>(b->ntiles[0], std::min(c.blocks_per_sm, b->occupancy[0]) * b->sms),
                         std::min<int>(b->ntiles[1], std::min(c.blocks_per_sm, b->occupancy[1]) * b->sms)};
    for (int s = 0; s < K; ++s) {
        for (int pass = 0; pass < 2; ++pass) {
            if (b->ntiles[0] > 0 && (pass == 1 || b->lps[0]))
                n += launch_batch_fast(b->d_inst, b->d_remaining, b->d_tiles[0][o], b->ntiles[0],
                                       K, s, pass, grid[0], b->stream);
            if (b->ntiles[1] > 0 && (pass == 1 || b->lps[1]))
                n += launch_batch_mixed(b->d_inst, b->d_remaining, b->d_tiles[1][o],
                                        b->ntiles[1], K, s, pass, grid[1], b->stream);
        }
    }
    const int count = (int)b->sys.size();
    k_batch_advance<<<(count + 127) / 128, 128, 0, b->stream>>>(b->d_remaining, count, K);
    return n + 1;
}

cpd_status chunk_graph(cpd_batch* b, int K, int cand, cudaGraphExec_t* out, int64_t* nodes)
{
    auto it = b->graphs.find({K, cand});
    if (it != b->graphs.end()) {
        *out = it->second.first;
        *nodes = it->second.second;
        return CPD_OK;
    }
    cudaGraph_t g = nullptr;
    CPD_BATCH_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    const int n = issue_chunk(b, K, b->cands[cand]);
    const cudaError_t le = cudaGetLastError();
    const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return check_cuda(le != cudaSuccess ? le : ce, "batch chunk capture");
    }
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CPD_BATCH_CUDA(ie);
    b->graphs[{K, cand}] = {ex, (int64_t)n};
    *out = ex;
    *nodes = n;
    return CPD_OK;
}

// Reads the timed chunk, if any, into its candidate's throughput; picks
// the fastest once every candidate has been timed. Without `wait`, a timed
// chunk still running is left for a later call (*pending).
cpd_status harvest(cpd_batch* b, bool wait, bool* pending = nullptr)
{
    if (pending) *pending = false;
    if (b->timing_cand < 0) return CPD_OK;
    if (wait) {
        CPD_BATCH_CUDA(cudaEventSynchronize(b->ev1));
    } else {
        const cudaError_t q = cudaEventQuery(b->ev1);
        if (q == cudaErrorNotReady) {
            if (pending) *pending = true;
            return CPD_OK;
        }
        CPD_BATCH_CUDA(q);
    }
    float ms = 0.f;
    CPD_BATCH_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    Candidate& c = b->cands[b->timing_cand];
    if (ms > 0.f) c.throughput = b->timing_work / (1e-3 * ms);
    b->timing_cand = -1;
    if (b->chosen < 0 && b->next_trial >= b->cands.size()) {
        int best = 0;
        for (size_t k = 1; k < b->cands.size(); ++k)
            if (b->cands[k].throughput > b->cands[best].throughput) best = (int)k;
        b->chosen = best;
    }
    return CPD_OK;
}

void release(cpd_batch* b)
{
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.first);
    b->graphs.clear();
    if (b->stream) {
        // Stream-ordered frees: no device-wide synchronisation.
        if (b->d_inst) dev_free(b->d_inst, b->stream);
        if (b->d_remaining) dev_free(b->d_remaining, b->stream);
        for (auto& row : b->d_tiles)
            for (BatchTile*& t : row)
                if (t) dev_free(t, b->stream);
        cudaStreamSynchronize(b->stream);
    }
    for (cudaEvent_t e : {b->ev0, b->ev1, b->done})
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (size_t k = 0; k < b->sys.size(); ++k)
        if (!b->released[k]) batch_detach(b->sys[k]);
    b->sys.clear();
}

}  // namespace

extern "C" {

cpd_status cpd_batch_create(cpd_system* const* systems, int32_t count, const int32_t* steps,
                            cpd_batch** out)
{
    if (!out || !systems || !steps || count <= 0)
        return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_batch_create: need systems, steps and out");
    *out = nullptr;
    for (int32_t k = 0; k < count; ++k) {
        if (!systems[k]) return fail(CPD_ERR_INVALID_ARGUMENT, "null system in the batch");
        if (steps[k] < 0) return fail(CPD_ERR_INVALID_ARGUMENT, "negative step count");
        for (int32_t j = 0; j < k; ++j)
            if (systems[j] == systems[k])
                return fail(CPD_ERR_INVALID_ARGUMENT, "a system appears twice in the batch");
    }
    const int dev = system_device(systems[0]);
    for (int32_t k = 1; k < count; ++k)
        if (system_device(systems[k]) != dev)
            return fail(CPD_ERR_INVALID_ARGUMENT, "the systems of a batch share one device");
    CPD_BATCH_CUDA(cudaSetDevice(dev));
    auto* b = new cpd_batch();
    b->device = dev;
    std::vector<BatchInstance> inst(count);
    std::vector<std::vector<BatchTile>> per[2];
    cpd_status st = CPD_OK;
    for (int32_t k = 0; k < count && st == CPD_OK; ++k) {
        int64_t bonds = 0;
        st = batch_attach(systems[k], b, &inst[k], &bonds);
        if (st != CPD_OK) break;
        b->sys.push_back(systems[k]);
        b->released.push_back(0);
        b->bonds.push_back(bonds);
        b->remaining.push_back(steps[k]);
        const int body = inst[k].body;
        const int64_t warps = (system_rows(systems[k]) + 31) / 32;
        std::vector<BatchTile> tiles;
        for (int64_t w0 = 0; w0 < warps; w0 += kBatchTileWarps)
            tiles.push_back(BatchTile{k, (int32_t)w0,
                                      (int32_t)std::min<int64_t>(kBatchTileWarps, warps - w0),
                                      inst[k].pd == CPD_PD_LPS ? 1 : 0});
        if (inst[k].pd == CPD_PD_LPS) b->lps[body] = true;
        per[body].push_back(std::move(tiles));
    }
    auto bail = [&](cpd_status code) {
        const std::string msg = cpd_last_error();
        release(b);
        delete b;
        set_last_error(msg);
        return code;
    };
    if (st != CPD_OK) return bail(st);
    auto cuda_or_bail = [&](cudaError_t e, const char* what) {
        return e == cudaSuccess ? CPD_OK : bail(check_cuda(e, what));
    };
#define CPD_BATCH_TRY(call)                                           \
    do {                                                              \
        cpd_status t_ = cuda_or_bail((call), #call);                  \
        if (t_ != CPD_OK) return t_;                                  \
    } while (0)
    CPD_BATCH_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CPD_BATCH_TRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev));
    b->occupancy[0] = batch_fast_blocks_per_sm();
    b->occupancy[1] = batch_mixed_blocks_per_sm();
    CPD_BATCH_TRY(dev_alloc(&b->d_inst, sizeof(BatchInstance) * count, b->stream));
    CPD_BATCH_TRY(dev_alloc(&b->d_remaining, sizeof(int32_t) * count, b->stream));
    // The systems' set-up work (and the frozen-row copies of batch_attach)
    // completes before the batch's first chunk.
    for (cpd_system* s : b->sys) CPD_BATCH_TRY(cudaStreamSynchronize(system_stream(s)));
    CPD_BATCH_TRY(cudaMemcpyAsync(b->d_inst, inst.data(), sizeof(BatchInstance) * count,
                                  cudaMemcpyHostToDevice, b->stream));
    CPD_BATCH_TRY(cudaMemcpyAsync(b->d_remaining, steps, sizeof(int32_t) * count,
                                  cudaMemcpyHostToDevice, b->stream));
    std::vector<BatchTile> tiles[2][2];
    for (int body = 0; body < 2; ++body) {
        for (int order = 0; order < 2; ++order) {
            tiles[body][order] = make_tiles(per[body], order);
            const std::vector<BatchTile>& t = tiles[body][order];
            b->ntiles[body] = (int32_t)t.size();
            if (t.empty()) continue;
            CPD_BATCH_TRY(dev_alloc(&b->d_tiles[body][order], sizeof(BatchTile) * t.size(),
                                    b->stream));
            CPD_BATCH_TRY(cudaMemcpyAsync(b->d_tiles[body][order], t.data(),
                                          sizeof(BatchTile) * t.size(), cudaMemcpyHostToDevice,
                                          b->stream));
        }
    }
    // The host arrays above are read by the copies: wait for them.
    CPD_BATCH_TRY(cudaStreamSynchronize(b->stream));
    const int occ = std::max(b->occupancy[0], b->occupancy[1]);
    std::vector<int> grids = {1, 2};
    if (occ > 2) grids.push_back(occ);
    for (int g : grids)
        for (int order = 0; order < 2; ++order) b->cands.push_back(Candidate{g, order});
    CPD_BATCH_TRY(cudaEventCreate(&b->ev0));
    CPD_BATCH_TRY(cudaEventCreate(&b->ev1));
    CPD_BATCH_TRY(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
#undef CPD_BATCH_TRY
    *out = b;
    return CPD_OK;
}

cpd_status cpd_batch_destroy(cpd_batch* b)
{
    if (!b) return CPD_OK;
    cudaSetDevice(b->device);
    release(b);
    delete b;
    return CPD_OK;
}

cpd_status cpd_batch_step(cpd_batch* b, int32_t K)
{
    if (!b) return fail(CPD_ERR_INVALID_ARGUMENT, "null batch");
    if (K <= 0) return fail(CPD_ERR_INVALID_ARGUMENT, "chunk_steps must be positive");
    CPD_BATCH_CUDA(cudaSetDevice(b->device));
    double work = 0.0;
    for (size_t k = 0; k < b->sys.size(); ++k)
        work += (double)b->bonds[k] * std::min(K, b->remaining[k]);
    if (work == 0.0 && std::all_of(b->remaining.begin(), b->remaining.end(),
                                   [](int32_t r) { return r == 0; }))
        return CPD_OK;
    // The tuner never blocks the caller: while a timed chunk runs, further
    // chunks take the same candidate untimed.
    bool pending = false;
    if (cpd_status st = harvest(b, false, &pending); st != CPD_OK) return st;
    int cand = b->forced;
    bool timed = false;
    if (cand < 0) {
        if (b->chosen >= 0) {
            cand = b->chosen;
        } else if (pending) {
            cand = b->timing_cand;
        } else {
            cand = (int)b->next_trial++;
            timed = true;
        }
    }
    cudaGraphExec_t g = nullptr;
    int64_t nodes = 0;
    if (cpd_status st = chunk_graph(b, K, cand, &g, &nodes); st != CPD_OK) return st;
    // Work queued on the systems' own streams (reads, snapshots) comes first.
    for (size_t k = 0; k < b->sys.size(); ++k) {
        if (b->released[k]) continue;
        CPD_BATCH_CUDA(cudaEventRecord(b->done, system_stream(b->sys[k])));
        CPD_BATCH_CUDA(cudaStreamWaitEvent(b->stream, b->done, 0));
    }
    if (timed) CPD_BATCH_CUDA(cudaEventRecord(b->ev0, b->stream));
    CPD_BATCH_CUDA(cudaGraphLaunch(g, b->stream));
    if (timed) {
        CPD_BATCH_CUDA(cudaEventRecord(b->ev1, b->stream));
        b->timing_cand = cand;
        b->timing_work = work;
    }
    b->launches += nodes;
    // Later work on the systems' streams waits for this chunk.
    CPD_BATCH_CUDA(cudaEventRecord(b->done, b->stream));
    for (size_t k = 0; k < b->sys.size(); ++k)
        if (!b->released[k])
            CPD_BATCH_CUDA(cudaStreamWaitEvent(system_stream(b->sys[k]), b->done, 0));
    for (auto& r : b->remaining) r -= std::min(K, r);
    return CPD_OK;
}

cpd_status cpd_batch_release(cpd_batch* b, int32_t instance)
{
    if (!b || instance < 0 || instance >= (int32_t)b->sys.size())
        return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_batch_release: bad batch or instance");
    if (b->released[instance]) return CPD_OK;
    if (b->remaining[instance] != 0)
        return fail(CPD_ERR_STATE, "cpd_batch_release: the instance still has steps to take");
    // The system's stream already waits for the chunk that finished the
    // instance, and later chunks skip it (no steps left), so it is free now.
    b->released[instance] = 1;
    batch_detach(b->sys[instance]);
    return CPD_OK;
}

cpd_status cpd_batch_remaining(const cpd_batch* b, int32_t instance, int32_t* steps)
{
    if (!b || !steps || instance < 0 || instance >= (int32_t)b->remaining.size())
        return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_batch_remaining: bad batch or instance");
    *steps = b->remaining[instance];
    return CPD_OK;
}

cpd_status cpd_batch_synchronize(cpd_batch* b)
{
    if (!b) return fail(CPD_ERR_INVALID_ARGUMENT, "null batch");
    CPD_BATCH_CUDA(cudaSetDevice(b->device));
    CPD_BATCH_CUDA(cudaStreamSynchronize(b->stream));
    return harvest(b, true);
}

cpd_status cpd_batch_set_candidate(cpd_batch* b, int32_t candidate)
{
    if (!b) return fail(CPD_ERR_INVALID_ARGUMENT, "null batch");
    if (candidate < -1 || candidate >= (int32_t)b->cands.size())
        return fail(CPD_ERR_INVALID_ARGUMENT, "no such launch-shape candidate");
    b->forced = candidate;
    return CPD_OK;
}

cpd_status cpd_batch_tuning(const cpd_batch* b, int32_t* count, int32_t* chosen,
                            int32_t* blocks_per_sm, int32_t* order, double* throughput)
{
    if (!b || !count) return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_batch_tuning: null argument");
    *count = (int32_t)b->cands.size();
    if (chosen) *chosen = b->forced >= 0 ? b->forced : b->chosen;
    for (size_t k = 0; k < b->cands.size(); ++k) {
        if (blocks_per_sm) blocks_per_sm[k] = b->cands[k].blocks_per_sm;
        if (order) order[k] = b->cands[k].order;
        if (throughput) throughput[k] = b->cands[k].throughput;
    }
    return CPD_OK;
}

int64_t cpd_batch_launches(const cpd_batch* b) { return b ? b->launches : 0; }

}  // extern "C"

namespace cpd {
cudaStream_t batch_stream(const cpd_batch* b) { return b->stream; }
}  // namespace cpd
