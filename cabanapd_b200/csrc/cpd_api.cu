// C ABI of the cabanapd_b200 library: system lifetime, host<->device
// transfers and the Solver orchestration of the per-timestep hot path
// (CabanaPD_Solver.hpp:229-477), issued asynchronously on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <utility>
#include <unordered_map>
#include <vector>

#include "cpd_internal.cuh"

using namespace cpd;

namespace {
constexpr int kPoolDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pool[kPoolDevices] = {};
int g_live_systems[kPoolDevices] = {};

cudaError_t device_pool(int dev, cudaMemPool_t* out)
{
    if (dev < 0 || dev >= kPoolDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaError_t e = cudaMemPoolCreate(&g_pool[dev], &props);
        if (e != cudaSuccess) {
            g_pool[dev] = nullptr;
            return e;
        }
        // Keep freed blocks for the next system instead of returning them
        // at every synchronisation; trimmed when no system is live.
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(g_pool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

void system_opened(int dev)
{
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    g_live_systems[dev]++;
}

// Device memory the pool keeps mapped once no system is live, so that the
// next system (a job after a job) does not map its memory again: one eighth
// of the device, at most 32 GiB, or CPD_POOL_KEEP_BYTES.
size_t pool_keep_bytes()
{
    const char* e = getenv("CPD_POOL_KEEP_BYTES");
    if (e) return (size_t)strtoull(e, nullptr, 10);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    return std::min(total_b / 8, (size_t)32 << 30);
}

// Called after the closing system's frees have completed.
void system_closed(int dev)
{
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (--g_live_systems[dev] == 0 && g_pool[dev]) cudaMemPoolTrimTo(g_pool[dev], pool_keep_bytes());
}

thread_local std::string g_last_error;

cpd_status set_error(cpd_status code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}
}  // namespace

namespace cpd {

cudaError_t dev_alloc(void** ptr, size_t bytes, cudaStream_t st)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = nullptr;
    e = device_pool(dev, &pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(ptr, bytes > 0 ? bytes : 16, pool, st);
}

cudaError_t dev_free(void* ptr, cudaStream_t st) { return cudaFreeAsync(ptr, st); }

void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace cpd

#define CPD_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess)                                                      \
            return set_error(e_ == cudaErrorMemoryAllocation ? CPD_ERR_OUT_OF_MEMORY \
                                                             : CPD_ERR_CUDA,        \
                             std::string(#call) + ": " + cudaGetErrorString(e_));   \
    } while (0)

#define CPD_LAUNCHED(count_expr)                                                    \
    do {                                                                            \
        s->launches += (count_expr);                                                \
        cudaError_t e_ = cudaGetLastError();                                        \
        if (e_ != cudaSuccess)                                                      \
            return set_error(CPD_ERR_CUDA, std::string("kernel launch: ") +         \
                                               cudaGetErrorString(e_));             \
    } while (0)

#define CPD_OK_OR_RETURN(expr)                                                      \
    do {                                                                            \
        cpd_status s_ = (expr);                                                     \
        if (s_ != CPD_OK) return s_;                                                \
    } while (0)

#define CPD_NOT_IN_BATCH(sys)                                                       \
    do {                                                                            \
        if ((sys) && (sys)->batch)                                                  \
            return set_error(CPD_ERR_STATE, "the system belongs to a batch "        \
                                            "(cpd_batch_destroy releases it)");     \
    } while (0)

struct cpd_system {
    cpd_params params{};
    Model md;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int64_t n = 0, frozen = 0, npad = 0;
    // Particle fields (component-major SoA, [3][npad] or [npad]).
    double *x = nullptr, *u = nullptr, *v = nullptr, *f = nullptr;
    double *vol = nullptr, *rho = nullptr, *m = nullptr, *theta = nullptr;
    double *lps_a = nullptr, *lps_b = nullptr, *W = nullptr, *phi = nullptr;
    double *radius = nullptr, *u_neigh = nullptr;
    uint8_t* nofail = nullptr;
    int32_t* perm = nullptr;  // internal -> caller index; nullptr = identity
    std::vector<int32_t> h_inv;  // caller -> internal
    double* staging = nullptr;   // [3 n] transfer buffer
    double* stress = nullptr;    // [9][npad] per-particle stress (cpd_compute_stress)
    double* stress_staging = nullptr;  // [9 n] its transfer buffer
    double* red = nullptr;       // reduction partials
    int red_cap = 0;
    double* red_out = nullptr;   // small result slots
    double* h_red = nullptr;     // pinned host mirror of red_out
    NeighborList pd, contact;
    MixedState mixed;  // CPD_MIXED: FP32 split copies and bond stencil codes
    std::vector<BoundaryCondition> bcs;
    // Host copy of the boundary conditions (internal indices), and the
    // per-row program the fused step applies (built on first use).
    struct HostBC {
        int kind, component;
        std::vector<int32_t> idx;
        std::vector<double> values;
    };
    std::vector<HostBC> hbcs;
    int bc_prog = 0;  // 0 not built, 1 built, -1 the conditions cannot be fused
    uint32_t* bc_bits = nullptr;
    int32_t* bc_row = nullptr;
    uint8_t* bc_keep = nullptr;
    double* bc_add = nullptr;
    int32_t nbc = 0;
    // Second displacement buffers of the fused step.
    double* u_alt = nullptr;
    double* v_alt = nullptr;  // contact-only fused step: second velocity buffer
    MixedU* u2_alt = nullptr;
    MixedU* u2_alt_base = nullptr;  // allocation: u2_alt with the split's guard records
    bool neighbors_built = false;
    bool initialized = false;
    // CPD_MIXED PMB whose lattice table is past the byte codes (over 253
    // entries: a horizon of four spacings): the FP64 stencil kernels run it.
    bool mixed_via_fp64 = false;
    // The batch that advances this system (cpd_batch_create); while set,
    // calls that change the system's state are refused.
    const void* batch = nullptr;
    bool stress_ready = false;  // cpd_compute_stress ran since the particles were set
    double max_disp = 0.0;
    int64_t steps_since_rebuild = 0;
    int64_t rebuilds = 0;
    int64_t launches = 0;
    // Kernel timing.
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    std::vector<cudaEvent_t> event_pool;
    double timed_ms = 0.0;
    int64_t timed_launches = 0;
};

namespace {

bool has_pd(const cpd_system* s) { return s->md.pd != CPD_PD_NONE; }
bool is_lps(const cpd_system* s)
{
    return s->md.pd == CPD_PD_LPS;
}
bool has_contact(const cpd_system* s) { return s->md.contact != CPD_CONTACT_NONE; }

ParticleView view(const cpd_system* s)
{
    ParticleView p;
    p.n = s->n;
    p.frozen = s->frozen;
    p.npad = s->npad;
    p.x = s->x;
    p.u = s->u;
    p.v = s->v;
    p.f = s->f;
    p.vol = s->vol;
    p.rho = s->rho;
    p.nofail = s->nofail;
    p.m = s->m;
    p.theta = s->theta;
    p.lps_a = s->lps_a;
    p.lps_b = s->lps_b;
    p.W = s->W;
    p.phi = s->phi;
    p.radius = s->radius;
    p.u_neigh = s->u_neigh;
    return p;
}

EllView pd_view(const cpd_system* s)
{
    EllView v = s->pd.view();
    if (!s->md.fracture) v.mu = nullptr;
    return v;
}

void free_bc_program(cpd_system* s)
{
    void* arrays[] = {s->bc_bits, s->bc_row, s->bc_keep, s->bc_add};
    for (void* a : arrays)
        if (a) dev_free(a, s->stream);
    s->bc_bits = nullptr;
    s->bc_row = nullptr;
    s->bc_keep = nullptr;
    s->bc_add = nullptr;
    s->nbc = 0;
    s->bc_prog = 0;
}

void free_particles(cpd_system* s)
{
    double** arrays[] = {&s->x,     &s->u,     &s->v,     &s->f,     &s->vol,
                         &s->rho,   &s->m,     &s->theta, &s->lps_a, &s->lps_b,
                         &s->W,     &s->phi,   &s->radius, &s->u_neigh, &s->staging,
                         &s->red,   &s->red_out, &s->stress, &s->stress_staging};
    for (double** a : arrays)
        if (*a) {
            dev_free(*a, s->stream);
            *a = nullptr;
        }
    if (s->nofail) dev_free(s->nofail, s->stream);
    s->nofail = nullptr;
    s->stress_ready = false;
    if (s->perm) dev_free(s->perm, s->stream);
    s->perm = nullptr;
    for (auto& bc : s->bcs) {
        if (bc.idx) dev_free(bc.idx, s->stream);
        if (bc.values) dev_free(bc.values, s->stream);
    }
    s->bcs.clear();
    s->hbcs.clear();
    free_bc_program(s);
    if (s->u_alt) dev_free(s->u_alt, s->stream);
    s->u_alt = nullptr;
    if (s->v_alt) dev_free(s->v_alt, s->stream);
    s->v_alt = nullptr;
    if (s->u2_alt_base) dev_free(s->u2_alt_base, s->stream);
    s->u2_alt = s->u2_alt_base = nullptr;
    free_neighbor_list(s->pd, s->stream);
    free_neighbor_list(s->contact, s->stream);
    free_mixed(s->mixed, s->stream);
    s->n = s->npad = s->frozen = 0;
    s->red_cap = 0;
    s->neighbors_built = false;
    s->initialized = false;
}

cudaEvent_t take_event(cpd_system* s)
{
    if (!s->event_pool.empty()) {
        cudaEvent_t e = s->event_pool.back();
        s->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

cpd_status harvest_timing(cpd_system* s)
{
    for (auto& pr : s->pending) {
        CPD_CUDA(cudaEventSynchronize(pr.second));
        float ms = 0.f;
        CPD_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
        s->timed_ms += ms;
        s->timed_launches++;
        s->event_pool.push_back(pr.first);
        s->event_pool.push_back(pr.second);
    }
    s->pending.clear();
    return CPD_OK;
}

// Morton code of the particle's cell (21 bits per axis).
uint64_t spread3(uint64_t v)
{
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

std::vector<int32_t> morton_order(const double* x, int64_t n, int64_t frozen, double cell)
{
    double lo[3] = {x[0], x[1], x[2]};
    for (int64_t p = 0; p < n; p++)
        for (int d = 0; d < 3; d++) lo[d] = std::min(lo[d], x[3 * p + d]);
    std::vector<uint64_t> code(n);
    for (int64_t p = 0; p < n; p++) {
        uint64_t c[3];
        for (int d = 0; d < 3; d++) c[d] = (uint64_t)std::floor((x[3 * p + d] - lo[d]) / cell);
        code[p] = spread3(c[0]) | spread3(c[1]) << 1 | spread3(c[2]) << 2;
    }
    std::vector<int32_t> order(n);
    std::iota(order.begin(), order.end(), 0);
    auto cmp = [&](int32_t a, int32_t b) { return code[a] < code[b]; };
    // Frozen particles stay in front (they are never integrated).
    std::stable_sort(order.begin(), order.begin() + frozen, cmp);
    std::stable_sort(order.begin() + frozen, order.end(), cmp);
    return order;
}

cpd_status upload_vector(cpd_system* s, const double* host, double* dst)
{
    CPD_CUDA(cudaMemcpyAsync(s->staging, host, sizeof(double) * 3 * s->n,
                             cudaMemcpyHostToDevice, s->stream));
    s->launches += launch_aos_to_soa(s->staging, dst, s->n, s->npad, 3, s->perm, s->stream);
    CPD_CUDA(cudaGetLastError());
    return CPD_OK;
}

cpd_status upload_scalar(cpd_system* s, const double* host, double* dst)
{
    CPD_CUDA(cudaMemcpyAsync(s->staging, host, sizeof(double) * s->n,
                             cudaMemcpyHostToDevice, s->stream));
    s->launches += launch_aos_to_soa(s->staging, dst, s->n, s->npad, 1, s->perm, s->stream);
    CPD_CUDA(cudaGetLastError());
    return CPD_OK;
}

cpd_status ensure_reduction(cpd_system* s, int blocks)
{
    if (blocks * 2 <= s->red_cap) return CPD_OK;
    if (s->red) CPD_CUDA(dev_free(s->red, s->stream));
    s->red = nullptr;
    CPD_CUDA(dev_alloc(&s->red, sizeof(double) * 2 * blocks, s->stream));
    s->red_cap = 2 * blocks;
    return CPD_OK;
}

// disp: the current displacement (the system's u unless a fused step holds
// it in its second buffer).
cpd_status rebuild_contact(cpd_system* s, double cutoff, const double* disp = nullptr)
{
    if (!disp) disp = s->u;
    std::string err;
    int l = build_neighbor_list(s->x, disp, s->n, s->npad, s->frozen, cutoff, s->perm,
                                false, s->contact, s->stream, err);
    if (l < 0) return set_error(CPD_ERR_CUDA, "contact neighbour build: " + err);
    s->launches += l;
    // CabanaPD_Neighbor.hpp:127-130: displacement at the last build.
    CPD_CUDA(cudaMemcpyAsync(s->u_neigh, disp, sizeof(double) * 3 * s->npad,
                             cudaMemcpyDeviceToDevice, s->stream));
    s->rebuilds++;
    s->steps_since_rebuild = 0;
    return CPD_OK;
}

// CabanaPD_Neighbor.hpp:107-132 Neighbor::update, or every rebuild_every steps.
cpd_status contact_update(cpd_system* s)
{
    bool rebuild;
    if (s->params.rebuild_every > 0) {
        rebuild = s->steps_since_rebuild >= s->params.rebuild_every;
    } else {
        CPD_CUDA(cudaMemcpyAsync(s->h_red, s->red_out, sizeof(double), cudaMemcpyDeviceToHost,
                                 s->stream));
        CPD_CUDA(cudaStreamSynchronize(s->stream));
        s->max_disp = s->h_red[0];
        rebuild = s->max_disp > s->md.radius_extend;
    }
    if (rebuild) return rebuild_contact(s, 2.0 * s->md.radius + s->md.radius_extend);
    return CPD_OK;
}

cpd_status timed_begin(cpd_system* s, cudaEvent_t& e0)
{
    e0 = nullptr;
    if (!s->timing) return CPD_OK;
    e0 = take_event(s);
    CPD_CUDA(cudaEventRecord(e0, s->stream));
    return CPD_OK;
}

cpd_status timed_end(cpd_system* s, cudaEvent_t e0)
{
    if (!e0) return CPD_OK;
    cudaEvent_t e1 = take_event(s);
    CPD_CUDA(cudaEventRecord(e1, s->stream));
    s->pending.emplace_back(e0, e1);
    if (s->pending.size() > 4096) return harvest_timing(s);
    return CPD_OK;
}

// CPD_MIXED set-up applies to PMB and LPS without contact; the LPS kernels
// then need every row to be a stencil row (mixed.lps_ok), else LPS keeps the
// FP64 kernels.
bool wants_mixed(const cpd_system* s)
{
    return s->params.precision == CPD_MIXED && s->md.contact == CPD_CONTACT_NONE &&
           (s->md.pd == CPD_PD_PMB || s->md.pd == CPD_PD_LPS) && !s->mixed_via_fp64;
}

bool use_mixed(const cpd_system* s)
{
    return wants_mixed(s) && (s->md.pd == CPD_PD_PMB || s->mixed.lps_ok);
}

// CPD_FP64 PMB without contact on a lattice: the stencil kernel takes the
// stencil rows (set up with the neighbour list when wants_stencil64). LPS
// keeps the FP64 throughput kernels: its dilatation and force sum strongly
// cancelling bond terms, which would turn the lattice offsets' departure
// from the positions' rounded differences (~1e-14) into errors above 1e-12.
bool wants_stencil64(const cpd_system* s)
{
    return (s->params.precision == CPD_FP64 || s->mixed_via_fp64) &&
           s->md.contact == CPD_CONTACT_NONE && s->md.pd == CPD_PD_PMB;
}

bool use_stencil64(const cpd_system* s)
{
    return wants_stencil64(s) && stencil64_ready(s->mixed);
}

// The throughput FP64 kernels serve CPD_FP64, and CPD_MIXED where the mixed
// kernels do not apply.
bool use_fast(const cpd_system* s)
{
    return (s->params.precision == CPD_FP64 ||
            (s->params.precision == CPD_MIXED && !use_mixed(s))) &&
           fast_supported(s->md);
}

// The bond kernel on particle view p (displacement buffer p.u; on the
// mixed path its split in m.u2), finishing each row as ep says.
cpd_status pd_force_on(cpd_system* s, const ParticleView& p, const MixedState& m,
                       const StepEpilogue& ep)
{
    cudaEvent_t e0;
    CPD_OK_OR_RETURN(timed_begin(s, e0));
    if (use_mixed(s)) {
        CPD_LAUNCHED(launch_pd_force_mixed(p, pd_view(s), s->md, m, ep, s->stream));
    } else if (use_stencil64(s)) {
        // Outside the fused step the gather records follow p.u here.
        if (ep.mode == 0)
            CPD_LAUNCHED(launch_pack_u4(p, p.u, 0, p.n, m.u4, s->stream, m.gcell));
        CPD_LAUNCHED(launch_pd_force_stencil64(p, pd_view(s), s->md, m, ep, s->stream));
    } else if (use_fast(s))
        CPD_LAUNCHED(launch_pd_force_fast(p, pd_view(s), s->md, ep, s->stream));
    else
        CPD_LAUNCHED(launch_pd_force(p, pd_view(s), s->md, s->stream));
    return timed_end(s, e0);
}

cpd_status pd_force(cpd_system* s) { return pd_force_on(s, view(s), s->mixed, StepEpilogue{}); }

// LPS weighted volume (when compute_m) and dilatation; on the mixed path m
// carries the displacement split of p.u.
cpd_status lps_prepare_on(cpd_system* s, const ParticleView& p, const MixedState& m,
                          bool compute_m)
{
    if (use_mixed(s)) {
        CPD_LAUNCHED(launch_lps_mtheta_mixed(p, pd_view(s), s->md, m, compute_m, s->stream));
        return CPD_OK;
    }
    if (use_fast(s)) {
        CPD_LAUNCHED(launch_lps_m_theta_fast(p, pd_view(s), s->md, compute_m, s->stream));
        return CPD_OK;
    }
    if (compute_m) CPD_LAUNCHED(launch_lps_weighted_volume(p, pd_view(s), s->md, s->stream));
    CPD_LAUNCHED(launch_lps_dilatation(p, pd_view(s), s->md, s->stream));
    return CPD_OK;
}

cpd_status lps_prepare(cpd_system* s, bool compute_m)
{
    return lps_prepare_on(s, view(s), s->mixed, compute_m);
}

cpd_status contact_force(cpd_system* s, bool reset)
{
    const ParticleView p = view(s);
    cudaEvent_t e0 = nullptr;
    if (!has_pd(s)) CPD_OK_OR_RETURN(timed_begin(s, e0));
    if (s->md.contact == CPD_CONTACT_NORMAL_REPULSION)
        CPD_LAUNCHED(launch_repulsion_force(p, s->contact.view(), s->md, reset, s->stream));
    else if (s->params.precision == CPD_MIXED)
        CPD_LAUNCHED(launch_hertz_force_mixed(p, s->contact.view(), s->md, reset, s->stream));
    else
        CPD_LAUNCHED(launch_hertz_force(p, s->contact.view(), s->md, reset, s->stream));
    return timed_end(s, e0);
}

cpd_status apply_force_bcs(cpd_system* s)
{
    const ParticleView p = view(s);
    for (const auto& bc : s->bcs) CPD_LAUNCHED(launch_force_bc(p, bc, s->stream));
    return CPD_OK;
}

// CabanaPD_Solver.hpp:462-477 updateForce, then the contact force.
cpd_status update_force(cpd_system* s)
{
    if (has_pd(s)) {
        if (is_lps(s)) CPD_OK_OR_RETURN(lps_prepare(s, s->md.fracture != 0));
        CPD_OK_OR_RETURN(pd_force(s));
    }
    if (has_contact(s)) {
        CPD_OK_OR_RETURN(contact_update(s));
        CPD_OK_OR_RETURN(contact_force(s, !has_pd(s)));
    }
    return CPD_OK;
}

cpd_status vv_initial(cpd_system* s)
{
    const ParticleView p = view(s);
    const bool track = has_contact(s);
    const int nb = vv_blocks(s->n - s->frozen);
    if (track) CPD_OK_OR_RETURN(ensure_reduction(s, nb));
    if (use_mixed(s))
        CPD_LAUNCHED(launch_vv_initial_mixed(p, s->md, s->params.dt, s->u, s->mixed.u2,
                                             s->stream));
    else
        CPD_LAUNCHED(launch_vv_initial(p, s->params.dt, track, s->red, nb, s->u, s->stream));
    if (track && s->n > s->frozen)
        CPD_LAUNCHED(launch_max_partials(s->red, nb, s->red_out, s->stream));
    s->steps_since_rebuild++;
    return CPD_OK;
}

// The boundary conditions as one program per row (see StepEpilogue):
// possible when every row and component is touched by at most one
// operation and no condition acts on a frozen particle; the program then
// applies exactly the operations of the separate kernel.
cpd_status build_bc_program(cpd_system* s)
{
    struct Row {
        uint8_t keep = 0;  // bits 0-2 keep f, bits 4-6 component touched
        double add[3] = {0.0, 0.0, 0.0};
    };
    std::vector<std::pair<int32_t, Row>> rows;
    size_t listed = 0;
    for (const auto& bc : s->hbcs) listed += bc.idx.size();
    std::unordered_map<int32_t, int32_t> where;  // row -> its entry in rows
    where.reserve(listed);
    bool ok = true;
    for (const auto& bc : s->hbcs) {
        for (size_t b = 0; b < bc.idx.size() && ok; ++b) {
            const int32_t q = bc.idx[b];
            if (q < s->frozen) {
                ok = false;
                break;
            }
            const auto ins = where.emplace(q, (int32_t)rows.size());
            if (ins.second) rows.push_back({q, Row{}});
            Row& r = rows[ins.first->second].second;
            for (int d = 0; d < 3; ++d) {
                const bool touched = bc.kind != CPD_BC_FORCE_ADD || d == bc.component;
                if (!touched) continue;
                if (r.keep & (16u << d)) {
                    ok = false;
                    break;
                }
                r.keep |= (uint8_t)(16u << d);
                if (bc.kind == CPD_BC_FORCE_VALUE) {
                    r.add[d] = bc.values[0];
                } else {
                    r.keep |= (uint8_t)(1u << d);
                    r.add[d] = bc.kind == CPD_BC_FORCE_UPDATE ? bc.values[0] : bc.values[b];
                }
            }
        }
        if (!ok) break;
    }
    if (!ok) {
        s->bc_prog = -1;
        return CPD_OK;
    }
    std::sort(rows.begin(), rows.end(),
              [](const std::pair<int32_t, Row>& a, const std::pair<int32_t, Row>& b) {
                  return a.first < b.first;
              });
    const int32_t m = (int32_t)rows.size();
    s->nbc = m;
    if (m > 0) {
        const size_t nwords = (size_t)(s->npad + 31) / 32;
        std::vector<uint32_t> bits(nwords, 0u);
        std::vector<int32_t> row(m);
        std::vector<uint8_t> keep(m);
        std::vector<double> add(3 * (size_t)m);
        for (int32_t k = 0; k < m; ++k) {
            const int32_t q = rows[k].first;
            bits[q >> 5] |= 1u << (q & 31);
            row[k] = q;
            keep[k] = rows[k].second.keep;
            for (int d = 0; d < 3; ++d) add[(size_t)d * m + k] = rows[k].second.add[d];
        }
        CPD_CUDA(dev_alloc(&s->bc_bits, sizeof(uint32_t) * nwords, s->stream));
        CPD_CUDA(dev_alloc(&s->bc_row, sizeof(int32_t) * m, s->stream));
        CPD_CUDA(dev_alloc(&s->bc_keep, m, s->stream));
        CPD_CUDA(dev_alloc(&s->bc_add, sizeof(double) * 3 * m, s->stream));
        CPD_CUDA(cudaMemcpyAsync(s->bc_bits, bits.data(), sizeof(uint32_t) * nwords,
                                 cudaMemcpyHostToDevice, s->stream));
        CPD_CUDA(cudaMemcpyAsync(s->bc_row, row.data(), sizeof(int32_t) * m,
                                 cudaMemcpyHostToDevice, s->stream));
        CPD_CUDA(cudaMemcpyAsync(s->bc_keep, keep.data(), m, cudaMemcpyHostToDevice, s->stream));
        CPD_CUDA(cudaMemcpyAsync(s->bc_add, add.data(), sizeof(double) * 3 * m,
                                 cudaMemcpyHostToDevice, s->stream));
        CPD_CUDA(cudaStreamSynchronize(s->stream));
    }
    s->bc_prog = 1;
    return CPD_OK;
}

// Whether cpd_step may run the fused step: PD without contact on the
// throughput kernels, with boundary conditions a row program can express.
// CPD_FUSED_STEP=0 selects the separate kernels (for comparisons).
bool fused_steps_enabled()
{
    static const bool on = [] {
        const char* e = getenv("CPD_FUSED_STEP");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Contact alone with a fixed rebuild interval: the host knows when the list
// is rebuilt, so the steps between rebuilds need no read-back.
bool contact_fusable(const cpd_system* s)
{
    return !has_pd(s) && has_contact(s) && s->params.rebuild_every > 0;
}

bool fusable_kind(const cpd_system* s)
{
    return (has_pd(s) && !has_contact(s) && (use_fast(s) || use_mixed(s))) ||
           contact_fusable(s);
}

// Builds what the fused step needs (second displacement buffers, the row
// program of the boundary conditions); allocates and synchronises, so it
// runs at init or when the conditions change, never inside a step.
cpd_status prepare_fused(cpd_system* s)
{
    if (!fusable_kind(s) || !fused_steps_enabled()) return CPD_OK;
    if (s->bc_prog == 0) CPD_OK_OR_RETURN(build_bc_program(s));
    if (s->bc_prog != 1) return CPD_OK;
    if (!s->u_alt) CPD_CUDA(dev_alloc(&s->u_alt, sizeof(double) * 3 * s->npad, s->stream));
    if (contact_fusable(s) && !s->v_alt)
        CPD_CUDA(dev_alloc(&s->v_alt, sizeof(double) * 3 * s->npad, s->stream));
    if (use_mixed(s) && !s->u2_alt) {
        const size_t recs = (size_t)(s->npad + 2 * s->mixed.guard);
        CPD_CUDA(dev_alloc(&s->u2_alt_base, sizeof(MixedU) * recs, s->stream));
        CPD_CUDA(cudaMemsetAsync(s->u2_alt_base, 0, sizeof(MixedU) * recs, s->stream));
        s->u2_alt = s->u2_alt_base + s->mixed.guard;
    }
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

// Whether cpd_step runs the fused step now (everything prepared).
bool fused_ready(const cpd_system* s)
{
    return fused_steps_enabled() && fusable_kind(s) && s->bc_prog == 1 && s->u_alt &&
           (!use_mixed(s) || s->u2_alt) && (!contact_fusable(s) || s->v_alt);
}

// Whether the last step of cpd_step_energy forms the energy itself: the
// PMB stencil kernels with one particle volume (mixed: beside any warps on
// the general kernels; FP64: when the stencil kernel holds every row).
bool fused_energy_ok(const cpd_system* s)
{
    const MixedState& m = s->mixed;
    if (s->md.pd != CPD_PD_PMB || !m.vol_sums || m.nstencil <= 0) return false;
    if (use_mixed(s)) return m.st32 && m.u2;
    return use_stencil64(s) && (m.st64 || m.st64w) && m.nirregular == 0;
}

// num_steps steps as: first half step, then one bond kernel per step whose
// epilogue applies the boundary conditions, the second half step and (but
// for the last step) the next first half step, alternating displacement
// buffers. The first half step writes to the buffer that makes the last
// step end in the system's own arrays.
// Contact alone (fixed rebuild interval): first half step, then per step the
// list rebuild when due (on the current displacement) and one contact kernel
// whose epilogue applies the boundary conditions, the second half step and
// the next first half step. Neighbours read velocities (damping) as well as
// displacements, so both alternate between two buffers; the velocity ends in
// the system's array (copied back after an odd number of steps).
cpd_status step_fused_contact(cpd_system* s, int32_t num_steps)
{
    const bool start_alt = ((num_steps - 1) & 1) != 0;
    double* ucur = start_alt ? s->u_alt : s->u;
    double* unxt = start_alt ? s->u : s->u_alt;
    double* vcur = s->v;
    double* vnxt = s->v_alt;
    const size_t vec = sizeof(double) * 3 * (size_t)s->npad;
    if (s->frozen > 0) {
        const size_t bytes = sizeof(double) * (size_t)s->frozen;
        for (int d = 0; d < 3; ++d) {
            CPD_CUDA(cudaMemcpyAsync(s->u_alt + (size_t)d * s->npad, s->u + (size_t)d * s->npad,
                                     bytes, cudaMemcpyDeviceToDevice, s->stream));
            CPD_CUDA(cudaMemcpyAsync(s->v_alt + (size_t)d * s->npad, s->v + (size_t)d * s->npad,
                                     bytes, cudaMemcpyDeviceToDevice, s->stream));
        }
    }
    const ParticleView p = view(s);
    CPD_LAUNCHED(launch_vv_initial(p, s->params.dt, false, nullptr, 0, ucur, s->stream));
    StepEpilogue ep;
    ep.dt = s->params.dt;
    ep.half_dt = 0.5 * s->params.dt;
    ep.bc_bits = s->bc_bits;
    ep.bc_row = s->bc_row;
    ep.bc_keep = s->bc_keep;
    ep.bc_add = s->bc_add;
    ep.nbc = s->nbc;
    for (int32_t k = 0; k < num_steps; ++k) {
        s->steps_since_rebuild++;
        // CabanaPD_Neighbor.hpp:107-132, every rebuild_every steps.
        if (s->steps_since_rebuild >= s->params.rebuild_every)
            CPD_OK_OR_RETURN(rebuild_contact(s, 2.0 * s->md.radius + s->md.radius_extend, ucur));
        ParticleView pk = p;
        pk.u = ucur;
        pk.v = vcur;
        ep.mode = k + 1 < num_steps ? 2 : 1;
        ep.u_next = unxt;
        ep.v_next = vnxt;
        cudaEvent_t e0;
        CPD_OK_OR_RETURN(timed_begin(s, e0));
        if (s->params.precision == CPD_MIXED)
            CPD_LAUNCHED(launch_hertz_force_mixed(pk, s->contact.view(), s->md, true, s->stream,
                                                  &ep));
        else
            CPD_LAUNCHED(launch_hertz_force(pk, s->contact.view(), s->md, true, s->stream, &ep));
        CPD_OK_OR_RETURN(timed_end(s, e0));
        std::swap(vcur, vnxt);
        if (k + 1 < num_steps) std::swap(ucur, unxt);
    }
    // The last kernel wrote the final velocity into vcur (after the swap).
    if (vcur != s->v)
        CPD_CUDA(cudaMemcpyAsync(s->v, vcur, vec, cudaMemcpyDeviceToDevice, s->stream));
    return CPD_OK;
}

// energy_part (mixed stencil path, one particle volume): the last step's
// bond kernel also forms W and phi of the stencil rows and their per-warp
// partial sums there.
cpd_status step_fused(cpd_system* s, int32_t num_steps, double* energy_part = nullptr)
{
    if (contact_fusable(s)) return step_fused_contact(s, num_steps);
    const bool mixed = use_mixed(s);
    const bool start_alt = ((num_steps - 1) & 1) != 0;
    double* ucur = start_alt ? s->u_alt : s->u;
    double* unxt = start_alt ? s->u : s->u_alt;
    MixedU* u2cur = mixed ? (start_alt ? s->u2_alt : s->mixed.u2) : nullptr;
    MixedU* u2nxt = mixed ? (start_alt ? s->mixed.u2 : s->u2_alt) : nullptr;
    const bool sten = use_stencil64(s);
    double4* u4cur = sten ? (start_alt ? s->mixed.u4_alt : s->mixed.u4) : nullptr;
    double4* u4nxt = sten ? (start_alt ? s->mixed.u4 : s->mixed.u4_alt) : nullptr;
    // Frozen rows are never integrated, so the kernels write only rows from
    // frozen on: the second buffer takes the frozen rows' displacement (and
    // its FP32 split) from the system's arrays, where every call starts.
    if (s->frozen > 0) {
        const size_t bytes = sizeof(double) * (size_t)s->frozen;
        for (int d = 0; d < 3; ++d)
            CPD_CUDA(cudaMemcpyAsync(s->u_alt + (size_t)d * s->npad, s->u + (size_t)d * s->npad,
                                     bytes, cudaMemcpyDeviceToDevice, s->stream));
        if (mixed)
            CPD_CUDA(cudaMemcpyAsync(s->u2_alt, s->mixed.u2, sizeof(MixedU) * (size_t)s->frozen,
                                     cudaMemcpyDeviceToDevice, s->stream));
    }
    const ParticleView p = view(s);
    if (mixed)
        CPD_LAUNCHED(launch_vv_initial_mixed(p, s->md, s->params.dt, ucur, u2cur, s->stream));
    else
        CPD_LAUNCHED(launch_vv_initial(p, s->params.dt, false, nullptr, 0, ucur, s->stream));
    if (sten) {
        // Gather records of the first step's displacement, and the frozen
        // rows of the second buffer (the kernels write rows from frozen on).
        CPD_LAUNCHED(launch_pack_u4(p, ucur, 0, s->n, u4cur, s->stream, s->mixed.gcell));
        CPD_LAUNCHED(launch_pack_u4(p, s->u, 0, s->frozen, u4nxt, s->stream, s->mixed.gcell));
    }
    StepEpilogue ep;
    ep.dt = s->params.dt;
    ep.half_dt = 0.5 * s->params.dt;
    ep.c = mixed_wscale(s->md);
    ep.bc_bits = s->bc_bits;
    ep.bc_row = s->bc_row;
    ep.bc_keep = s->bc_keep;
    ep.bc_add = s->bc_add;
    ep.nbc = s->nbc;
    ep.u4_cell = sten ? s->mixed.gcell : nullptr;
    for (int32_t k = 0; k < num_steps; ++k) {
        ParticleView pk = p;
        pk.u = ucur;
        MixedState mk = s->mixed;
        mk.u2 = u2cur;
        mk.u4 = u4cur;
        ep.mode = k + 1 < num_steps ? 2 : 1;
        ep.u_next = unxt;
        ep.u2_next = u2nxt;
        ep.u4_next = u4nxt;
        ep.energy_part = k + 1 < num_steps ? nullptr : energy_part;
        if (is_lps(s)) CPD_OK_OR_RETURN(lps_prepare_on(s, pk, mk, s->md.fracture != 0));
        CPD_OK_OR_RETURN(pd_force_on(s, pk, mk, ep));
        std::swap(ucur, unxt);
        std::swap(u2cur, u2nxt);
        std::swap(u4cur, u4nxt);
    }
    s->steps_since_rebuild += num_steps;
    return CPD_OK;
}

cpd_status check_ready(const cpd_system* s, bool need_neighbors)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    if (s->n == 0) return set_error(CPD_ERR_STATE, "no particles uploaded");
    if (need_neighbors && !s->neighbors_built)
        return set_error(CPD_ERR_STATE, "neighbour list not built");
    return CPD_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Hooks for the batched step (cpd_batch.cu).
namespace cpd {

cpd_status batch_attach(cpd_system* s, const void* batch, BatchInstance* out, int64_t* bonds)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    if (s->batch) return set_error(CPD_ERR_STATE, "the system already belongs to a batch");
    if (!s->initialized) return set_error(CPD_ERR_STATE, "call cpd_init before batching a system");
    if (!has_pd(s) || has_contact(s))
        return set_error(CPD_ERR_INVALID_ARGUMENT,
                         "a batch takes peridynamic systems without contact");
    if (s->params.precision == CPD_FP64_EXACT)
        return set_error(CPD_ERR_INVALID_ARGUMENT,
                         "a batch runs the CPD_FP64 or CPD_MIXED kernels, not CPD_FP64_EXACT");
    if (!fused_ready(s))
        return set_error(CPD_ERR_STATE,
                         "the system's boundary conditions do not fit the fused step");
    CPD_CUDA(cudaSetDevice(s->device));
    BatchInstance b;
    std::memset(static_cast<void*>(&b), 0, sizeof b);
    b.p = view(s);
    b.nl = pd_view(s);
    b.ep.dt = s->params.dt;
    b.ep.half_dt = 0.5 * s->params.dt;
    b.ep.c = mixed_wscale(s->md);
    b.ep.bc_bits = s->bc_bits;
    b.ep.bc_row = s->bc_row;
    b.ep.bc_keep = s->bc_keep;
    b.ep.bc_add = s->bc_add;
    b.ep.nbc = s->nbc;
    b.u_alt = s->u_alt;
    b.fm = to_fast(s->md);
    b.wscale = mixed_wscale(s->md);
    b.pd = s->md.pd;
    b.fracture = s->md.fracture;
    b.influence = s->md.influence;
    const MixedState& m = s->mixed;
    if (use_mixed(s)) {
        b.body = kBatchMixed;
        b.mv = MixedView{m.xh, m.xl, m.u2, m.code, m.table, m.warp_kind, m.pmask, m.warp_pmask};
        b.u2_alt = s->u2_alt;
        b.ab = m.ab;
        b.mm = to_mixed_model(s->md, m);
        b.ml = to_mixed_lps(s->md, m);
    } else if (use_fast(s)) {
        b.body = kBatchFast;
    } else {
        return set_error(CPD_ERR_INVALID_ARGUMENT, "no batch kernel for this model");
    }
    // Frozen rows are never integrated: the second buffers take them once.
    if (s->frozen > 0) {
        const size_t bytes = sizeof(double) * (size_t)s->frozen;
        for (int d = 0; d < 3; ++d)
            CPD_CUDA(cudaMemcpyAsync(s->u_alt + (size_t)d * s->npad, s->u + (size_t)d * s->npad,
                                     bytes, cudaMemcpyDeviceToDevice, s->stream));
        if (b.body == kBatchMixed)
            CPD_CUDA(cudaMemcpyAsync(s->u2_alt, m.u2, sizeof(MixedU) * (size_t)s->frozen,
                                     cudaMemcpyDeviceToDevice, s->stream));
    }
    *out = b;
    *bonds = s->pd.total;
    s->batch = batch;
    return CPD_OK;
}

void batch_detach(cpd_system* s)
{
    if (s) s->batch = nullptr;
}

cudaStream_t system_stream(const cpd_system* s) { return s->stream; }
int system_device(const cpd_system* s) { return s->device; }
int64_t system_rows(const cpd_system* s) { return s->n - s->frozen; }

}  // namespace cpd

// ===========================================================================
extern "C" {

int32_t cpd_abi_version(void) { return CPD_ABI_VERSION; }

cpd_status cpd_stencil_stats(const cpd_system* s, int64_t* stencil_warps,
                             int64_t* irregular_warps, int32_t* table_entries)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    const bool sten = (use_mixed(s) && s->mixed.st32) ||
                      (use_stencil64(s) && (s->mixed.st64 || s->mixed.st64w));
    if (stencil_warps) *stencil_warps = sten ? s->mixed.nstencil : 0;
    if (irregular_warps) *irregular_warps = sten ? s->mixed.nirregular : 0;
    if (table_entries) *table_entries = sten ? s->mixed.ntab : 0;
    return CPD_OK;
}
const char* cpd_last_error(void) { return g_last_error.c_str(); }

cpd_status cpd_system_create(const cpd_params* params, cpd_system** out)
{
    if (!params || !out) return set_error(CPD_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    const cpd_params& P = *params;
    if (P.pd_model < CPD_PD_NONE || P.pd_model > CPD_PD_LINEAR_LPS)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "unknown pd_model");
    if (P.contact_model != CPD_CONTACT_NONE && P.contact_model != CPD_CONTACT_HERTZ &&
        P.contact_model != CPD_CONTACT_NORMAL_REPULSION)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "unknown contact_model");
    if (P.pd_model == CPD_PD_NONE && P.contact_model == CPD_CONTACT_NONE)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "need a PD model or a contact model");
    // Force<LinearPMB, Fracture> is not defined (force/CabanaPD_PMB.hpp:407).
    if (P.pd_model == CPD_PD_LINEAR_PMB && P.fracture)
        return set_error(CPD_ERR_UNSUPPORTED, "LinearPMB has no fracture variant");
    if (P.pd_model != CPD_PD_NONE && !(P.horizon > 0))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "horizon must be > 0");
    if (P.contact_model != CPD_CONTACT_NONE && !(P.contact_radius > 0))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "contact_radius must be > 0");
    if (P.contact_model == CPD_CONTACT_NORMAL_REPULSION && !(P.contact_horizon > 0))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "contact_horizon must be > 0");
    if (P.precision != CPD_FP64_EXACT && P.precision != CPD_FP64 && P.precision != CPD_MIXED)
        return set_error(CPD_ERR_UNSUPPORTED, "unknown precision mode");
    if (P.ordering != CPD_ORDER_INPUT && P.ordering != CPD_ORDER_MORTON)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "unknown ordering");
    const bool lps = P.pd_model == CPD_PD_LPS || P.pd_model == CPD_PD_LINEAR_LPS;
    const int infl = P.influence_type >= 0 ? P.influence_type : (lps ? 0 : 1);
    if (infl != 0 && infl != 1)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "Influence function type must be 0 or 1.");

    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return set_error(CPD_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (P.device < 0 || P.device >= ndev)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    CPD_CUDA(cudaSetDevice(P.device));

    cpd_system* s = new cpd_system();
    s->params = P;
    s->device = P.device;
    Model& md = s->md;
    // LinearLPS computes with the LPS kernels: ForceModel<LinearLPS>
    // (force_models/CabanaPD_LPS.hpp:255-272) keeps the base model's
    // force_tag = LPS (:32), and the Solver instantiates
    // Force<memory_space, force_tag, fracture_type> (CabanaPD_Solver.hpp:96-99),
    // so the linearised Force<LinearLPS> is never selected.
    md.pd = P.pd_model == CPD_PD_LINEAR_LPS ? CPD_PD_LPS : P.pd_model;
    md.fracture = P.fracture ? 1 : 0;
    md.contact = P.contact_model;
    md.influence = infl;
    md.horizon = P.horizon;
    md.K = P.K;
    md.G = P.G;
    md.G0 = P.G0;
    if (md.pd != CPD_PD_NONE) {
        const double h = md.horizon;
        // force_models/CabanaPD_PMB.hpp:44-46
        md.c = 18.0 * md.K / (kPi * h * h * h * h);
        // force_models/CabanaPD_LPS.hpp:66-67
        md.theta_coeff = 3.0 * md.K - 5.0 * md.G;
        md.s_coeff = 15.0 * md.G;
        if (md.fracture) {
            // CabanaPD_ForceModels.hpp:97-101 (LPS ctor :209-223 agrees)
            md.s0 = std::sqrt(5.0 * md.G0 / 9.0 / md.K / h);
            if (md.influence == 0) md.s0 = std::sqrt(8.0 * md.G0 / 15.0 / md.K / h);
            md.bond_break_coeff = (1.0 + md.s0) * (1.0 + md.s0);
        }
    }
    if (md.contact == CPD_CONTACT_HERTZ) {
        // force_models/CabanaPD_Hertzian.hpp:40-56
        md.radius = P.contact_radius;
        md.radius_extend = P.radius_extend;
        md.nu = P.nu;
        md.E = P.E;
        md.e = P.restitution;
        md.Rs = 0.5 * md.radius;
        md.Es = md.E / (2.0 * (1.0 - std::pow(md.nu, 2.0)));
        const double ln_e = std::log(md.e);
        md.beta = -ln_e / std::sqrt(std::pow(ln_e, 2.0) + std::pow(kPi, 2.0));
        md.coeff_h_n = 4.0 / 3.0 * md.Es * std::sqrt(md.Rs);
        md.coeff_h_d = -2.0 * std::sqrt(5.0 / 6.0) * md.beta;
        md.per_particle_radius = P.per_particle_radius ? 1 : 0;
    }
    if (md.contact == CPD_CONTACT_NORMAL_REPULSION) {
        // force_models/CabanaPD_Contact.hpp:70-79 (c as the PMB model's)
        md.radius = P.contact_radius;
        md.radius_extend = P.radius_extend;
        md.contact_horizon = P.contact_horizon;
        const double h = md.contact_horizon;
        md.c_contact = 18.0 * P.contact_K / (kPi * h * h * h * h);
    }
    e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete s;
        return set_error(CPD_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
    }
    s->stream = s->own_stream;
    e = cudaMallocHost(&s->h_red, sizeof(double) * 8);
    if (e != cudaSuccess) {
        cudaStreamDestroy(s->own_stream);
        delete s;
        return set_error(CPD_ERR_CUDA, std::string("pinned: ") + cudaGetErrorString(e));
    }
    system_opened(s->device);
    *out = s;
    return CPD_OK;
}

cpd_status cpd_system_destroy(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    if (!s) return CPD_OK;
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_particles(s);
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto& pr : s->pending) {
        cudaEventDestroy(pr.first);
        cudaEventDestroy(pr.second);
    }
    for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
    if (s->h_red) cudaFreeHost(s->h_red);
    if (s->own_stream) cudaStreamDestroy(s->own_stream);
    system_closed(s->device);
    delete s;
    return CPD_OK;
}

cpd_status cpd_set_stream(cpd_system* s, void* stream)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    s->stream = stream ? (cudaStream_t)stream : s->own_stream;
    return CPD_OK;
}

cpd_status cpd_get_stream(cpd_system* s, void** stream)
{
    if (!s || !stream) return set_error(CPD_ERR_INVALID_ARGUMENT, "null argument");
    *stream = (void*)s->stream;
    return CPD_OK;
}

cpd_status cpd_model_constants(const cpd_system* s, double* o)
{
    if (!s || !o) return set_error(CPD_ERR_INVALID_ARGUMENT, "null argument");
    const Model& m = s->md;
    const double v[10] = {m.c,  m.s0, m.bond_break_coeff, m.theta_coeff, m.s_coeff,
                          m.Rs, m.Es, m.beta,             m.coeff_h_n,   m.coeff_h_d};
    std::memcpy(o, v, sizeof(v));
    return CPD_OK;
}

cpd_status cpd_upload_particles(cpd_system* s, int64_t n, int64_t n_frozen, const double* x,
                                const double* vol, const double* rho, const int32_t* nofail,
                                const double* radius)
{
    CPD_NOT_IN_BATCH(s);
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    if (n <= 0 || n >= (int64_t)1 << 31 || n_frozen < 0 || n_frozen > n || !x || !vol)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_upload_particles: bad arguments");
    if (s->md.per_particle_radius && !radius)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "per-particle radius model needs radius");
    CPD_CUDA(cudaSetDevice(s->device));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    PhaseTrace tr("upload");
    free_particles(s);
    s->n = n;
    s->frozen = n_frozen;
    s->npad = std::max<int64_t>(128, (n + 127) / 128 * 128);
    const size_t sv = sizeof(double) * 3 * s->npad, ss = sizeof(double) * s->npad;
    double** vec[] = {&s->x, &s->u, &s->v, &s->f, &s->u_neigh};
    for (double** a : vec) {
        CPD_CUDA(dev_alloc(a, sv, s->stream));
        CPD_CUDA(cudaMemsetAsync(*a, 0, sv, s->stream));
    }
    double** sca[] = {&s->vol, &s->rho, &s->m, &s->theta, &s->lps_a, &s->lps_b,
                      &s->W,   &s->phi, &s->radius};
    for (double** a : sca) {
        CPD_CUDA(dev_alloc(a, ss, s->stream));
        CPD_CUDA(cudaMemsetAsync(*a, 0, ss, s->stream));
    }
    CPD_CUDA(dev_alloc(&s->nofail, s->npad, s->stream));
    CPD_CUDA(cudaMemsetAsync(s->nofail, 0, s->npad, s->stream));
    CPD_CUDA(dev_alloc(&s->staging, sizeof(double) * 3 * n, s->stream));
    CPD_CUDA(dev_alloc(&s->red_out, sizeof(double) * 8, s->stream));
    CPD_CUDA(cudaMemsetAsync(s->red_out, 0, sizeof(double) * 8, s->stream));
    tr.mark("alloc", s->stream);

    // Internal order: the caller's (no permutation) or Morton (perm[k] =
    // caller index of internal particle k, h_inv its inverse).
    s->h_inv.clear();
    if (s->params.ordering == CPD_ORDER_MORTON) {
        double cell = has_pd(s) ? s->md.horizon : 2.0 * s->md.radius + s->md.radius_extend;
        const std::vector<int32_t> order = morton_order(x, n, n_frozen, cell);
        CPD_CUDA(dev_alloc(&s->perm, sizeof(int32_t) * n, s->stream));
        CPD_CUDA(cudaMemcpyAsync(s->perm, order.data(), sizeof(int32_t) * n,
                                 cudaMemcpyHostToDevice, s->stream));
        s->h_inv.assign(n, 0);
        for (int64_t k = 0; k < n; k++) s->h_inv[order[k]] = (int32_t)k;
        CPD_CUDA(cudaStreamSynchronize(s->stream));
    }
    tr.mark("order", s->stream);

    // Each upload goes through the staging buffer, so one waits for the
    // previous conversion kernel (stream order).
    CPD_OK_OR_RETURN(upload_vector(s, x, s->x));
    CPD_OK_OR_RETURN(upload_scalar(s, vol, s->vol));
    if (rho)
        CPD_OK_OR_RETURN(upload_scalar(s, rho, s->rho));
    else
        s->launches += launch_fill_value(s->rho, n, 1.0, s->stream);
    if (radius)
        CPD_OK_OR_RETURN(upload_scalar(s, radius, s->radius));
    else
        s->launches += launch_fill_value(s->radius, n, s->md.radius, s->stream);
    if (nofail) {
        CPD_CUDA(cudaMemcpyAsync(s->staging, nofail, sizeof(int32_t) * n, cudaMemcpyHostToDevice,
                                 s->stream));
        s->launches += launch_nofail_to_u8(reinterpret_cast<const int32_t*>(s->staging),
                                           s->nofail, n, s->perm, s->stream);
    }
    CPD_CUDA(cudaGetLastError());
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    tr.mark("fields", s->stream);
    return CPD_OK;
}

cpd_status cpd_set_state(cpd_system* s, const double* u, const double* v)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, false));
    CPD_CUDA(cudaSetDevice(s->device));
    if (u) CPD_OK_OR_RETURN(upload_vector(s, u, s->u));
    if (v) CPD_OK_OR_RETURN(upload_vector(s, v, s->v));
    if (use_mixed(s) && s->mixed.u2)
        s->launches += launch_split_u(view(s), s->md, s->mixed, s->stream);
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

cpd_status cpd_build_neighbors(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, false));
    CPD_CUDA(cudaSetDevice(s->device));
    std::string err;
    PhaseTrace tr("neighbors");
    // The fused step's second split buffer carries the guard of the stencil
    // set up below: it is allocated again when the step is next prepared.
    if (s->u2_alt_base) dev_free(s->u2_alt_base, s->stream);
    s->u2_alt = s->u2_alt_base = nullptr;
    s->mixed_via_fp64 = false;
    if (has_pd(s)) {
        // CabanaPD_Neighbor.hpp:56-59: reference positions, cutoff + 1e-14.
        double hmin[3];
        const bool spacing = wants_mixed(s) || wants_stencil64(s);
        int l = build_neighbor_list(s->x, nullptr, s->n, s->npad, s->frozen,
                                    s->md.horizon + 1e-14, s->perm, s->md.fracture != 0,
                                    s->pd, s->stream, err, spacing ? hmin : nullptr);
        if (l < 0) return set_error(CPD_ERR_CUDA, "neighbour build: " + err);
        s->pd.hmin_valid = spacing;
        if (spacing)
            for (int d = 0; d < 3; ++d) s->pd.hmin[d] = hmin[d];
        s->launches += l;
        tr.mark("list", s->stream);
        const int entries = wants_mixed(s) && s->md.pd == CPD_PD_PMB
                                ? lattice_table_entries(s->pd.hmin, s->md.horizon + 1e-14)
                                : 0;
        const bool wide = entries >= kMixedGeneric && entries <= kStencilMaxWide;
        if (wide || (entries > 0 && entries <= kStencilMax &&
                     lattice_layout_probe(view(s), s->pd.hmin, s->stream) == 2)) {
            // CPD_MIXED PMB where the FP64 stencil kernel takes rows the mixed
            // kernels would give to their general form, and runs faster:
            // - a horizon whose lattice table is past the byte codes (four
            //   spacings: 256 entries), where the mixed kernels would take
            //   FP32 positions on every bond (1.04 vs 2.83 ms per step on a
            //   1.44 M-particle plate);
            // - a lattice body whose particle order is not one box of lattice
            //   lines (holes), where the FP64 records go by lattice cell and
            //   keep every row, the mixed ones only the majority's (a holed
            //   1.44 M-particle plate: 0.49 vs 0.61 ms).
            // Results are FP64's. It runs when the lattice allows it.
            s->mixed_via_fp64 = true;
            l = prepare_mixed(view(s), s->pd, s->md.horizon + 1e-14, false, s->mixed,
                              s->stream, err, &s->md);
            if (l < 0) return set_error(CPD_ERR_CUDA, "stencil set-up: " + err);
            s->launches += l;
            if (!stencil64_ready(s->mixed)) {
                free_mixed(s->mixed, s->stream);
                s->mixed_via_fp64 = false;
            }
        }
        if (wants_mixed(s)) {
            l = prepare_mixed(view(s), s->pd, s->md.horizon + 1e-14, is_lps(s), s->mixed,
                              s->stream, err, nullptr,
                              s->md.pd == CPD_PD_PMB ? &s->md : nullptr);
            if (l < 0) return set_error(CPD_ERR_CUDA, "mixed-precision set-up: " + err);
            s->launches += l;
        } else if (wants_stencil64(s) && !s->mixed_via_fp64) {
            l = prepare_mixed(view(s), s->pd, s->md.horizon + 1e-14, false, s->mixed,
                              s->stream, err, &s->md);
            if (l < 0) return set_error(CPD_ERR_CUDA, "stencil set-up: " + err);
            s->launches += l;
        }
    }
    if (has_contact(s)) {
        // CabanaPD_Neighbor.hpp:60-63: current positions, cutoff + 1e-14.
        CPD_OK_OR_RETURN(rebuild_contact(s, 2.0 * s->md.radius + s->md.radius_extend + 1e-14));
        s->rebuilds = 0;
    }
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    s->neighbors_built = true;
    s->initialized = false;
    return CPD_OK;
}

cpd_status cpd_neighbor_stats(const cpd_system* s, int32_t* max_n, int64_t* total)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    const NeighborList& nl = has_pd(s) ? s->pd : s->contact;
    if (max_n) *max_n = nl.max_n;
    if (total) *total = nl.total;
    return CPD_OK;
}

cpd_status cpd_download_neighbors(cpd_system* s, int32_t* counts, int32_t* indices,
                                  int32_t* mu)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    const NeighborList& nl = has_pd(s) ? s->pd : s->contact;
    const size_t cells = (size_t)s->n * std::max(nl.max_n, 1);
    int32_t *dc = nullptr, *di = nullptr, *dm = nullptr;
    CPD_CUDA(dev_alloc(&dc, sizeof(int32_t) * s->n, s->stream));
    CPD_CUDA(dev_alloc(&di, sizeof(int32_t) * cells, s->stream));
    CPD_CUDA(dev_alloc(&dm, sizeof(int32_t) * cells, s->stream));
    NeighborList tmp = nl;
    if (!(has_pd(s) && s->md.fracture)) tmp.mu = nullptr;
    s->launches += launch_ell_to_rows(tmp, s->n, s->npad, s->perm, s->perm, dc, di, dm, s->stream);
    CPD_CUDA(cudaGetLastError());
    if (counts)
        CPD_CUDA(cudaMemcpyAsync(counts, dc, sizeof(int32_t) * s->n, cudaMemcpyDeviceToHost,
                                 s->stream));
    if (indices && nl.max_n > 0)
        CPD_CUDA(cudaMemcpyAsync(indices, di, sizeof(int32_t) * cells, cudaMemcpyDeviceToHost,
                                 s->stream));
    if (mu && nl.max_n > 0)
        CPD_CUDA(cudaMemcpyAsync(mu, dm, sizeof(int32_t) * cells, cudaMemcpyDeviceToHost,
                                 s->stream));
    dev_free(dc, s->stream);
    dev_free(di, s->stream);
    dev_free(dm, s->stream);
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

cpd_status cpd_prenotch(cpd_system* s, int32_t count, const double* v1, const double* v2,
                        const double* p0)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!has_pd(s) || !s->md.fracture)
        return set_error(CPD_ERR_STATE, "Cannot create prenotch in system without fracture.");
    if (count < 0 || (count > 0 && (!v1 || !v2 || !p0)))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_prenotch: bad arguments");
    CPD_CUDA(cudaSetDevice(s->device));
    const ParticleView p = view(s);
    const double cutoff = s->md.horizon + 1e-14;
    for (int32_t q = 0; q < count; q++) {
        const double* a = v1 + 3 * q;
        const double* b = v2 + 3 * q;
        const double na = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        const double nb = std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
        const double cx = a[1] * b[2] - a[2] * b[1], cy = a[2] * b[0] - a[0] * b[2],
                     cz = a[0] * b[1] - a[1] * b[0];
        const double sin_ab = std::sqrt(cx * cx + cy * cy + cz * cz) / (na * nb);
        if (!(sin_ab > 1e-12))
            return set_error(CPD_ERR_INVALID_ARGUMENT, "notch vectors are parallel");
        // A bond (length <= cutoff) that can meet the notch within the
        // reference's 1e-10 parametric tolerances starts no farther than this
        // from the notch's bounding box (coplanar case: parametric extents
        // of the bond are bounded by |l| / sin(angle(v1, v2))).
        const double margin = cutoff * (2.0 + 2.0 / sin_ab) + 1e-6 * (na + nb + cutoff);
        CPD_LAUNCHED(launch_prenotch(p, s->pd.view(), a, b, p0 + 3 * q, margin, s->stream));
    }
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

cpd_status cpd_add_boundary_condition(cpd_system* s, int32_t kind, int32_t component,
                                      int64_t count, const int64_t* indices,
                                      const double* values)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, false));
    if (kind < CPD_BC_FORCE_VALUE || kind > CPD_BC_FORCE_ADD || count < 0 || !values ||
        (count > 0 && !indices))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_add_boundary_condition: bad arguments");
    if (kind == CPD_BC_FORCE_ADD && (component < 0 || component > 2))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "component must be 0, 1 or 2");
    CPD_CUDA(cudaSetDevice(s->device));
    BoundaryCondition bc;
    bc.kind = kind;
    bc.component = component;
    bc.count = count;
    bc.value = values[0];
    std::vector<int32_t> idx(count);
    for (int64_t b = 0; b < count; b++) {
        if (indices[b] < 0 || indices[b] >= s->n)
            return set_error(CPD_ERR_INVALID_ARGUMENT, "boundary index out of range");
        idx[b] = s->h_inv.empty() ? (int32_t)indices[b] : s->h_inv[indices[b]];
    }
    if (count > 0) {
        CPD_CUDA(dev_alloc(&bc.idx, sizeof(int32_t) * count, s->stream));
        CPD_CUDA(cudaMemcpyAsync(bc.idx, idx.data(), sizeof(int32_t) * count,
                                 cudaMemcpyHostToDevice, s->stream));
        if (kind == CPD_BC_FORCE_ADD) {
            CPD_CUDA(dev_alloc(&bc.values, sizeof(double) * count, s->stream));
            CPD_CUDA(cudaMemcpyAsync(bc.values, values, sizeof(double) * count,
                                     cudaMemcpyHostToDevice, s->stream));
        }
        CPD_CUDA(cudaStreamSynchronize(s->stream));
    }
    s->bcs.push_back(bc);
    cpd_system::HostBC hb;
    hb.kind = kind;
    hb.component = component;
    hb.idx = idx;
    hb.values.assign(values, values + (kind == CPD_BC_FORCE_ADD ? count : 1));
    s->hbcs.push_back(std::move(hb));
    free_bc_program(s);
    if (s->initialized) CPD_OK_OR_RETURN(prepare_fused(s));
    return CPD_OK;
}

cpd_status cpd_clear_boundary_conditions(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    for (auto& bc : s->bcs) {
        if (bc.idx) dev_free(bc.idx, s->stream);
        if (bc.values) dev_free(bc.values, s->stream);
    }
    s->bcs.clear();
    s->hbcs.clear();
    free_bc_program(s);
    if (s->initialized) CPD_OK_OR_RETURN(prepare_fused(s));
    return CPD_OK;
}

cpd_status cpd_compute_weighted_volume(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    if (is_lps(s)) CPD_LAUNCHED(launch_lps_weighted_volume(view(s), pd_view(s), s->md, s->stream));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

cpd_status cpd_compute_dilatation(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    if (is_lps(s)) CPD_OK_OR_RETURN(lps_prepare(s, false));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

// The mixed kernel reads the FP32 split of u; refresh it where u may have
// changed outside the integrator (set_state, init, kernel-level calls).
cpd_status refresh_mixed_u(cpd_system* s)
{
    if (use_mixed(s) && s->mixed.u2)
        CPD_LAUNCHED(launch_split_u(view(s), s->md, s->mixed, s->stream));
    return CPD_OK;
}

cpd_status cpd_compute_force(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    CPD_OK_OR_RETURN(refresh_mixed_u(s));
    if (has_pd(s)) CPD_OK_OR_RETURN(pd_force(s));
    if (has_contact(s)) CPD_OK_OR_RETURN(contact_force(s, !has_pd(s)));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

// The energy kernel of the system's arithmetic path: the stencil form on the
// mixed path, the fast FP64 form on the FP64 path (PMB, LPS), the exact form
// otherwise. Writes W and phi through p and block partials [rows][2] into a
// buffer of capacity rows (at least energy_blocks(rows), nb); returns the
// partial rows written (nb, or up to nb + 1 for the mixed split form).
static int launch_energy(cpd_system* s, const ParticleView& p, double* partials, int nb,
                         int capacity)
{
    if (use_mixed(s) && s->mixed.u2) {
        int l = 0;
        const int rows = launch_energy_mixed(p, pd_view(s), s->md, s->mixed, partials, nb,
                                             capacity, &l, s->stream);
        s->launches += l;
        if (rows >= 0) return rows;
    }
    if (s->params.precision != CPD_FP64_EXACT) {
        const int l = launch_pd_energy_fast(p, pd_view(s), s->md, partials, nb, s->stream);
        if (l >= 0) {
            s->launches += l;
            return nb;
        }
    }
    s->launches += launch_pd_energy(p, pd_view(s), s->md, partials, nb, s->stream);
    return nb;
}

// Totals from rows of (W_i vol_i, phi_i) partial sums in s->red.
static cpd_status sum_energy_partials(cpd_system* s, int rows, double* total_W, double* total_D)
{
    CPD_CUDA(cudaGetLastError());
    CPD_LAUNCHED(launch_sum_partials(s->red, rows, 2, s->red_out + 2, s->stream));
    CPD_CUDA(cudaMemcpyAsync(s->h_red + 2, s->red_out + 2, sizeof(double) * 2,
                             cudaMemcpyDeviceToHost, s->stream));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    if (total_W) *total_W = s->h_red[2];
    if (total_D) *total_D = s->h_red[3];
    return CPD_OK;
}

cpd_status cpd_compute_energy(cpd_system* s, double* total_W, double* total_D)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    if (has_pd(s)) {
        const int nb = energy_blocks(s->n - s->frozen);
        CPD_OK_OR_RETURN(ensure_reduction(s, nb + 1));
        const int rows = launch_energy(s, view(s), s->red, nb, nb + 1);
        return sum_energy_partials(s, rows, total_W, total_D);
    }
    if (total_W) *total_W = 0.0;
    if (total_D) *total_D = 0.0;
    return CPD_OK;
}

// CabanaPD_Force.hpp:222-235 computeStress: the stress of the current state
// (bond bits and, for LPS, the m / theta of the last force update), zeroed
// first. Allocates its arrays on the first call.
cpd_status cpd_compute_stress(cpd_system* s)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    if (!s->stress) {
        CPD_CUDA(dev_alloc(&s->stress, sizeof(double) * 9 * s->npad, s->stream));
        CPD_CUDA(dev_alloc(&s->stress_staging, sizeof(double) * 9 * std::max<int64_t>(s->n, 1),
                           s->stream));
    }
    CPD_CUDA(cudaMemsetAsync(s->stress, 0, sizeof(double) * 9 * s->npad, s->stream));
    if (has_pd(s)) CPD_LAUNCHED(launch_pd_stress(view(s), pd_view(s), s->md, s->stress, s->stream));
    s->stress_ready = true;
    return CPD_OK;
}

// CabanaPD_Solver.hpp:229-279 init(bc): weighted volume once without
// fracture, updateForce (no contact force unless the contact model is the
// force model), energy, force BCs at t = 0.
cpd_status cpd_init(cpd_system* s)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    CPD_CUDA(cudaSetDevice(s->device));
    CPD_OK_OR_RETURN(refresh_mixed_u(s));
    if (has_pd(s)) {
        // Weighted volume once here without fracture (Solver.hpp:235-239),
        // inside updateForce with fracture (Solver.hpp:466-470): once either way.
        if (is_lps(s)) CPD_OK_OR_RETURN(lps_prepare(s, true));
        CPD_OK_OR_RETURN(pd_force(s));
    } else if (has_contact(s)) {
        CPD_OK_OR_RETURN(contact_force(s, true));
    }
    PhaseTrace tr("init");
    // Solver.hpp:240-242: the energy and damage of the initial state (the
    // fields; the totals are not kept).
    if (has_pd(s)) CPD_OK_OR_RETURN(cpd_compute_energy(s, nullptr, nullptr));
    tr.mark("energy", s->stream);
    CPD_OK_OR_RETURN(apply_force_bcs(s));
    CPD_OK_OR_RETURN(prepare_fused(s));
    tr.mark("bcs+fused", s->stream);
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    s->initialized = true;
    return CPD_OK;
}

// CabanaPD_Solver.hpp:332-375 runStep(step, bc), num_steps times.
cpd_status cpd_step(cpd_system* s, int32_t num_steps)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!s->initialized) return set_error(CPD_ERR_STATE, "call cpd_init before cpd_step");
    if (num_steps < 0) return set_error(CPD_ERR_INVALID_ARGUMENT, "num_steps < 0");
    CPD_CUDA(cudaSetDevice(s->device));
    if (num_steps > 0 && !fused_ready(s)) {
        // Prepare now unless the stream is being captured (then the steps
        // run as separate kernels, which need nothing prepared).
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CPD_CUDA(cudaStreamIsCapturing(s->stream, &cs));
        if (cs == cudaStreamCaptureStatusNone) CPD_OK_OR_RETURN(prepare_fused(s));
    }
    if (num_steps > 0 && fused_ready(s)) return step_fused(s, num_steps);
    const ParticleView p = view(s);
    for (int32_t k = 0; k < num_steps; k++) {
        CPD_OK_OR_RETURN(vv_initial(s));
        CPD_OK_OR_RETURN(update_force(s));
        CPD_OK_OR_RETURN(apply_force_bcs(s));
        CPD_LAUNCHED(launch_vv_final(p, s->params.dt, s->stream));
    }
    return CPD_OK;
}

cpd_status cpd_step_energy(cpd_system* s, int32_t num_steps, double* total_W, double* total_D)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!s->initialized) return set_error(CPD_ERR_STATE, "call cpd_init before cpd_step_energy");
    if (num_steps < 0) return set_error(CPD_ERR_INVALID_ARGUMENT, "num_steps < 0");
    CPD_CUDA(cudaSetDevice(s->device));
    if (num_steps > 0 && !fused_ready(s)) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        CPD_CUDA(cudaStreamIsCapturing(s->stream, &cs));
        if (cs == cudaStreamCaptureStatusNone) CPD_OK_OR_RETURN(prepare_fused(s));
    }
    if (num_steps > 0 && fused_ready(s) && fused_energy_ok(s)) {
        // The last step's mixed stencil kernel forms W and phi of its rows
        // (after that step's bond breaking, on the displacement the step
        // ends with) and one partial row per stencil warp; the irregular
        // rows take the energy kernel afterwards, on the same final state.
        const int64_t wrows = s->mixed.nstencil;
        const int64_t gi = (s->mixed.nirregular + 7) / 8;
        CPD_OK_OR_RETURN(ensure_reduction(s, (int)(wrows + gi + 1)));
        CPD_OK_OR_RETURN(step_fused(s, num_steps, s->red));
        int rows = (int)wrows;
        if (s->mixed.nirregular > 0) {
            int l = 0;
            const int r = launch_energy_mixed_rows(view(s), pd_view(s), s->md, s->mixed,
                                                   s->mixed.irregular_list,
                                                   s->mixed.nirregular, s->red + 2 * wrows, &l,
                                                   s->stream);
            s->launches += l;
            if (r < 0) return set_error(CPD_ERR_STATE, "energy of the irregular rows");
            rows += r;
        }
        return sum_energy_partials(s, rows, total_W, total_D);
    }
    CPD_OK_OR_RETURN(cpd_step(s, num_steps));
    return cpd_compute_energy(s, total_W, total_D);
}

cpd_status cpd_step_stage(cpd_system* s, int32_t stage)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!s->initialized) return set_error(CPD_ERR_STATE, "call cpd_init before cpd_step_stage");
    CPD_CUDA(cudaSetDevice(s->device));
    switch (stage) {
    case CPD_STAGE_INITIAL_HALF: return vv_initial(s);
    case CPD_STAGE_FORCE:
        // Device code run between stages may have written u: re-split it for
        // the mixed kernels (a no-op in the FP64 modes).
        CPD_OK_OR_RETURN(refresh_mixed_u(s));
        return update_force(s);
    case CPD_STAGE_FORCE_BC: return apply_force_bcs(s);
    case CPD_STAGE_FINAL_HALF:
        CPD_LAUNCHED(launch_vv_final(view(s), s->params.dt, s->stream));
        return CPD_OK;
    default: return set_error(CPD_ERR_INVALID_ARGUMENT, "unknown step stage");
    }
}

cpd_status cpd_synchronize(cpd_system* s)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    CPD_CUDA(cudaSetDevice(s->device));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

cpd_status cpd_download(cpd_system* s, int32_t field, double* out)
{
    CPD_OK_OR_RETURN(check_ready(s, false));
    if (!out) return set_error(CPD_ERR_INVALID_ARGUMENT, "null output");
    CPD_CUDA(cudaSetDevice(s->device));
    const double* src = nullptr;
    double* staging = s->staging;
    int comps = 1;
    switch (field) {
    case CPD_FIELD_STRESS:
        if (!s->stress_ready)
            return set_error(CPD_ERR_STATE, "stress: call cpd_compute_stress first");
        src = s->stress;
        staging = s->stress_staging;
        comps = 9;
        break;
    case CPD_FIELD_X: src = s->x; comps = 3; break;
    case CPD_FIELD_U: src = s->u; comps = 3; break;
    case CPD_FIELD_V: src = s->v; comps = 3; break;
    case CPD_FIELD_F: src = s->f; comps = 3; break;
    case CPD_FIELD_VOL: src = s->vol; break;
    case CPD_FIELD_RHO: src = s->rho; break;
    case CPD_FIELD_M: src = s->m; break;
    case CPD_FIELD_THETA: src = s->theta; break;
    case CPD_FIELD_W: src = s->W; break;
    case CPD_FIELD_PHI: src = s->phi; break;
    case CPD_FIELD_RADIUS: src = s->radius; break;
    default: return set_error(CPD_ERR_INVALID_ARGUMENT, "unknown field");
    }
    s->launches += launch_soa_to_aos(src, staging, s->n, s->npad, comps, s->perm, s->stream);
    CPD_CUDA(cudaGetLastError());
    CPD_CUDA(cudaMemcpyAsync(out, staging, sizeof(double) * comps * s->n,
                             cudaMemcpyDeviceToHost, s->stream));
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

// ---------------------------------------------------------------------------
// State snapshots: a header, then the device arrays in internal order.
namespace {

struct StateHeader {
    uint64_t magic;
    int64_t version, n, frozen, npad, pd_model, contact, fracture, ordering;
    int64_t max_n, nwords, total_bonds, contact_max_n, steps_since_rebuild, rebuilds;
    double max_disp;
};
constexpr uint64_t kStateMagic = 0x4554415453445043ull;  // "CPDSTATE" in little-endian bytes
constexpr int64_t kStateVersion = 1;

// The device arrays of a snapshot, in file order.
std::vector<std::pair<void*, size_t>> state_sections(cpd_system* s)
{
    const size_t vec = sizeof(double) * 3 * (size_t)s->npad;
    const size_t sca = sizeof(double) * (size_t)s->npad;
    std::vector<std::pair<void*, size_t>> out = {
        {s->u, vec}, {s->v, vec}, {s->f, vec},
        {s->m, sca}, {s->theta, sca}, {s->lps_a, sca}, {s->lps_b, sca}};
    if (has_pd(s) && s->pd.mu)
        out.push_back({s->pd.mu, sizeof(uint32_t) * (size_t)s->pd.nwords * (size_t)s->npad});
    if (has_contact(s)) out.push_back({s->u_neigh, vec});
    return out;
}

StateHeader state_header(const cpd_system* s)
{
    StateHeader h{};
    h.magic = kStateMagic;
    h.version = kStateVersion;
    h.n = s->n;
    h.frozen = s->frozen;
    h.npad = s->npad;
    h.pd_model = s->md.pd;
    h.contact = s->md.contact;
    h.fracture = s->md.fracture;
    h.ordering = s->params.ordering;
    h.max_n = s->pd.max_n;
    h.nwords = s->pd.nwords;
    h.total_bonds = s->pd.total;
    h.contact_max_n = has_contact(s) ? s->contact.max_n : 0;
    h.steps_since_rebuild = s->steps_since_rebuild;
    h.rebuilds = s->rebuilds;
    h.max_disp = s->max_disp;
    return h;
}

uint64_t state_bytes(cpd_system* s)
{
    uint64_t b = sizeof(StateHeader);
    for (const auto& sec : state_sections(s)) b += sec.second;
    return b;
}

}  // namespace

cpd_status cpd_state_bytes(cpd_system* s, uint64_t* bytes)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!bytes) return set_error(CPD_ERR_INVALID_ARGUMENT, "null output");
    *bytes = state_bytes(s);
    return CPD_OK;
}

cpd_status cpd_save_state(cpd_system* s, void* buf, uint64_t bytes)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!s->initialized) return set_error(CPD_ERR_STATE, "cpd_save_state: call cpd_init first");
    if (!buf || bytes < state_bytes(s))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_save_state: buffer smaller than cpd_state_bytes");
    CPD_CUDA(cudaSetDevice(s->device));
    const StateHeader h = state_header(s);
    std::memcpy(buf, &h, sizeof(h));
    char* dst = static_cast<char*>(buf) + sizeof(h);
    for (const auto& sec : state_sections(s)) {
        CPD_CUDA(cudaMemcpyAsync(dst, sec.first, sec.second, cudaMemcpyDeviceToHost, s->stream));
        dst += sec.second;
    }
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

cpd_status cpd_load_state(cpd_system* s, const void* buf, uint64_t bytes)
{
    CPD_NOT_IN_BATCH(s);
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!s->initialized) return set_error(CPD_ERR_STATE, "cpd_load_state: call cpd_init first");
    if (!buf || bytes < sizeof(StateHeader))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_load_state: no snapshot");
    StateHeader h;
    std::memcpy(&h, buf, sizeof(h));
    if (h.magic != kStateMagic || h.version != kStateVersion)
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_load_state: not a state snapshot of this version");
    const StateHeader mine = state_header(s);
    if (h.n != mine.n || h.frozen != mine.frozen || h.npad != mine.npad ||
        h.pd_model != mine.pd_model || h.contact != mine.contact ||
        h.fracture != mine.fracture || h.ordering != mine.ordering || h.max_n != mine.max_n ||
        h.nwords != mine.nwords || h.total_bonds != mine.total_bonds)
        return set_error(CPD_ERR_INVALID_ARGUMENT,
                         "cpd_load_state: the snapshot is of a system set up differently");
    if (bytes < state_bytes(s))
        return set_error(CPD_ERR_INVALID_ARGUMENT, "cpd_load_state: truncated snapshot");
    CPD_CUDA(cudaSetDevice(s->device));
    const char* src = static_cast<const char*>(buf) + sizeof(h);
    for (const auto& sec : state_sections(s)) {
        CPD_CUDA(cudaMemcpyAsync(sec.first, src, sec.second, cudaMemcpyHostToDevice, s->stream));
        src += sec.second;
    }
    // Derived device state: the FP32 split of u, and the contact list, which
    // was built on x + u_neigh (with the 1e-14 tolerance of the set-up build
    // when no rebuild had happened yet).
    if (use_mixed(s) && s->mixed.u2)
        s->launches += launch_split_u(view(s), s->md, s->mixed, s->stream);
    if (has_contact(s)) {
        const double cutoff = 2.0 * s->md.radius + s->md.radius_extend + (h.rebuilds == 0 ? 1e-14 : 0.0);
        std::string err;
        const int l = build_neighbor_list(s->x, s->u_neigh, s->n, s->npad, s->frozen, cutoff,
                                          s->perm, false, s->contact, s->stream, err);
        if (l < 0) return set_error(CPD_ERR_CUDA, "contact neighbour build: " + err);
        s->launches += l;
    }
    s->steps_since_rebuild = h.steps_since_rebuild;
    s->rebuilds = h.rebuilds;
    s->max_disp = h.max_disp;
    s->stress_ready = false;
    CPD_CUDA(cudaStreamSynchronize(s->stream));
    return CPD_OK;
}

double cpd_max_displacement(const cpd_system* s) { return s ? s->max_disp : 0.0; }
int64_t cpd_contact_rebuilds(const cpd_system* s) { return s ? s->rebuilds : 0; }

cpd_status cpd_device_field(cpd_system* s, int32_t field, void** ptr, int64_t* stride)
{
    CPD_OK_OR_RETURN(check_ready(s, false));
    if (!ptr) return set_error(CPD_ERR_INVALID_ARGUMENT, "null output");
    void* p = nullptr;
    switch (field) {
    case CPD_FIELD_X: p = s->x; break;
    case CPD_FIELD_U: p = s->u; break;
    case CPD_FIELD_V: p = s->v; break;
    case CPD_FIELD_F: p = s->f; break;
    case CPD_FIELD_VOL: p = s->vol; break;
    case CPD_FIELD_RHO: p = s->rho; break;
    case CPD_FIELD_M: p = s->m; break;
    case CPD_FIELD_THETA: p = s->theta; break;
    case CPD_FIELD_W: p = s->W; break;
    case CPD_FIELD_PHI: p = s->phi; break;
    case CPD_FIELD_RADIUS: p = s->radius; break;
    case CPD_FIELD_STRESS:
        if (!s->stress)
            return set_error(CPD_ERR_STATE, "stress: call cpd_compute_stress first");
        p = s->stress;
        break;
    default: return set_error(CPD_ERR_INVALID_ARGUMENT, "unknown field");
    }
    *ptr = p;
    if (stride) *stride = s->npad;
    return CPD_OK;
}

cpd_status cpd_bond_bits(cpd_system* s, void** bits, int32_t* words, int64_t* stride)
{
    if (!s || !bits) return set_error(CPD_ERR_INVALID_ARGUMENT, "null argument");
    CPD_OK_OR_RETURN(check_ready(s, true));
    *bits = s->md.fracture ? s->pd.mu : nullptr;
    if (words) *words = s->md.fracture ? s->pd.nwords : 0;
    if (stride) *stride = s->npad;
    return CPD_OK;
}

cpd_status cpd_set_kernel_timing(cpd_system* s, int32_t enable)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    CPD_OK_OR_RETURN(harvest_timing(s));
    s->timing = enable != 0;
    s->timed_ms = 0.0;
    s->timed_launches = 0;
    return CPD_OK;
}

cpd_status cpd_kernel_time(cpd_system* s, double* total_ms, int64_t* launches,
                           double* bytes_per_launch)
{
    if (!s) return set_error(CPD_ERR_INVALID_ARGUMENT, "null system");
    CPD_OK_OR_RETURN(harvest_timing(s));
    if (total_ms) *total_ms = s->timed_ms;
    if (launches) *launches = s->timed_launches;
    if (bytes_per_launch) {
        // Compulsory traffic of one plain-FP64 bond-kernel launch (the same
        // denominator for every precision mode, so fractions compare the
        // modes on the same work) in a step of cpd_step: per row, read x, u
        // (48 B), vol (8 B), count (4 B), write f (24 B); per bond the 4-byte
        // neighbour index; with fracture the 1-bit bond state read and
        // written (0.25 B) and the 1-byte no-fail flag per row; LPS adds the
        // two per-particle coefficient arrays (16 B). Neighbour gathers are
        // counted once (ideal reuse).
        const NeighborList& nl = has_pd(s) ? s->pd : s->contact;
        const double rows = (double)(s->n - s->frozen);
        double per_row = 48.0 + 8.0 + 4.0 + 24.0;
        double per_bond = 4.0;
        if (has_pd(s) && s->md.fracture) {
            per_row += 1.0;
            per_bond += 0.25;
        }
        if (is_lps(s)) per_row += 16.0;
        if (!has_pd(s)) per_row += 24.0 + 16.0;  // Hertz: v, rho (+vol already)
        // The fused step's bond kernel also integrates: read v and rho,
        // write v and the next u (48 + 8 + 24 + 24 B) instead of writing f.
        if (fused_ready(s)) per_row += 48.0 + 8.0 + 24.0 + 24.0 - 24.0;
        *bytes_per_launch = per_row * rows + per_bond * (double)nl.total;
    }
    return CPD_OK;
}

int64_t cpd_kernel_launches(const cpd_system* s) { return s ? s->launches : 0; }

cpd_status cpd_device_bytes(const cpd_system* s, uint64_t* bytes)
{
    if (!s || !bytes) return set_error(CPD_ERR_INVALID_ARGUMENT, "null argument");
    const uint64_t np = (uint64_t)s->npad, n = (uint64_t)s->n;
    uint64_t b = 0;
    if (s->x) {
        b += 5 * 24 * np + 9 * 8 * np + np;  // vectors, scalars, nofail
        b += 24 * n + 64 + 8 * (uint64_t)s->red_cap;  // staging, reduction
        if (s->perm) b += 4 * n;
    }
    for (const auto& bc : s->bcs) b += (uint64_t)bc.count * (bc.values ? 12 : 4);
    if (s->u_alt) b += 24 * np;
    if (s->stress) b += 72 * np + 72 * std::max<uint64_t>(n, 1);
    if (s->u2_alt) b += sizeof(MixedU) * (np + 2 * (uint64_t)s->mixed.guard);
    if (s->bc_bits) b += 4 * ((np + 31) / 32) + 29 * (uint64_t)s->nbc;
    b += s->pd.bytes + s->contact.bytes + s->mixed.bytes;
    *bytes = b;
    return CPD_OK;
}

}  // extern "C"

// ===========================================================================
// Energy and damage without any device allocation.
//
// cpd_compute_energy lazily cudaMallocs its reduction scratch on first use.
// Some callers cannot allow that: a job server that reserves each
// simulation's device memory when it admits the job and must never allocate
// while jobs are running (an allocation mid-run can fail under the budget or
// fragment the pool), or a host framework that owns all device memory
// through its own allocator and forbids raw cudaMalloc. For them this entry
// point keeps its scratch -- one pair of partial sums per 256-row block -- in
// the file-scope array below, which exists on every GPU that loads this
// library until the process exits.
namespace {

constexpr int kNoAllocMaxBlocks = 16384;  // 256-row blocks: 4,194,304 rows
static __device__ __align__(256) double g_noalloc_scratch[2 * kNoAllocMaxBlocks];

constexpr int kMaxDevices = 64;
// Several host threads (the job server's set-up threads, or a caller's own)
// may make the first call on a device at the same time, so each entry is an
// atomic: every thread that finds it empty looks the address up and stores
// the same value.
std::atomic<double*> g_noalloc_ptr[kMaxDevices] = {};

// Host code may not use g_noalloc_scratch's name as a device address; the
// address is fetched once per device, with that device current.
cpd_status noalloc_scratch(int device, double** out)
{
    if (device < 0 || device >= kMaxDevices)
        return set_error(CPD_ERR_UNSUPPORTED, "device ordinal above the no-allocation table");
    double* ptr = g_noalloc_ptr[device].load(std::memory_order_acquire);
    if (!ptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return set_error(CPD_ERR_CUDA, std::string("cudaGetSymbolAddress(no-allocation "
                                                       "scratch): ") +
                                               cudaGetErrorString(e));
        ptr = static_cast<double*>(p);
        g_noalloc_ptr[device].store(ptr, std::memory_order_release);
    }
    *out = ptr;
    return CPD_OK;
}

}  // namespace

extern "C" cpd_status cpd_compute_energy_noalloc(cpd_system* s, double* W_out,
                                                 double* phi_out, double* totals_out)
{
    CPD_OK_OR_RETURN(check_ready(s, true));
    if (!W_out || !phi_out || !totals_out)
        return set_error(CPD_ERR_INVALID_ARGUMENT,
                         "cpd_compute_energy_noalloc: W, phi and totals must be device pointers");
    const int64_t rows = s->n - s->frozen;
    const int nb = energy_blocks(rows);
    if (nb > kNoAllocMaxBlocks)
        return set_error(CPD_ERR_INVALID_ARGUMENT,
                         "cpd_compute_energy_noalloc: " + std::to_string(rows) +
                             " particle rows exceed the no-allocation scratch limit of " +
                             std::to_string((int64_t)kNoAllocMaxBlocks * 256) + " rows");
    CPD_CUDA(cudaSetDevice(s->device));
    double* scratch = nullptr;
    CPD_OK_OR_RETURN(noalloc_scratch(s->device, &scratch));
    if (!has_pd(s)) {
        // A DEM-only system has no strain energy or damage (cpd_compute_energy
        // returns zeros as well): every row of both buffers is zero.
        CPD_CUDA(cudaMemsetAsync(W_out, 0, sizeof(double) * (size_t)s->npad, s->stream));
        CPD_CUDA(cudaMemsetAsync(phi_out, 0, sizeof(double) * (size_t)s->npad, s->stream));
        CPD_CUDA(cudaMemsetAsync(totals_out, 0, 2 * sizeof(double), s->stream));
        return CPD_OK;
    }
    // The energy kernels write rows [frozen, n); frozen rows read 0, as in
    // cpd_compute_energy.
    if (s->frozen > 0) {
        CPD_CUDA(cudaMemsetAsync(W_out, 0, sizeof(double) * (size_t)s->frozen, s->stream));
        CPD_CUDA(cudaMemsetAsync(phi_out, 0, sizeof(double) * (size_t)s->frozen, s->stream));
    }
    ParticleView p = view(s);
    p.W = W_out;
    p.phi = phi_out;
    // Every partial slot the sum reads is written by this launch first, so
    // nothing left in the scratch by an earlier call reaches the result.
    const int prows = launch_energy(s, p, scratch, nb, kNoAllocMaxBlocks);
    CPD_CUDA(cudaGetLastError());
    CPD_LAUNCHED(launch_sum_partials(scratch, prows, 2, totals_out, s->stream));
    return CPD_OK;
}
