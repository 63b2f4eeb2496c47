// Job server: continuous batching of independent simulations on one GPU.
//
// No counterpart in the reference, which runs one simulation per process.
// A job is a host-side description (the same calls that set up a cpd_system:
// particles, state, pre-notches, boundary conditions, step count). The server
// runs two threads:
//   workers  -- (setup_threads of them) admit queued jobs in arrival order
//               while the device bytes of
//               the resident jobs stay within the budget (builds the job's
//               system on its own stream, captures its k-step chunk as a
//               CUDA graph), and retires finished jobs (energy, result
//               fields to the host, frees the system);
//   launcher -- keeps up to two k-step chunks of every resident job in
//               flight on the job's stream and notices completed chunks by
//               event queries.
// Resident jobs advance concurrently: their kernels share the SMs through the
// hardware scheduler, and jobs with less work run on higher-priority streams
// so they are not queued behind large ones. Device memory comes from the
// library's stream-ordered pool, so admitting or retiring a job does not
// synchronise the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cpd_internal.cuh"

namespace {

cpd_status fail(cpd_status code, const std::string& msg)
{
    cpd::set_last_error(msg);
    return code;
}

struct Notch {
    int32_t count = 0;
    std::vector<double> v1, v2, p0;
};
struct JobBC {
    int32_t kind = 0, component = 0;
    std::vector<int64_t> idx;
    std::vector<double> values;
};

}  // namespace

struct cpd_job {
    cpd_params params{};
    int32_t steps = 0;
    int64_t n = 0, frozen = 0;
    std::vector<double> x, vol, rho, radius, u, v;
    std::vector<int32_t> nofail;
    std::vector<Notch> notches;
    std::vector<JobBC> bcs;
    uint32_t keep = 1u << CPD_FIELD_U;
};

namespace {

constexpr int kInflight = 2;

struct Chunk {
    cudaEvent_t ev = nullptr;
    int32_t steps = 0;
};

// Fields written by the launcher thread and read by status queries are
// atomics; the rest change only under the server mutex or while one thread
// owns the job (worker during set-up and retirement, launcher in between).
struct Job {
    int64_t id = 0;
    std::unique_ptr<cpd_job> spec;
    uint32_t keep = 0;
    int32_t state = CPD_JOB_QUEUED;
    std::string error;
    int32_t steps = 0, steps_launched = 0;
    std::atomic<int32_t> steps_done{0};
    int64_t n = 0, bonds = 0;
    uint64_t est_bytes = 0, bytes = 0;
    int32_t priority = 0;
    double t_submit = 0, t_admit = 0, t_ready = 0, t_finish = 0;
    std::atomic<double> t_start{-1.0};
    double W = 0, D = 0;
    bool contact = false;
    bool batched = false;  // advanced in a batch group (small PD job)
    cpd_system* sys = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int32_t graph_steps = 0;
    int64_t graph_nodes = 0;
    std::atomic<int64_t> launches{0};  // kernels run (direct + graph replays x nodes)
    int64_t captured = 0;  // launches counted by the library during capture
    std::deque<Chunk> inflight;
    std::vector<cudaEvent_t> spare;
    std::map<int32_t, std::vector<double>> results;
    // Eviction: requested (the launcher stops issuing chunks and hands the
    // job to a worker once its chunks are done), and the host snapshot of
    // the evolving state it resumes from when set up again.
    std::atomic<bool> evict_request{false};
    int32_t evictions = 0;
    std::vector<uint8_t> snapshot;
};

// A batch group: small jobs advanced together by one cpd_batch (one
// persistent-block launch per step for all of them). Chunks complete in
// order; each records how many steps every job took in it.
struct GroupChunk {
    cudaEvent_t ev = nullptr;
    std::vector<int32_t> steps;
};
struct Group {
    cpd_batch* batch = nullptr;
    std::vector<Job*> jobs;
    std::vector<int32_t> left;       // steps not yet launched, per job
    std::vector<char> done;          // finished and handed back
    std::deque<GroupChunk> inflight;
    std::vector<cudaEvent_t> spare;
};

bool vector_field(int32_t f)
{
    return f == CPD_FIELD_X || f == CPD_FIELD_U || f == CPD_FIELD_V || f == CPD_FIELD_F;
}

// Device bytes a job will hold, estimated before its neighbour list exists:
// the particle arrays, plus a padded neighbour list whose width is 1.2x the
// number of lattice neighbours within the horizon at the job's mean particle
// volume (the library pads every row to the widest one), plus the
// mixed-precision copies where they apply. Replaced by the exact figure
// (cpd_device_bytes) once the job is set up.
uint64_t estimate_bytes(const cpd_job& j)
{
    const double np = std::ceil(std::max<double>(j.n, 1) / 128.0) * 128.0;
    double mean_vol = 0.0;
    for (double a : j.vol) mean_vol += a;
    mean_vol = j.vol.empty() ? 1.0 : mean_vol / (double)j.vol.size();
    double b = (5 * 24 + 9 * 8 + 1) * np + 24.0 * j.n + 4096.0;
    auto neighbours = [&](double radius) {
        if (!(mean_vol > 0)) return std::min<double>(j.n, 256.0);
        const double k = 1.2 * 4.0 / 3.0 * 3.14159265358979323846 * radius * radius * radius /
                             mean_vol + 8.0;
        return std::min<double>(k, (double)j.n);
    };
    if (j.params.pd_model != CPD_PD_NONE) {
        const double w = neighbours(j.params.horizon);
        b += 4.0 * np * (1.0 + w);
        if (j.params.fracture) b += 4.0 * np * std::ceil(w / 32.0);
        if (j.params.precision == CPD_MIXED && j.params.pd_model == CPD_PD_PMB &&
            j.params.contact_model == CPD_CONTACT_NONE)
            b += 64.0 * np + w * np + 4.0 * np * std::ceil(w / 32.0) + 16384.0;
    }
    if (j.params.contact_model != CPD_CONTACT_NONE) {
        const double w = neighbours(2.0 * j.params.contact_radius + j.params.radius_extend);
        b += 4.0 * np * (1.0 + 1.5 * w);
    }
    for (const auto& bc : j.bcs) b += 12.0 * bc.idx.size();
    return (uint64_t)(1.1 * b);
}

}  // namespace

struct cpd_server {
    cpd_server_config cfg{};
    std::chrono::steady_clock::time_point t0;
    int prio_least = 0, prio_greatest = 0;

    std::mutex mu;
    std::condition_variable cv_worker, cv_launcher, cv_done;
    bool stopping = false;
    bool accepting = true;
    int64_t next_id = 1;
    std::map<int64_t, std::unique_ptr<Job>> jobs;
    std::deque<Job*> queue;     // submitted, not admitted
    std::vector<Job*> admitted; // set up, not yet picked by the launcher
    std::vector<Job*> pending_batch;  // set up small jobs for the next batch group
    std::vector<Job*> retire;   // all steps done, not yet finalised
    std::vector<Job*> evicting; // chunks drained, to be saved and freed
    int evictions_pending = 0;
    int64_t resident = 0;
    uint64_t resident_bytes = 0, peak_bytes = 0;
    int64_t n_submitted = 0, n_done = 0, n_failed = 0, launches = 0;
    double bond_updates = 0;

    std::vector<std::thread> workers;
    std::thread launcher;

    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }

    // ---- worker thread ----------------------------------------------------
    void finish_failed(Job* j, const std::string& msg)
    {
        // Caller holds mu.
        j->state = CPD_JOB_FAILED;
        j->error = msg;
        j->t_finish = now();
        j->spec.reset();
        n_failed++;
        cv_done.notify_all();
    }

    void release_device(Job* j)
    {
        for (auto& c : j->inflight) cudaEventDestroy(c.ev);
        j->inflight.clear();
        for (cudaEvent_t e : j->spare) cudaEventDestroy(e);
        j->spare.clear();
        if (j->graph) cudaGraphExecDestroy(j->graph);
        j->graph = nullptr;
        if (j->sys) cpd_system_destroy(j->sys);
        j->sys = nullptr;
        if (j->stream) cudaStreamDestroy(j->stream);
        j->stream = nullptr;
    }

    int32_t priority_for(const cpd_job& s) const
    {
        // log10(particles x steps) from 5 (tiny) to 11 (largest jobs) spread
        // over the device's priority levels; less work, higher priority.
        const double w = std::log10(std::max(1.0, (double)s.n * std::max(1, s.steps)));
        const double t = std::min(1.0, std::max(0.0, (w - 5.0) / 6.0));
        return prio_greatest + (int32_t)std::lround(t * (prio_least - prio_greatest));
    }

    // Small peridynamic jobs without contact, in the throughput precisions,
    // go to batch groups (cfg.batch_max_particles > 0).
    bool batchable(const cpd_job& s) const
    {
        const int32_t pd = s.params.pd_model;
        return cfg.batch_max_particles > 0 && s.n <= cfg.batch_max_particles &&
               s.steps > 0 && (pd == CPD_PD_PMB || pd == CPD_PD_LPS) &&
               s.params.contact_model == CPD_CONTACT_NONE &&
               (s.params.precision == CPD_FP64 || s.params.precision == CPD_MIXED);
    }

    // Builds the job's system. Returns an empty string on success.
    std::string setup(Job* j)
    {
        const cpd_job& s = *j->spec;
        auto lib_error = [&](const char* what) { return std::string(what) + ": " + cpd_last_error(); };
        j->priority = priority_for(s);
        j->keep = s.keep;
        if (cudaStreamCreateWithPriority(&j->stream, cudaStreamNonBlocking, j->priority) !=
            cudaSuccess)
            return "stream creation failed";
        cpd_params p = s.params;
        p.device = cfg.device;
        if (cpd_system_create(&p, &j->sys) != CPD_OK) return lib_error("cpd_system_create");
        if (cpd_set_stream(j->sys, j->stream) != CPD_OK) return lib_error("cpd_set_stream");
        if (cpd_upload_particles(j->sys, s.n, s.frozen, s.x.data(), s.vol.data(),
                                 s.rho.empty() ? nullptr : s.rho.data(),
                                 s.nofail.empty() ? nullptr : s.nofail.data(),
                                 s.radius.empty() ? nullptr : s.radius.data()) != CPD_OK)
            return lib_error("cpd_upload_particles");
        if ((!s.u.empty() || !s.v.empty()) &&
            cpd_set_state(j->sys, s.u.empty() ? nullptr : s.u.data(),
                          s.v.empty() ? nullptr : s.v.data()) != CPD_OK)
            return lib_error("cpd_set_state");
        if (cpd_build_neighbors(j->sys) != CPD_OK) return lib_error("cpd_build_neighbors");
        for (const auto& nt : s.notches)
            if (cpd_prenotch(j->sys, nt.count, nt.v1.data(), nt.v2.data(), nt.p0.data()) != CPD_OK)
                return lib_error("cpd_prenotch");
        for (const auto& bc : s.bcs)
            if (cpd_add_boundary_condition(j->sys, bc.kind, bc.component, (int64_t)bc.idx.size(),
                                           bc.idx.data(), bc.values.data()) != CPD_OK)
                return lib_error("cpd_add_boundary_condition");
        if (cpd_init(j->sys) != CPD_OK) return lib_error("cpd_init");
        // A kept stress is computed at the end; computing it once here (as
        // the reference does at init) allocates its arrays before the job's
        // device bytes are measured.
        if ((j->keep >> CPD_FIELD_STRESS) & 1u)
            if (cpd_compute_stress(j->sys) != CPD_OK) return lib_error("cpd_compute_stress");
        int32_t max_n = 0;
        cpd_neighbor_stats(j->sys, &max_n, &j->bonds);
        j->contact = s.params.contact_model != CPD_CONTACT_NONE;
        j->batched = batchable(s);
        // Contact systems decide neighbour rebuilds on the host between
        // steps, so only the PD-only step is captured; batched jobs run in
        // their group's graphs.
        const int32_t k = std::min(cfg.steps_per_launch, j->steps);
        if (cfg.use_graphs && !j->contact && !j->batched && k > 0) {
            const int64_t before = cpd_kernel_launches(j->sys);
            cudaGraph_t g = nullptr;
            bool ok = cudaStreamBeginCapture(j->stream, cudaStreamCaptureModeThreadLocal) ==
                      cudaSuccess;
            cpd_status st = ok ? cpd_step(j->sys, k) : CPD_ERR_CUDA;
            if (ok) ok = cudaStreamEndCapture(j->stream, &g) == cudaSuccess && st == CPD_OK;
            if (ok) ok = cudaGraphInstantiate(&j->graph, g, 0) == cudaSuccess;
            size_t nodes = 0;
            if (ok) ok = cudaGraphGetNodes(g, nullptr, &nodes) == cudaSuccess;
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            if (ok) {
                j->graph_steps = k;
                j->graph_nodes = (int64_t)nodes;
            } else {
                if (j->graph) cudaGraphExecDestroy(j->graph);
                j->graph = nullptr;
            }
            j->captured = cpd_kernel_launches(j->sys) - before;
        }
        for (int e = 0; e < kInflight; e++) {
            cudaEvent_t ev;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
                return "event creation failed";
            j->spare.push_back(ev);
        }
        // A resumed job continues from its snapshot (the state it was evicted
        // with), bit-identical to an uninterrupted run.
        if (!j->snapshot.empty()) {
            if (cpd_load_state(j->sys, j->snapshot.data(), (uint64_t)j->snapshot.size()) != CPD_OK)
                return lib_error("cpd_load_state");
            std::vector<uint8_t>().swap(j->snapshot);
        }
        cpd_device_bytes(j->sys, &j->bytes);
        // The host copy of the input stays for jobs that may be evicted (a
        // resumed job is set up again from it).
        if (j->batched) j->spec.reset();
        return std::string();
    }

    // Saves an evicted job's state to the host, frees its device memory and
    // queues it again right behind the queue's head (the job it made room
    // for). Caller holds no lock.
    void evict(Job* j)
    {
        std::string err;
        uint64_t bytes = 0;
        std::vector<uint8_t> snap;
        if (cpd_state_bytes(j->sys, &bytes) != CPD_OK)
            err = std::string("cpd_state_bytes: ") + cpd_last_error();
        if (err.empty()) {
            snap.resize((size_t)bytes);
            if (cpd_save_state(j->sys, snap.data(), bytes) != CPD_OK)
                err = std::string("cpd_save_state: ") + cpd_last_error();
        }
        const int64_t direct = j->sys ? cpd_kernel_launches(j->sys) - j->captured : 0;
        release_device(j);
        std::lock_guard<std::mutex> lk(mu);
        evictions_pending--;
        resident--;
        resident_bytes -= std::max(j->bytes, j->est_bytes);
        j->launches += direct;
        j->evict_request = false;
        if (!err.empty()) {
            finish_failed(j, err);
            return;
        }
        j->snapshot.swap(snap);
        j->evictions++;
        j->state = CPD_JOB_QUEUED;
        j->captured = 0;
        j->inflight.clear();
        queue.insert(queue.empty() ? queue.end() : queue.begin() + 1, j);
        cv_worker.notify_all();
    }

    // Automatic eviction (cfg.evict_after_s > 0): when the queue's head has
    // waited that long for memory, the resident job with the most work left
    // (particles x steps, larger than the head's, never evicted before) is
    // asked to make room. One eviction at a time. Caller holds mu.
    void consider_eviction()
    {
        if (cfg.evict_after_s <= 0.0 || evictions_pending > 0 || queue.empty()) return;
        Job* head = queue.front();
        if (head->est_bytes > cfg.hbm_budget_bytes || resident == 0 ||
            resident_bytes + head->est_bytes <= cfg.hbm_budget_bytes)
            return;
        if (now() - head->t_submit < cfg.evict_after_s) return;
        const double head_work = (double)head->n * std::max(1, head->steps);
        Job* victim = nullptr;
        double most = head_work;
        for (auto& kv : jobs) {
            Job* j = kv.second.get();
            if (j->state != CPD_JOB_RUNNING || j->batched || j->evictions > 0 ||
                j->evict_request || !j->spec)
                continue;
            const double left = (double)j->n * std::max(0, j->steps - j->steps_done.load());
            if (left > most) {
                most = left;
                victim = j;
            }
        }
        if (victim) {
            victim->evict_request = true;
            evictions_pending++;
        }
    }

    void finalize(Job* j)
    {
        std::string err;
        double W = 0, D = 0;
        if (cpd_compute_energy(j->sys, &W, &D) != CPD_OK)
            err = std::string("cpd_compute_energy: ") + cpd_last_error();
        if (err.empty() && ((j->keep >> CPD_FIELD_STRESS) & 1u) &&
            cpd_compute_stress(j->sys) != CPD_OK)
            err = std::string("cpd_compute_stress: ") + cpd_last_error();
        std::map<int32_t, std::vector<double>> results;
        for (int32_t f = 0; f <= CPD_FIELD_STRESS && err.empty(); f++) {
            if (!(j->keep & (1u << f))) continue;
            const size_t comps = f == CPD_FIELD_STRESS ? 9 : (vector_field(f) ? 3 : 1);
            std::vector<double> buf(comps * (size_t)j->n);
            if (cpd_download(j->sys, f, buf.data()) != CPD_OK)
                err = std::string("cpd_download: ") + cpd_last_error();
            results[f].swap(buf);
        }
        const int64_t direct = cpd_kernel_launches(j->sys) - j->captured;
        release_device(j);
        std::lock_guard<std::mutex> lk(mu);
        resident--;
        resident_bytes -= std::max(j->bytes, j->est_bytes);
        j->launches += direct;
        launches += j->launches;
        if (!err.empty()) {
            finish_failed(j, err);
            return;
        }
        j->W = W;
        j->D = D;
        j->results.swap(results);
        j->spec.reset();
        j->state = CPD_JOB_DONE;
        j->t_finish = now();
        bond_updates += (double)j->bonds * j->steps;
        n_done++;
        cv_done.notify_all();
    }

    // Whether the head of the queue can be admitted (or must be failed as
    // too large) now. Caller holds mu.
    bool admissible() const
    {
        if (queue.empty() || resident >= cfg.max_active) return false;
        const uint64_t b = queue.front()->est_bytes;
        return b > cfg.hbm_budget_bytes || resident == 0 ||
               resident_bytes + b <= cfg.hbm_budget_bytes;
    }

    void worker_loop()
    {
        cudaSetDevice(cfg.device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv_worker.wait_for(lk, std::chrono::milliseconds(50), [&] {
                return (stopping && resident == 0) || !retire.empty() || !evicting.empty() ||
                       admissible() || (!accepting && !queue.empty());
            });
            if (!evicting.empty()) {
                std::vector<Job*> out;
                out.swap(evicting);
                lk.unlock();
                for (Job* j : out) evict(j);
                lk.lock();
                continue;
            }
            if (accepting && !stopping) consider_eviction();
            if (!retire.empty()) {
                std::vector<Job*> done;
                done.swap(retire);
                lk.unlock();
                for (Job* j : done) finalize(j);
                lk.lock();
                continue;  // retire everything finished before admitting
            }
            if (!accepting) {
                while (!queue.empty()) {
                    finish_failed(queue.front(), "server shut down before admission");
                    queue.pop_front();
                }
            }
            if (stopping && resident == 0 && queue.empty()) break;
            while (accepting && admissible()) {
                Job* j = queue.front();
                queue.pop_front();
                if (j->est_bytes > cfg.hbm_budget_bytes) {
                    finish_failed(j, "job needs about " + std::to_string(j->est_bytes) +
                                         " device bytes, more than the budget");
                    continue;
                }
                resident++;
                resident_bytes += j->est_bytes;
                j->t_admit = now();
                lk.unlock();
                const std::string err = setup(j);
                lk.lock();
                if (!err.empty()) {
                    lk.unlock();
                    release_device(j);
                    lk.lock();
                    resident--;
                    resident_bytes -= j->est_bytes;
                    finish_failed(j, err);
                    continue;
                }
                resident_bytes += std::max(j->bytes, j->est_bytes) - j->est_bytes;
                peak_bytes = std::max(peak_bytes, resident_bytes);
                j->state = CPD_JOB_RUNNING;
                j->t_ready = now();
                if (j->batched)
                    pending_batch.push_back(j);
                else
                    admitted.push_back(j);
                cv_launcher.notify_one();
                // Retire finished jobs before setting up the next one.
                if (!retire.empty()) break;
            }
        }
    }

    // ---- launcher thread --------------------------------------------------
    // Returns false if the job failed.
    bool launch_chunk(Job* j)
    {
        const int32_t left = j->steps - j->steps_launched;
        const bool replay = j->graph && left >= j->graph_steps;
        const int32_t k = replay ? j->graph_steps : std::min(left, cfg.steps_per_launch);
        if (replay) {
            if (cudaGraphLaunch(j->graph, j->stream) != cudaSuccess) {
                j->error = "cudaGraphLaunch failed";
                return false;
            }
            j->launches += j->graph_nodes;
        } else if (cpd_step(j->sys, k) != CPD_OK) {
            j->error = std::string("cpd_step: ") + cpd_last_error();
            return false;
        }
        Chunk c;
        c.ev = j->spare.back();
        j->spare.pop_back();
        c.steps = k;
        if (cudaEventRecord(c.ev, j->stream) != cudaSuccess) {
            j->spare.push_back(c.ev);
            j->error = "cudaEventRecord failed";
            return false;
        }
        j->inflight.push_back(c);
        j->steps_launched += k;
        return true;
    }

    // ---- batch groups (launcher thread) -----------------------------------
    // A group of the pending small jobs; a job the batch refuses (e.g. its
    // boundary conditions do not fit the fused step) runs on its own.
    void form_group(const std::vector<Job*>& jobs, std::vector<Group*>& groups,
                    std::vector<Job*>& running)
    {
        std::vector<cpd_system*> sys;
        std::vector<int32_t> steps;
        for (Job* j : jobs) {
            sys.push_back(j->sys);
            steps.push_back(j->steps);
        }
        cpd_batch* b = nullptr;
        if (cpd_batch_create(sys.data(), (int32_t)sys.size(), steps.data(), &b) != CPD_OK) {
            if (jobs.size() > 1) {
                for (Job* j : jobs) form_group({j}, groups, running);
            } else {
                jobs[0]->batched = false;
                running.push_back(jobs[0]);
            }
            return;
        }
        auto g = std::make_unique<Group>();
        g->batch = b;
        g->jobs = jobs;
        g->left = steps;
        g->done.assign(jobs.size(), 0);
        for (int e = 0; e < kInflight; e++) {
            cudaEvent_t ev = nullptr;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess)
                g->spare.push_back(ev);
        }
        groups.push_back(g.release());
    }

    // Completed chunks (finished jobs are handed back by the batch and go to
    // `finished`) and new chunks, up to kInflight. False on a device or
    // launch error.
    bool service_group(Group* g, bool& progressed, std::vector<Job*>& finished, std::string& err)
    {
        while (!g->inflight.empty()) {
            const cudaError_t q = cudaEventQuery(g->inflight.front().ev);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) {
                err = std::string("device error: ") + cudaGetErrorString(q);
                return false;
            }
            const GroupChunk& c = g->inflight.front();
            for (size_t k = 0; k < g->jobs.size(); ++k) {
                Job* j = g->jobs[k];
                j->steps_done += c.steps[k];
                if (!g->done[k] && j->steps_done == j->steps) {
                    if (cpd_batch_release(g->batch, (int32_t)k) != CPD_OK) {
                        err = std::string("cpd_batch_release: ") + cpd_last_error();
                        return false;
                    }
                    g->done[k] = 1;
                    finished.push_back(j);
                }
            }
            g->spare.push_back(c.ev);
            g->inflight.pop_front();
            progressed = true;
        }
        const bool more = std::any_of(g->left.begin(), g->left.end(), [](int32_t v) { return v > 0; });
        if (more && (int)g->inflight.size() < kInflight && !g->spare.empty()) {
            const int32_t K = cfg.steps_per_launch;
            if (cpd_batch_step(g->batch, K) != CPD_OK) {
                err = std::string("cpd_batch_step: ") + cpd_last_error();
                return false;
            }
            GroupChunk c;
            c.ev = g->spare.back();
            g->spare.pop_back();
            c.steps.resize(g->jobs.size());
            for (size_t k = 0; k < g->jobs.size(); ++k) {
                c.steps[k] = std::min(K, g->left[k]);
                g->left[k] -= c.steps[k];
                Job* j = g->jobs[k];
                j->steps_launched += c.steps[k];
                if (c.steps[k] > 0 && j->t_start < 0) j->t_start = now();
            }
            if (cudaEventRecord(c.ev, cpd::batch_stream(g->batch)) != cudaSuccess) {
                g->spare.push_back(c.ev);
                err = "cudaEventRecord failed";
                return false;
            }
            g->inflight.push_back(std::move(c));
            progressed = true;
        }
        return true;
    }

    // Destroys a group whose jobs all finished, or (failed) fails the rest.
    void close_group(Group* g, const std::string& err)
    {
        const int64_t n = cpd_batch_launches(g->batch);
        cpd_batch_destroy(g->batch);
        for (auto& c : g->inflight) cudaEventDestroy(c.ev);
        for (cudaEvent_t e : g->spare) cudaEventDestroy(e);
        std::vector<Job*> failed;
        for (size_t k = 0; k < g->jobs.size(); ++k)
            if (!g->done[k]) failed.push_back(g->jobs[k]);
        for (Job* j : failed) {
            if (j->stream) cudaStreamSynchronize(j->stream);
            release_device(j);
        }
        std::lock_guard<std::mutex> lk(mu);
        launches += n;
        for (Job* j : failed) {
            resident--;
            resident_bytes -= std::max(j->bytes, j->est_bytes);
            finish_failed(j, err.empty() ? std::string("batch group failed") : err);
        }
        delete g;
    }

    void launcher_loop()
    {
        cudaSetDevice(cfg.device);
        std::vector<Job*> running;
        std::vector<Group*> groups;
        for (;;) {
            std::vector<Job*> grouping;
            {
                std::unique_lock<std::mutex> lk(mu);
                if (running.empty() && groups.empty())
                    cv_launcher.wait_for(lk, std::chrono::milliseconds(2), [&] {
                        return stopping || !admitted.empty() || !pending_batch.empty();
                    });
                for (Job* j : admitted) running.push_back(j);
                admitted.clear();
                grouping.swap(pending_batch);
                if (stopping && running.empty() && groups.empty() && grouping.empty() &&
                    resident == 0 && queue.empty() && admitted.empty())
                    break;
            }
            if (!grouping.empty()) form_group(grouping, groups, running);
            bool progressed = false;
            std::vector<Job*> finished, failed;
            for (auto it = groups.begin(); it != groups.end();) {
                Group* g = *it;
                std::string err;
                const bool ok = service_group(g, progressed, finished, err);
                const bool all = std::all_of(g->done.begin(), g->done.end(),
                                             [](char d) { return d != 0; });
                if (!ok || all) {
                    if (!finished.empty()) {
                        // Hand the finished jobs to the workers before the
                        // group's batch goes.
                        std::lock_guard<std::mutex> lk(mu);
                        for (Job* j : finished) retire.push_back(j);
                        finished.clear();
                        cv_worker.notify_one();
                    }
                    close_group(g, ok ? std::string() : err);
                    it = groups.erase(it);
                } else {
                    ++it;
                }
            }
            for (auto it = running.begin(); it != running.end();) {
                Job* j = *it;
                bool bad = false;
                while (!j->inflight.empty()) {
                    const cudaError_t q = cudaEventQuery(j->inflight.front().ev);
                    if (q == cudaErrorNotReady) break;
                    if (q != cudaSuccess) {
                        j->error = std::string("device error: ") + cudaGetErrorString(q);
                        bad = true;
                        break;
                    }
                    j->steps_done += j->inflight.front().steps;
                    j->spare.push_back(j->inflight.front().ev);
                    j->inflight.pop_front();
                    progressed = true;
                }
                const bool evicting_now = j->evict_request.load();
                while (!bad && !evicting_now && j->steps_launched < j->steps &&
                       (int)j->inflight.size() < kInflight) {
                    if (j->t_start < 0) j->t_start = now();
                    if (!launch_chunk(j)) bad = true;
                    progressed = true;
                }
                if (bad) {
                    failed.push_back(j);
                    it = running.erase(it);
                } else if (j->steps_done == j->steps) {
                    if (evicting_now) {
                        // Finished before it could be evicted.
                        j->evict_request = false;
                        std::lock_guard<std::mutex> lk(mu);
                        evictions_pending--;
                    }
                    finished.push_back(j);
                    it = running.erase(it);
                } else if (evicting_now && j->inflight.empty()) {
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        evicting.push_back(j);
                        cv_worker.notify_one();
                    }
                    progressed = true;
                    it = running.erase(it);
                } else {
                    ++it;
                }
            }
            if (!finished.empty() || !failed.empty()) {
                for (Job* j : failed) {
                    if (j->stream) cudaStreamSynchronize(j->stream);
                    release_device(j);
                }
                std::lock_guard<std::mutex> lk(mu);
                for (Job* j : finished) retire.push_back(j);
                for (Job* j : failed) {
                    resident--;
                    resident_bytes -= std::max(j->bytes, j->est_bytes);
                    finish_failed(j, j->error);
                }
                cv_worker.notify_one();
            }
            if (!progressed && (!running.empty() || !groups.empty()))
                std::this_thread::sleep_for(std::chrono::microseconds(20));
        }
    }
};

extern "C" {

cpd_status cpd_job_create(const cpd_params* params, int32_t num_steps, cpd_job** out)
{
    if (!params || !out) return fail(CPD_ERR_INVALID_ARGUMENT, "null argument");
    if (num_steps < 0) return fail(CPD_ERR_INVALID_ARGUMENT, "num_steps < 0");
    auto j = std::make_unique<cpd_job>();
    j->params = *params;
    j->steps = num_steps;
    *out = j.release();
    return CPD_OK;
}

cpd_status cpd_job_destroy(cpd_job* job)
{
    delete job;
    return CPD_OK;
}

cpd_status cpd_job_set_particles(cpd_job* j, int64_t n, int64_t n_frozen, const double* x,
                                 const double* vol, const double* rho, const int32_t* nofail,
                                 const double* radius)
{
    if (!j || n <= 0 || n_frozen < 0 || n_frozen > n || !x || !vol)
        return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_job_set_particles: bad arguments");
    j->n = n;
    j->frozen = n_frozen;
    j->x.assign(x, x + 3 * n);
    j->vol.assign(vol, vol + n);
    if (rho) j->rho.assign(rho, rho + n); else j->rho.clear();
    if (nofail) j->nofail.assign(nofail, nofail + n); else j->nofail.clear();
    if (radius) j->radius.assign(radius, radius + n); else j->radius.clear();
    j->u.clear();
    j->v.clear();
    return CPD_OK;
}

cpd_status cpd_job_set_state(cpd_job* j, const double* u, const double* v)
{
    if (!j || j->n == 0) return fail(CPD_ERR_STATE, "cpd_job_set_state before particles");
    if (u) j->u.assign(u, u + 3 * j->n);
    if (v) j->v.assign(v, v + 3 * j->n);
    return CPD_OK;
}

cpd_status cpd_job_prenotch(cpd_job* j, int32_t count, const double* v1, const double* v2,
                            const double* p0)
{
    if (!j || count < 0 || (count > 0 && (!v1 || !v2 || !p0)))
        return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_job_prenotch: bad arguments");
    Notch nt;
    nt.count = count;
    nt.v1.assign(v1, v1 + 3 * count);
    nt.v2.assign(v2, v2 + 3 * count);
    nt.p0.assign(p0, p0 + 3 * count);
    j->notches.push_back(std::move(nt));
    return CPD_OK;
}

cpd_status cpd_job_add_boundary_condition(cpd_job* j, int32_t kind, int32_t component,
                                          int64_t count, const int64_t* indices,
                                          const double* values)
{
    if (!j || count < 0 || !values || (count > 0 && !indices))
        return fail(CPD_ERR_INVALID_ARGUMENT, "cpd_job_add_boundary_condition: bad arguments");
    JobBC bc;
    bc.kind = kind;
    bc.component = component;
    bc.idx.assign(indices, indices + count);
    bc.values.assign(values, values + (kind == CPD_BC_FORCE_ADD ? count : 1));
    if (bc.values.empty()) bc.values.push_back(0.0);
    j->bcs.push_back(std::move(bc));
    return CPD_OK;
}

cpd_status cpd_job_keep_fields(cpd_job* j, uint32_t mask)
{
    if (!j) return fail(CPD_ERR_INVALID_ARGUMENT, "null job");
    if (mask >> (CPD_FIELD_STRESS + 1)) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown field bit");
    j->keep = mask;
    return CPD_OK;
}

cpd_status cpd_server_create(const cpd_server_config* cfg, cpd_server** out)
{
    if (!cfg || !out) return fail(CPD_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (cfg->max_active < 1 || cfg->steps_per_launch < 1 || cfg->hbm_budget_bytes == 0 ||
        cfg->setup_threads < 0 || cfg->evict_after_s < 0.0)
        return fail(CPD_ERR_INVALID_ARGUMENT,
                    "max_active, steps_per_launch and hbm_budget_bytes must be positive");
    int ndev = 0;
    const cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(CPD_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (cfg->device < 0 || cfg->device >= ndev)
        return fail(CPD_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    auto s = std::make_unique<cpd_server>();
    s->cfg = *cfg;
    s->t0 = std::chrono::steady_clock::now();
    cudaSetDevice(cfg->device);
    cudaDeviceGetStreamPriorityRange(&s->prio_least, &s->prio_greatest);
    if (s->cfg.setup_threads == 0) s->cfg.setup_threads = 4;
    for (int w = 0; w < s->cfg.setup_threads; w++)
        s->workers.emplace_back([p = s.get()] { p->worker_loop(); });
    s->launcher = std::thread([p = s.get()] { p->launcher_loop(); });
    *out = s.release();
    return CPD_OK;
}

cpd_status cpd_server_destroy(cpd_server* s)
{
    if (!s) return CPD_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->accepting = false;
        s->stopping = true;
    }
    s->cv_worker.notify_all();
    s->cv_launcher.notify_all();
    for (auto& w : s->workers) w.join();
    s->launcher.join();
    delete s;
    return CPD_OK;
}

cpd_status cpd_server_submit(cpd_server* s, cpd_job* job, int64_t* job_id)
{
    std::unique_ptr<cpd_job> owned(job);
    if (!s || !job) return fail(CPD_ERR_INVALID_ARGUMENT, "null argument");
    if (owned->n == 0) return fail(CPD_ERR_STATE, "job has no particles");
    auto j = std::make_unique<Job>();
    j->steps = owned->steps;
    j->n = owned->n;
    j->est_bytes = estimate_bytes(*owned);
    j->spec = std::move(owned);
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->accepting) return fail(CPD_ERR_STATE, "server is shutting down");
    j->id = s->next_id++;
    j->t_submit = s->now();
    Job* raw = j.get();
    s->jobs[j->id] = std::move(j);
    s->queue.push_back(raw);
    s->n_submitted++;
    if (job_id) *job_id = raw->id;
    s->cv_worker.notify_one();
    return CPD_OK;
}

double cpd_server_clock(const cpd_server* s) { return s ? s->now() : 0.0; }

cpd_status cpd_server_wait(cpd_server* s, int64_t id, double timeout_s)
{
    if (!s) return fail(CPD_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown job id");
    Job* j = it->second.get();
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        return j->state == CPD_JOB_DONE || j->state == CPD_JOB_FAILED;
    });
    return ok ? CPD_OK : fail(CPD_ERR_STATE, "timed out waiting for the job");
}

cpd_status cpd_server_drain(cpd_server* s, double timeout_s)
{
    if (!s) return fail(CPD_ERR_INVALID_ARGUMENT, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
        return s->n_done + s->n_failed == s->n_submitted;
    });
    return ok ? CPD_OK : fail(CPD_ERR_STATE, "timed out draining the server");
}

cpd_status cpd_server_job_status(cpd_server* s, int64_t id, cpd_job_status* out)
{
    if (!s || !out) return fail(CPD_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown job id");
    const Job& j = *it->second;
    cpd_job_status st{};
    st.state = j.state;
    st.steps = j.steps;
    st.steps_done = j.steps_done;
    st.priority = j.priority;
    st.n = j.n;
    st.bonds = j.bonds;
    st.device_bytes = std::max(j.bytes, j.est_bytes);
    st.submit_time = j.t_submit;
    st.admit_time = j.t_admit;
    st.ready_time = j.t_ready;
    st.start_time = j.t_start;
    st.finish_time = j.t_finish;
    st.total_strain_energy = j.W;
    st.total_damage = j.D;
    st.kernel_launches = j.launches;
    st.evictions = j.evictions;
    *out = st;
    return CPD_OK;
}

cpd_status cpd_server_job_error(cpd_server* s, int64_t id, char* buf, int64_t size)
{
    if (!s || !buf || size <= 0) return fail(CPD_ERR_INVALID_ARGUMENT, "bad arguments");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown job id");
    const std::string& m = it->second->error;
    const size_t k = std::min<size_t>(m.size(), (size_t)size - 1);
    std::memcpy(buf, m.data(), k);
    buf[k] = '\0';
    return CPD_OK;
}

cpd_status cpd_server_download(cpd_server* s, int64_t id, int32_t field, double* host_out)
{
    if (!s || !host_out) return fail(CPD_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown job id");
    const Job& j = *it->second;
    if (j.state != CPD_JOB_DONE) return fail(CPD_ERR_STATE, "job is not done");
    auto r = j.results.find(field);
    if (r == j.results.end()) return fail(CPD_ERR_STATE, "field was not kept for this job");
    std::memcpy(host_out, r->second.data(), sizeof(double) * r->second.size());
    return CPD_OK;
}

cpd_status cpd_server_evict(cpd_server* s, int64_t id)
{
    if (!s) return fail(CPD_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown job id");
    Job* j = it->second.get();
    if (j->state != CPD_JOB_RUNNING || j->batched || !j->spec)
        return fail(CPD_ERR_STATE, "only a running job that is not in a batch group is evicted");
    if (j->evict_request) return CPD_OK;
    j->evict_request = true;
    s->evictions_pending++;
    return CPD_OK;
}

cpd_status cpd_server_release(cpd_server* s, int64_t id)
{
    if (!s) return fail(CPD_ERR_INVALID_ARGUMENT, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if (it == s->jobs.end()) return fail(CPD_ERR_INVALID_ARGUMENT, "unknown job id");
    if (it->second->state != CPD_JOB_DONE && it->second->state != CPD_JOB_FAILED)
        return fail(CPD_ERR_STATE, "job is still queued or running");
    s->jobs.erase(it);
    return CPD_OK;
}

cpd_status cpd_server_stats_get(cpd_server* s, cpd_server_stats* out)
{
    if (!s || !out) return fail(CPD_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    cpd_server_stats st{};
    st.submitted = s->n_submitted;
    st.done = s->n_done;
    st.failed = s->n_failed;
    st.resident = s->resident;
    st.queued = (int64_t)s->queue.size();
    st.resident_bytes = s->resident_bytes;
    st.peak_resident_bytes = s->peak_bytes;
    st.kernel_launches = s->launches;
    st.bond_updates = s->bond_updates;
    *out = st;
    return CPD_OK;
}

}  // extern "C"
