/*
 * cabanapd_b200 — C ABI of the B200-native CabanaPD per-timestep hot path.
 *
 * One opaque handle (cpd_system) owns every device buffer of one simulation:
 * particle fields in structure-of-arrays layout, the padded-ELL neighbour
 * list with 1-bit-per-bond broken-bond masks, the contact list, boundary
 * condition index lists and reduction scratch. Host arrays passed in or out
 * are owned by the caller and are copied; no pointer is retained after a
 * call returns. Calls are synchronous with respect to the host unless they
 * say otherwise; work is issued on the system's CUDA stream.
 *
 * The entry points replace the reference's template interface as follows
 * (paths relative to the CabanaPD source tree):
 *
 *   cpd_system_create        ForceModel(...) constructors
 *                            (force_models/CabanaPD_PMB.hpp:165-231,
 *                             force_models/CabanaPD_LPS.hpp:151-253,
 *                             force_models/CabanaPD_Hertzian.hpp:40-56,
 *                             force_models/CabanaPD_Contact.hpp:70-79),
 *                            VelocityVerlet(dt) (CabanaPD_Integrate.hpp:80-86)
 *   cpd_upload_particles     Particles::create + Particles::update
 *                            (CabanaPD_Particles.hpp:242-307, 429-443)
 *   cpd_set_state            Particles::update of u / v (same lines)
 *   cpd_build_neighbors      Neighbor ctor (CabanaPD_Neighbor.hpp:44-66,
 *                            199-210): full list, cutoff + 1e-14, mu = 1
 *   cpd_neighbor_stats       Neighbor::getStatistics (Neighbor.hpp:80-102)
 *   cpd_bond_bits            Neighbor::brokenBonds (Neighbor.hpp:219), as bits
 *   cpd_prenotch             Prenotch<N>::create (CabanaPD_Prenotch.hpp:215-263)
 *   cpd_add_boundary_condition  createBoundaryCondition / BodyTerm
 *                            (CabanaPD_Boundary.hpp:34-204, CabanaPD_BodyTerm.hpp:25-69)
 *   cpd_compute_weighted_volume / cpd_compute_dilatation / cpd_compute_force /
 *   cpd_compute_energy       Force<...>::computeWeightedVolume /
 *                            computeDilatation / computeForceFull /
 *                            computeEnergyFull and the free functions
 *                            computeForce / computeEnergy (CabanaPD_Force.hpp:176-219)
 *   cpd_compute_stress       computeStress + Force<...>::computeStressFull
 *                            (CabanaPD_Force.hpp:222-235; force/CabanaPD_PMB.hpp:
 *                            157-202, 341-401, 492-537; force/CabanaPD_LPS.hpp:
 *                            221-267, 506-572)
 *   cpd_init                 Solver::init(bc[, prenotch]) (CabanaPD_Solver.hpp:229-297)
 *   cpd_step                 Solver::runStep(step, bc) x num_steps
 *                            (CabanaPD_Solver.hpp:332-375)
 *   cpd_step_energy          runStep x num_steps, then the output step's
 *                            computeEnergy (CabanaPD_Solver.hpp:479-494)
 *   cpd_download             Particles::slice*() + deep_copy to host
 *
 * Entry points without a reference counterpart (each says so where it is
 * declared): cpd_step_stage, cpd_device_field, cpd_set_stream, the kernel
 * timing calls, cpd_compute_energy_noalloc, the state snapshots
 * (cpd_state_bytes / cpd_save_state / cpd_load_state), the batched step
 * (cpd_batch_*) and the job server (cpd_job_*, cpd_server_*).
 *
 * Errors: every call returns a cpd_status; cpd_last_error() gives the
 * message of the last failure on the calling thread. The reference throws
 * std::runtime_error in the same situations (e.g. Solver.hpp:172-174).
 * Handles are not thread-safe: drive one handle from one host thread.
 */
#ifndef CABANAPD_B200_H
#define CABANAPD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CPD_ABI_VERSION 4

typedef struct cpd_system cpd_system;
typedef int32_t cpd_status;

enum {
    CPD_OK = 0,
    CPD_ERR_INVALID_ARGUMENT = 1,
    CPD_ERR_OUT_OF_MEMORY = 2,
    CPD_ERR_CUDA = 3,
    CPD_ERR_STATE = 4,       /* call out of order (e.g. step before init) */
    CPD_ERR_UNSUPPORTED = 5
};

/* Peridynamic force models (CabanaPD_Types.hpp:145-163). LINEAR_PMB uses the
 * linearised bond stretch (force/CabanaPD_PMB.hpp:406-538) and has no
 * fracture variant. LINEAR_LPS computes exactly like LPS, with or without
 * fracture, as the reference's Solver does: ForceModel<LinearLPS> keeps
 * force_tag = LPS (force_models/CabanaPD_LPS.hpp:32, 255-272) and the Solver
 * selects Force<force_tag, ...> (CabanaPD_Solver.hpp:96-99). */
enum {
    CPD_PD_NONE = 0,
    CPD_PD_PMB = 1,
    CPD_PD_LPS = 2,
    CPD_PD_LINEAR_PMB = 3,
    CPD_PD_LINEAR_LPS = 4
};

/* Contact models. HERTZ: force_models/CabanaPD_Hertzian.hpp.
 * NORMAL_REPULSION: force_models/CabanaPD_Contact.hpp:54-89 with
 * force/CabanaPD_Contact.hpp:42-104, the short-range repulsion that keeps
 * fragments of a PD body apart: a pair whose current distance r is below
 * contact_radius adds 15 c (r - contact_radius) / contact_horizon vol_j along
 * the pair, with c = 18 contact_K / (pi contact_horizon^4). Both search their
 * pairs on current positions within 2 contact_radius + radius_extend. */
enum { CPD_CONTACT_NONE = 0, CPD_CONTACT_HERTZ = 1, CPD_CONTACT_NORMAL_REPULSION = 2 };

/* Kernel arithmetic. EXACT evaluates every per-bond expression with IEEE
 * double operations in the reference's operand order (no FMA contraction),
 * so per-particle results equal a scalar CPU evaluation bit for bit.
 * FP64 is the throughput form of the same double-precision model: one
 * reciprocal square root per bond length instead of two square roots and
 * four divisions, FMA allowed; forces agree with EXACT to ~1e-13 relative
 * (norm-wise) and the broken-bond decision is re-evaluated exactly inside a
 * 1e-12 guard band, so broken-bond sets are identical. PMB and LPS use it;
 * the linearized models, Hertz contact (outside MIXED) and normal repulsion
 * always run EXACT.
 * MIXED (PMB and LPS without contact): FP32 bond arithmetic with bond
 * reference vectors precomputed in FP64 (lattice stencil tables where rows
 * share one), FP32 sums of 8-bond chunks added into FP64 row totals, FP64
 * integration and reductions, and an exact FP64 re-test of every bond whose
 * stretch is within 1e-4 s0 of s0, so broken-bond sets match FP64. Hertz
 * contact evaluates its force law in FP32 on FP64 overlaps. The PD kernels
 * of a system with contact, and the other models, run FP64 under MIXED. */
enum { CPD_FP64_EXACT = 0, CPD_FP64 = 1, CPD_MIXED = 2 };

/* Internal particle order: INPUT keeps the caller's order; MORTON sorts by
 * the Morton code of the particle's cell (results are returned in the
 * caller's order either way). */
enum { CPD_ORDER_INPUT = 0, CPD_ORDER_MORTON = 1 };

/* Force boundary conditions, applied after the force every step and once at
 * init (Solver.hpp:270-273, 365-367), in the order they were added. */
enum {
    CPD_BC_FORCE_VALUE = 0,  /* f(p, d) = values[0], d = 0..2 (ForceValueBCTag) */
    CPD_BC_FORCE_UPDATE = 1, /* f(p, d) += values[0], d = 0..2 (ForceUpdateBCTag) */
    CPD_BC_FORCE_ADD = 2     /* f(p, component) += values[b]: the custom-functor
                                traction / body-force form f(p, d) += g(p) */
};

/* Fields for cpd_download / cpd_device_field. Vector fields are returned as
 * [n][3] (x, y, z interleaved, the reference's slice layout); the stress as
 * [n][3][3] (sliceStress() layout), on the device component-major
 * [9][stride] with component 3 a + b. */
enum {
    CPD_FIELD_X = 0,      /* reference position */
    CPD_FIELD_U = 1,      /* displacement */
    CPD_FIELD_V = 2,      /* velocity */
    CPD_FIELD_F = 3,      /* force density */
    CPD_FIELD_VOL = 4,
    CPD_FIELD_RHO = 5,
    CPD_FIELD_M = 6,      /* LPS weighted volume */
    CPD_FIELD_THETA = 7,  /* LPS dilatation */
    CPD_FIELD_W = 8,      /* strain energy density */
    CPD_FIELD_PHI = 9,    /* damage */
    CPD_FIELD_RADIUS = 10, /* contact radius (per-particle model) */
    CPD_FIELD_STRESS = 11  /* per-particle stress (after cpd_compute_stress) */
};

typedef struct cpd_params {
    int32_t pd_model;            /* CPD_PD_* */
    int32_t fracture;            /* 1: critical-stretch bond breaking */
    int32_t influence_type;      /* LPS/fracture influence: -1 model default
                                    (PMB 1, LPS 0), else 0 or 1 */
    int32_t contact_model;       /* CPD_CONTACT_* */
    double horizon;              /* PD force horizon delta */
    double K, G, G0;             /* bulk modulus, shear modulus, fracture energy */
    double contact_radius;       /* Hertz particle radius (largest radius when
                                    per_particle_radius = 1); normal
                                    repulsion: the contact radius */
    double radius_extend;        /* contact search-radius extension (skin) */
    double nu, E, restitution;   /* Hertz material */
    double dt;                   /* time step */
    int32_t rebuild_every;       /* contact list: 0 = rebuild when the largest
                                    displacement since the last build exceeds
                                    radius_extend (Neighbor.hpp:118-119);
                                    k > 0 = rebuild every k steps */
    int32_t per_particle_radius; /* 1: Hertz with per-particle radii */
    int32_t precision;           /* CPD_FP64_EXACT, CPD_FP64 or CPD_MIXED */
    int32_t ordering;            /* CPD_ORDER_* */
    int32_t device;              /* CUDA device ordinal */
    double contact_horizon;      /* normal repulsion: the delta of its
                                    stiffness (NormalRepulsionModel delta) */
    double contact_K;            /* normal repulsion: the bulk modulus of its
                                    stiffness (NormalRepulsionModel K) */
} cpd_params;

int32_t cpd_abi_version(void);
const char* cpd_last_error(void);

cpd_status cpd_system_create(const cpd_params* params, cpd_system** out);
cpd_status cpd_system_destroy(cpd_system* sys);

/* Use a caller-owned CUDA stream (a cudaStream_t passed as void*) instead of
 * the system's own. NULL restores the system's own stream. */
cpd_status cpd_set_stream(cpd_system* sys, void* cuda_stream);
cpd_status cpd_get_stream(cpd_system* sys, void** cuda_stream);

/* Model constants derived by the reference constructors:
 * out[0]=c, [1]=s0, [2]=bond_break_coeff, [3]=theta_coeff, [4]=s_coeff,
 * [5]=Rs, [6]=Es, [7]=beta, [8]=coeff_h_n, [9]=coeff_h_d. */
cpd_status cpd_model_constants(const cpd_system* sys, double* out10);

/* Particles [0, n_frozen) are frozen: never integrated, no neighbour rows,
 * but still neighbours of others (CabanaPD_Particles.hpp:543-556).
 * x: [n][3]; vol: [n]; rho, nofail, radius may be NULL (1.0, 0, contact_radius).
 * Resets u, v, f to zero. */
cpd_status cpd_upload_particles(cpd_system* sys, int64_t n, int64_t n_frozen,
                                const double* x, const double* vol,
                                const double* rho, const int32_t* nofail,
                                const double* radius);
/* u, v: [n][3] or NULL to leave unchanged. */
cpd_status cpd_set_state(cpd_system* sys, const double* u, const double* v);

cpd_status cpd_build_neighbors(cpd_system* sys);
cpd_status cpd_neighbor_stats(const cpd_system* sys, int32_t* max_neighbors,
                              int64_t* total_neighbors);
/* Row i (caller's order) lists neighbours in ascending caller index:
 * counts [n]; indices and mu [n][max_neighbors] (padding -1 / 0).
 * mu[i][k] = 1 while bond k of particle i is intact. Any pointer may be NULL.
 * Returns the PD list, or the contact list for a DEM-only system. */
cpd_status cpd_download_neighbors(cpd_system* sys, int32_t* counts,
                                  int32_t* indices, int32_t* mu);

/* v1, v2, p0: [count][3] (plane vectors and corner of each notch). */
cpd_status cpd_prenotch(cpd_system* sys, int32_t count, const double* v1,
                        const double* v2, const double* p0);

/* indices: caller particle indices [count]; values: 1 scalar for
 * FORCE_VALUE / FORCE_UPDATE, [count] for FORCE_ADD. */
cpd_status cpd_add_boundary_condition(cpd_system* sys, int32_t kind,
                                      int32_t component, int64_t count,
                                      const int64_t* indices,
                                      const double* values);
cpd_status cpd_clear_boundary_conditions(cpd_system* sys);

/* Kernel-level seam, as the reference's unit tests call Force directly. */
cpd_status cpd_compute_weighted_volume(cpd_system* sys);
cpd_status cpd_compute_dilatation(cpd_system* sys);
cpd_status cpd_compute_force(cpd_system* sys);
/* W_i, damage phi_i and the totals sum(W_i vol_i), sum(phi_i). */
cpd_status cpd_compute_energy(cpd_system* sys, double* total_strain_energy,
                              double* total_damage);
/* Per-particle stress sigma_i = sum over row i of (1/2) f_pair (x) xi (the
 * reference's computeStressFull: half the pair force times the reference bond
 * vector; LPS with fracture over intact bonds only), of the current state:
 * bond bits and, for LPS, the m / theta of the last force update. The
 * reference computes it at init and output steps of particles built with
 * EnergyStressOutput (Solver.hpp:243, 486). Frozen particles get zero.
 * Allocates 72 B per particle on the first call. Queued on the stream;
 * cpd_download(CPD_FIELD_STRESS) waits. */
cpd_status cpd_compute_stress(cpd_system* sys);
/* No counterpart in the reference. The same energy and damage computation
 * for callers that may not allocate device memory after set-up (a job
 * server that reserved each job's memory at admission, or a framework that
 * owns all device memory through its own pool). W_out and phi_out are caller
 * device buffers of at least the system's stride (cpd_device_field) doubles,
 * filled in the internal particle order (frozen rows, and every row of a
 * system without a PD model, are set to 0); totals_out is a caller device
 * buffer of 2 doubles (sum W_i vol_i, sum phi_i). Queued on the system's
 * stream without waiting. Scratch is a fixed 256 KB array inside the library
 * (held on every GPU that loads it until exit), which limits a call to
 * 4,194,304 particle rows; larger systems are rejected with
 * CPD_ERR_INVALID_ARGUMENT. The first call on a device looks up that array's
 * device address, so make it before any stream capture. All calls share the
 * one array: calls whose work overlaps on the GPU (other streams, other
 * systems on the same device) race; calls queued on one stream do not. */
cpd_status cpd_compute_energy_noalloc(cpd_system* sys, double* W_out, double* phi_out,
                                      double* totals_out);

/* State snapshots, for checkpoint / restart and for evicting a job and
 * resuming it later. No counterpart in the reference. A snapshot holds the
 * evolving state: displacement, velocity and force, the broken-bond bits,
 * the LPS weighted volume, dilatation and their force coefficients, and
 * the contact list's rebuild state (displacement at the last build, step
 * and rebuild counters). It restores into a system set up the same way
 * (same parameters, particles, ordering, pre-notches and boundary
 * conditions, after cpd_init); the continued run is then bit-identical to
 * the uninterrupted one. A snapshot of a differently set-up system is
 * rejected with CPD_ERR_INVALID_ARGUMENT. Strain energy, damage and stress
 * are outputs, not state: compute them again after a restore. Both calls
 * wait for the stream. */
cpd_status cpd_state_bytes(cpd_system* sys, uint64_t* bytes);
cpd_status cpd_save_state(cpd_system* sys, void* host_buf, uint64_t bytes);
cpd_status cpd_load_state(cpd_system* sys, const void* host_buf, uint64_t bytes);

cpd_status cpd_init(cpd_system* sys);
/* num_steps velocity-Verlet steps. Asynchronous: returns once the work is
 * queued on the stream (cpd_synchronize or any download waits for it).
 * For PD systems without contact on the FP64 and MIXED kernels, each step is
 * one bond-kernel launch that also applies the force boundary conditions and
 * both half steps (when every particle and force component has at most one
 * boundary-condition operation); results are bit-identical to the separate
 * stages of cpd_step_stage. */
cpd_status cpd_step(cpd_system* sys, int32_t num_steps);
/* num_steps steps, then the strain energy and damage totals of the final
 * state: the Solver's output step (CabanaPD_Solver.hpp:479-494) in one
 * call, the same as cpd_step followed by cpd_compute_energy (W and phi
 * fields included; damage bit for bit, strain energy within FP32 rounding
 * of its bond terms on the MIXED path). On the MIXED PMB fracture fused
 * step of a one-volume particle set, the last step's bond pass also forms
 * the energy of its lean rows, so only the other rows take the separate
 * energy pass. Waits for the stream. */
cpd_status cpd_step_energy(cpd_system* sys, int32_t num_steps, double* total_strain_energy,
                           double* total_damage);
cpd_status cpd_synchronize(cpd_system* sys);
/* One stage of one time step, for callers that run their own device code
 * between stages (CabanaPD_Solver.hpp:332-375 order): INITIAL_HALF is the
 * first velocity-Verlet half step, FORCE the weighted volume / dilatation /
 * bond force / contact force, FORCE_BC the boundary conditions added with
 * cpd_add_boundary_condition, FINAL_HALF the second half step. Running the
 * four stages in order equals cpd_step(sys, 1). Device code between stages
 * may write the fields of cpd_device_field on the system's stream (FORCE
 * re-reads u for the MIXED kernels). Asynchronous. */
enum {
    CPD_STAGE_INITIAL_HALF = 0,
    CPD_STAGE_FORCE = 1,
    CPD_STAGE_FORCE_BC = 2,
    CPD_STAGE_FINAL_HALF = 3
};
cpd_status cpd_step_stage(cpd_system* sys, int32_t stage);

/* Copy a field to host memory in the caller's particle order. */
cpd_status cpd_download(cpd_system* sys, int32_t field, double* host_out);
double cpd_max_displacement(const cpd_system* sys);
int64_t cpd_contact_rebuilds(const cpd_system* sys);

/* Device pointer of a field in the internal order, component-major
 * ([3][stride] for vectors), for user kernels between steps. */
cpd_status cpd_device_field(cpd_system* sys, int32_t field, void** ptr,
                            int64_t* stride);

/* Device view of the broken-bond state (Neighbor::brokenBonds,
 * CabanaPD_Neighbor.hpp:219, which hands out the mu view): one bit per bond,
 * uint32 bits[words][stride] in the internal particle order, bit b of word w
 * of row i covering bond slot 32 w + b of that row (1 = intact). Slots follow
 * the row order of cpd_download_neighbors. Systems built from the same
 * particles in the same order have the same layout, so their bond states
 * compare word for word on the device. *bits is NULL for systems without
 * fracture. Read it between steps; the bond kernels rewrite it. */
cpd_status cpd_bond_bits(cpd_system* sys, void** bits, int32_t* words, int64_t* stride);

/* Per-kernel device time: when enabled, the bond kernels of every step are
 * bracketed by CUDA events on the system stream.
 * cpd_kernel_time returns the summed milliseconds and launch count of the
 * main bond kernel since timing was enabled, and the bytes the plain-FP64
 * bond algorithm is required to move per launch (the same denominator in
 * every precision mode). */
cpd_status cpd_set_kernel_timing(cpd_system* sys, int32_t enable);
cpd_status cpd_kernel_time(cpd_system* sys, double* total_ms,
                           int64_t* launches, double* bytes_per_launch);
/* Number of kernels this library launched on the system since creation. */
int64_t cpd_kernel_launches(const cpd_system* sys);
/* No counterpart in the reference. Which bond kernels hold the rows (after
 * cpd_build_neighbors): the warps of 32 rows the lattice-stencil kernels
 * walk (CPD_FP64 and CPD_MIXED PMB on a lattice whose offset table fits the
 * unrolled kernels), the warps the general kernels take beside them, and
 * the entries of the offset table; all 0 when the general kernels run
 * every row. */
cpd_status cpd_stencil_stats(const cpd_system* sys, int64_t* stencil_warps,
                             int64_t* irregular_warps, int32_t* table_entries);
/* No counterpart in the reference. Device bytes the system holds (particle
 * fields, neighbour and contact lists, mixed-precision copies, boundary
 * lists), for admission against a memory budget. */
cpd_status cpd_device_bytes(const cpd_system* sys, uint64_t* bytes);

/* ===========================================================================
 * Batched step. No counterpart in the reference, which advances one
 * specimen per process with one kernel per phase (CabanaPD_Solver.hpp:332-404).
 * A batch advances many set-up systems together: one table of per-instance
 * device views (offsets into the device memory pool) and one tile list over
 * all their particle rows; per time step one launch of a persistent-block
 * kernel runs the bond force, bond breaking and both velocity-Verlet half
 * steps of every instance (two launches when an LPS instance needs its
 * dilatation pass), and a chunk of k steps is replayed from a CUDA graph.
 * Each instance runs the arithmetic of its system's general (non-stencil)
 * kernels: CPD_FP64 systems the FP64 throughput kernels, CPD_MIXED systems
 * the mixed ones, so results do not depend on the other instances or on the
 * launch shape. An autotuner picks the persistent grid (blocks per SM) and
 * the tile order by timing the first chunks, one candidate each (all
 * candidates give identical results), and keeps the fastest.
 *
 * Systems must be set up and initialised (cpd_init), peridynamic without
 * contact, CPD_FP64 or CPD_MIXED, on one device, with boundary conditions
 * that fit the fused step. While a system belongs to a batch, calls that
 * change its state (cpd_step*, cpd_set_state, cpd_load_state, cpd_init, set-up
 * calls, cpd_system_destroy) return CPD_ERR_STATE; reads (cpd_compute_energy,
 * cpd_download, cpd_save_state, ...) are ordered after the batch's chunks.
 * cpd_batch_destroy releases the systems (it does not destroy them).
 */
typedef struct cpd_batch cpd_batch;

/* steps[i]: the number of time steps instance i is to take in total. */
cpd_status cpd_batch_create(cpd_system* const* systems, int32_t count, const int32_t* steps,
                            cpd_batch** out);
cpd_status cpd_batch_destroy(cpd_batch* batch);
/* One chunk: every instance with steps left advances min(chunk_steps, its
 * steps left) steps. Asynchronous with respect to the host. */
cpd_status cpd_batch_step(cpd_batch* batch, int32_t chunk_steps);
/* Hands back instance i once it has no steps left: its system takes
 * state-changing calls again (and may be destroyed) while the batch runs
 * on; work later issued on the system's stream still follows the chunk that
 * finished it. */
cpd_status cpd_batch_release(cpd_batch* batch, int32_t instance);
/* Steps instance i still has to take (as of the chunks issued so far). */
cpd_status cpd_batch_remaining(const cpd_batch* batch, int32_t instance, int32_t* steps);
cpd_status cpd_batch_synchronize(cpd_batch* batch);
/* Fix the launch shape to candidate `candidate` (0 <= candidate <
 * *count), or -1 to let the autotuner choose. */
cpd_status cpd_batch_set_candidate(cpd_batch* batch, int32_t candidate);
/* The autotuner's state: candidates, the chosen one (-1 while tuning), and
 * per candidate its persistent grid in blocks per SM, its tile order (0 by
 * instance, 1 interleaved across instances) and its measured throughput in
 * bond-updates/s (0 if not timed). Arrays hold at least *count entries when
 * non-NULL (query *count first with NULL arrays). */
cpd_status cpd_batch_tuning(const cpd_batch* batch, int32_t* count, int32_t* chosen,
                            int32_t* blocks_per_sm, int32_t* order, double* throughput);
/* Kernels the batch launched (graph replays count each kernel node). */
int64_t cpd_batch_launches(const cpd_batch* batch);

/* ===========================================================================
 * Job server. No counterpart in the reference, which runs one simulation per
 * process. Continuous batching of independent simulations on one GPU: jobs
 * are described on the host (cpd_job_*: the same inputs as a cpd_system),
 * submitted at any time, admitted in arrival order while the device bytes of
 * the resident jobs stay within a budget, advanced concurrently (each on its
 * own CUDA stream, in k-step chunks replayed from a CUDA graph, jobs with less
 * work on higher-priority streams) and retired when done; their totals and
 * the fields asked for stay on the host until released. A job's results do
 * not depend on what else runs: it owns its arrays and stream, and every
 * kernel is deterministic. Thread-safe: any host thread may submit, wait,
 * query, download or release while the server's two threads run the jobs.
 * Contact (DEM) jobs run too, without graphs (their neighbour rebuilds are
 * decided on the host between steps).
 */
typedef struct cpd_job cpd_job;
typedef struct cpd_server cpd_server;

enum { CPD_JOB_QUEUED = 0, CPD_JOB_RUNNING = 1, CPD_JOB_DONE = 2, CPD_JOB_FAILED = 3 };

typedef struct cpd_server_config {
    int32_t device;
    int32_t max_active;         /* resident jobs at once (one stream each) */
    int32_t steps_per_launch;   /* k: steps per launched chunk */
    int32_t use_graphs;         /* 1: replay the k-step chunk as a CUDA graph */
    uint64_t hbm_budget_bytes;  /* admission budget on resident device bytes */
    int32_t setup_threads;      /* host threads that admit / set up / retire
                                   jobs concurrently; 0 = 4 */
    int32_t batch_max_particles; /* > 0: peridynamic jobs without contact in
                                   CPD_FP64 / CPD_MIXED with at most this many
                                   particles are advanced in batch groups
                                   (cpd_batch_*: one launch per step for the
                                   group, jobs set up together form a group);
                                   0: every job on its own */
    double evict_after_s;       /* > 0: when the queue's head has waited this
                                   long for memory, the resident job with the
                                   most work left (more than the head's) is
                                   evicted: its state is saved to the host
                                   (cpd_save_state), its device memory freed,
                                   and it is queued again right behind the
                                   head; set up again later, it resumes from
                                   the snapshot (cpd_load_state), bit-identical
                                   to an uninterrupted run. 0: never */
} cpd_server_config;

typedef struct cpd_job_status {
    int32_t state;              /* CPD_JOB_* */
    int32_t steps;              /* requested */
    int32_t steps_done;
    int32_t priority;           /* CUDA stream priority of the job */
    int64_t n;                  /* particles */
    int64_t bonds;              /* directed neighbour entries at admission */
    uint64_t device_bytes;      /* held while resident */
    /* server clock, s: submitted, admitted (set-up begins), set up, first
     * chunk launched, finished */
    double submit_time, admit_time, ready_time, start_time, finish_time;
    double total_strain_energy, total_damage;                 /* at the end */
    int64_t kernel_launches;    /* kernels run (graph replays count each node) */
    int64_t evictions;          /* times the job was evicted and resumed */
} cpd_job_status;

typedef struct cpd_server_stats {
    int64_t submitted, done, failed, resident, queued;
    uint64_t resident_bytes, peak_resident_bytes;
    int64_t kernel_launches;
    double bond_updates;        /* sum over finished jobs of bonds x steps */
} cpd_server_stats;

cpd_status cpd_job_create(const cpd_params* params, int32_t num_steps, cpd_job** out);
/* Only for a job that was never submitted (submission takes ownership). */
cpd_status cpd_job_destroy(cpd_job* job);
cpd_status cpd_job_set_particles(cpd_job* job, int64_t n, int64_t n_frozen, const double* x,
                                 const double* vol, const double* rho, const int32_t* nofail,
                                 const double* radius);
cpd_status cpd_job_set_state(cpd_job* job, const double* u, const double* v);
cpd_status cpd_job_prenotch(cpd_job* job, int32_t count, const double* v1, const double* v2,
                            const double* p0);
cpd_status cpd_job_add_boundary_condition(cpd_job* job, int32_t kind, int32_t component,
                                          int64_t count, const int64_t* indices,
                                          const double* values);
/* Fields (bit 1 << CPD_FIELD_*) copied to the host when the job finishes;
 * default: U only. */
cpd_status cpd_job_keep_fields(cpd_job* job, uint32_t field_mask);

cpd_status cpd_server_create(const cpd_server_config* config, cpd_server** out);
/* Fails queued jobs, lets resident ones finish, then stops the threads. */
cpd_status cpd_server_destroy(cpd_server* server);
/* Takes ownership of job, also when it returns an error. */
cpd_status cpd_server_submit(cpd_server* server, cpd_job* job, int64_t* job_id);
/* Seconds since the server was created (the clock of cpd_job_status). */
double cpd_server_clock(const cpd_server* server);
/* Block until the job is DONE or FAILED; CPD_ERR_STATE after timeout_s. */
cpd_status cpd_server_wait(cpd_server* server, int64_t job_id, double timeout_s);
/* Block until every submitted job is DONE or FAILED. */
cpd_status cpd_server_drain(cpd_server* server, double timeout_s);
cpd_status cpd_server_job_status(cpd_server* server, int64_t job_id, cpd_job_status* out);
/* Error message of a FAILED job (empty otherwise), NUL-terminated. */
cpd_status cpd_server_job_error(cpd_server* server, int64_t job_id, char* buf, int64_t size);
/* A kept field of a DONE job, in the caller's particle order. */
cpd_status cpd_server_download(cpd_server* server, int64_t job_id, int32_t field,
                               double* host_out);
/* Evict a running job (not one in a batch group): once its chunks in
 * flight complete, its state is saved to the host and its device memory
 * freed; it is queued again behind the queue's head and resumes from the
 * snapshot, bit-identical to an uninterrupted run. */
cpd_status cpd_server_evict(cpd_server* server, int64_t job_id);
cpd_status cpd_server_release(cpd_server* server, int64_t job_id);
cpd_status cpd_server_stats_get(cpd_server* server, cpd_server_stats* out);

#ifdef __cplusplus
}
#endif
#endif
