/*
 * CPU oracle for the CabanaPD per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA
 * product path is compared against, and the CPU baseline that bench.py
 * times. Nothing in the product (cabanapd_b200/, include/) links or calls
 * it. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
 *
 * It restates, in plain C++17 + OpenMP, the reference's algorithms for:
 * particle kernels of PMB / LPS / LinearPMB / LinearLPS peridynamics (with
 * and without critical-stretch fracture), Hertzian contact, normal
 * repulsion contact, velocity Verlet,
 * pre-notch bond cutting, force boundary conditions and the Solver's
 * init/runStep orchestration. Each function in oracle.cpp cites the
 * reference file:line it follows (paths relative to the CabanaPD tree).
 *
 * The reference itself (Kokkos + Cabana + MPI) cannot be compiled on this
 * machine, so parity of this restatement is pinned against the reference's
 * own unit- and regression-test expectations (tests/test_oracle_*.py).
 *
 * Summation order: every per-particle sum walks its neighbour row in
 * ascending neighbour-index order. Global totals are summed serially in
 * ascending particle order. Built with -ffp-contract=off so no FMA
 * contraction changes the rounding of the reference's expressions.
 */
#ifndef CPD_ORACLE_H
#define CPD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system orc_system;

/* Same numbering as the product ABI (include/cabanapd_b200.h). */
enum {
    ORC_PD_NONE = 0,
    ORC_PD_PMB = 1,
    ORC_PD_LPS = 2,
    ORC_PD_LINEAR_PMB = 3,
    ORC_PD_LINEAR_LPS = 4
};
enum { ORC_CONTACT_NONE = 0, ORC_CONTACT_HERTZ = 1, ORC_CONTACT_NORMAL_REPULSION = 2 };
enum {
    ORC_BC_FORCE_VALUE = 0,   /* f(p, d) = value, d = 0..2 */
    ORC_BC_FORCE_UPDATE = 1,  /* f(p, d) += value, d = 0..2 */
    ORC_BC_FORCE_ADD = 2      /* f(p, component) += values[b] */
};
enum {
    ORC_FIELD_X = 0,
    ORC_FIELD_U = 1,
    ORC_FIELD_V = 2,
    ORC_FIELD_F = 3,
    ORC_FIELD_VOL = 4,
    ORC_FIELD_RHO = 5,
    ORC_FIELD_M = 6,
    ORC_FIELD_THETA = 7,
    ORC_FIELD_W = 8,
    ORC_FIELD_PHI = 9,
    ORC_FIELD_RADIUS = 10,
    ORC_FIELD_STRESS = 11  /* [n][3][3] per-particle stress */
};

typedef struct orc_params {
    int32_t pd_model;        /* ORC_PD_* */
    int32_t fracture;        /* 0 / 1 */
    int32_t influence_type;  /* -1: model default (PMB 1, LPS 0) */
    int32_t contact_model;   /* ORC_CONTACT_* */
    double horizon;          /* PD force horizon (delta) */
    double K, G, G0;         /* bulk, shear modulus, fracture energy */
    double contact_radius;   /* Hertz: particle radius (single-radius model) */
    double radius_extend;    /* Hertz: search-radius extension (skin) */
    double nu, E, restitution;
    double dt;
    int32_t rebuild_every;   /* contact list: 0 = displacement trigger */
    int32_t per_particle_radius; /* 1: use radius array (polydisperse) */
    double contact_horizon;  /* normal repulsion: delta of its stiffness */
    double contact_K;        /* normal repulsion: bulk modulus of its stiffness */
} orc_params;

orc_system* orc_create(const orc_params* p);
void orc_destroy(orc_system* s);
const char* orc_last_error(void);

/* Model constants as derived by the reference constructors, for pinning:
 * out[0]=c (PMB), [1]=s0, [2]=bond_break_coeff, [3]=theta_coeff,
 * [4]=s_coeff, [5]=Rs, [6]=Es, [7]=beta, [8]=coeff_h_n, [9]=coeff_h_d. */
int orc_model_constants(const orc_system* s, double* out10);

int orc_set_particles(orc_system* s, int64_t n, int64_t n_frozen,
                      const double* x, const double* vol, const double* rho,
                      const int32_t* nofail, const double* radius);
int orc_set_state(orc_system* s, const double* u, const double* v);
int orc_set_field(orc_system* s, int32_t field, const double* in);
int orc_build_neighbors(orc_system* s);
int orc_neighbor_stats(const orc_system* s, int32_t* max_n, int64_t* total);
/* counts[n]; idx/mu padded [n][max_n] */
int orc_get_neighbors(const orc_system* s, int32_t* counts, int32_t* idx,
                      int32_t* mu);
/* bits[w][n]: bit b of word w of row i = mu of slot 32 w + b (the product's
 * packing, cpd_bond_bits, without its row padding). */
int orc_get_bond_bits(const orc_system* s, uint32_t* bits);
int orc_prenotch(orc_system* s, int32_t k, const double* v1, const double* v2,
                 const double* p0);
int orc_add_bc(orc_system* s, int32_t kind, int32_t component, int64_t count,
               const int64_t* idx, const double* values);

/* Kernel-level seam (Force::computeWeightedVolume / computeDilatation /
 * computeForceFull / computeEnergyFull as used by the reference unit tests). */
int orc_compute_weighted_volume(orc_system* s);
int orc_compute_dilatation(orc_system* s);
int orc_compute_force(orc_system* s);
int orc_compute_energy(orc_system* s, double* total_W, double* total_D);
/* CabanaPD_Force.hpp:222-235 computeStress: zeroes and fills the stress. */
int orc_compute_stress(orc_system* s);

/* Solver-level: init (Solver::init with force BCs) and num_steps runSteps. */
int orc_init(orc_system* s);
int orc_run(orc_system* s, int32_t num_steps);
int orc_get(const orc_system* s, int32_t field, double* out);
double orc_max_displacement(const orc_system* s);
int64_t orc_contact_rebuilds(const orc_system* s);

/* Input.hpp computeCriticalTimeStep restated (returns dt_crit, not scaled). */
double orc_critical_timestep(double dx, double dy, double dz, int32_t m,
                             double horizon, double K, double rho);

int orc_num_threads(void);
void orc_set_num_threads(int32_t n);

#ifdef __cplusplus
}
#endif
#endif
