// Step epilogue of the throughput bond kernels: the force boundary
// conditions, the second velocity-Verlet half step of this step and the first
// half step of the next one, applied by the thread that just summed row i's
// force. One kernel per time step replaces bond kernel + boundary-condition
// kernels + two integrator kernels (CabanaPD_Solver.hpp:332-375 order,
// CabanaPD_Integrate.hpp:89-145 arithmetic).
//
// Neighbours of other rows may still be reading this row's displacement
// (and, in contact steps, its velocity), so the next displacement goes to a
// second buffer (u_next, and v_next when set); the caller swaps buffers
// between steps. Every operation is a separately rounded IEEE
// operation in the order of the separate kernels (k_force_bc, k_vv_final,
// k_vv_initial), so fused and separate steps give identical bits.
#pragma once

#include "cpd_internal.cuh"

namespace cpd {

// FP32 split of a displacement for the mixed kernel (see MixedU).
__device__ __forceinline__ MixedU split_u(double u0, double u1, double u2, double cvol,
                                          uint8_t nofail)
{
    MixedU m;
    m.hi = make_float4(__double2float_rn(u0), __double2float_rn(u1), __double2float_rn(u2),
                       __double2float_rn(cvol));
    m.lo = make_float4(__double2float_rn(u0 - (double)m.hi.x),
                       __double2float_rn(u1 - (double)m.hi.y),
                       __double2float_rn(u2 - (double)m.hi.z), (float)nofail);
    return m;
}

// Row i's force boundary condition, if it has one: for each component d the
// condition touches (bit 4 + d of keep), f_d becomes f_d + add_d if keep bit
// d is set (ForceUpdate, the force-add form), else add_d (ForceValue).
// Rows are found by a bitmap test and a binary search of the sorted list.
__device__ __forceinline__ void apply_row_bc(const StepEpilogue& ep, int64_t i, double (&f)[3])
{
    if (!ep.bc_bits || !((ep.bc_bits[i >> 5] >> (i & 31)) & 1u)) return;
    int lo = 0, hi = ep.nbc - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (ep.bc_row[mid] < i)
            lo = mid + 1;
        else
            hi = mid;
    }
    const uint8_t keep = ep.bc_keep[lo];
    for (int d = 0; d < 3; ++d) {
        if (!((keep >> (4 + d)) & 1u)) continue;
        const double a = ep.bc_add[(int64_t)d * ep.nbc + lo];
        f[d] = ((keep >> d) & 1u) ? __dadd_rn(f[d], a) : a;
    }
}

// Finishes row i after its force sum f (mode 0: store f only).
template <bool MIXED>
__device__ __forceinline__ void step_epilogue(const ParticleView& p, const StepEpilogue& ep,
                                              int64_t i, double f0, double f1, double f2)
{
    const int64_t np = p.npad;
    double f[3] = {f0, f1, f2};
    if (ep.mode == 0) {
        p.f[i] = f[0];
        p.f[np + i] = f[1];
        p.f[2 * np + i] = f[2];
        return;
    }
    apply_row_bc(ep, i, f);
    const double hm = __ddiv_rn(ep.half_dt, p.rho[i]);
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = __dadd_rn(p.v[d * np + i], __dmul_rn(hm, f[d]));
    double* const v_out = ep.v_next ? ep.v_next : p.v;
    if (ep.mode == 1) {
        for (int d = 0; d < 3; ++d) {
            p.f[d * np + i] = f[d];
            v_out[d * np + i] = v[d];
        }
        return;
    }
    // mode 2: the next step's first half step; this step's f is not kept.
    double u[3];
    for (int d = 0; d < 3; ++d) {
        v[d] = __dadd_rn(v[d], __dmul_rn(hm, f[d]));
        v_out[d * np + i] = v[d];
        u[d] = __dadd_rn(p.u[d * np + i], __dmul_rn(ep.dt, v[d]));
        ep.u_next[d * np + i] = u[d];
    }
    if (MIXED) ep.u2_next[i] = split_u(u[0], u[1], u[2], ep.c * p.vol[i], p.nofail[i]);
    if (!MIXED && ep.u4_next)
        ep.u4_next[ep.u4_cell ? (int64_t)ep.u4_cell[i] : i] =
            make_double4(u[0], u[1], u[2], p.vol[i]);
}

}  // namespace cpd
