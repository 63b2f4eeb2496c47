"""Backend-agnostic restatement of unit_test/tstForce.hpp testForce /
checkResults (tstForce.hpp:666-978): build the [-1, 1]^3 lattice, impose a
linear or quadratic displacement, run weighted volume, dilatation, force and
energy through the backend's kernel-level seam, and check every interior
particle against the single-point reference sums and analytic values."""
import numpy as np

import reference_sums as R
from cabanapd_b200 import problems as P

CASES = {
    # name: (pd model, dx, boundary_width, fracture G0, influence, kind label)
    "pmb": (P.PD_PMB, 2.0 / 11.0, 1.1, None, None, "pmb"),
    "pmb_damage": (P.PD_PMB, 2.0 / 11.0, 1.1, 1000.0, None, "pmb"),
    "linear_pmb": (P.PD_LINEAR_PMB, 2.0 / 11.0, 1.1, None, None, "pmb"),
    "lps": (P.PD_LPS, 2.0 / 15.0, 2.1, None, 1, "lps"),
    "lps_damage": (P.PD_LPS, 2.0 / 15.0, 2.1, 1000.0, 1, "lps"),
    "linear_lps": (P.PD_LINEAR_LPS, 2.0 / 15.0, 2.1, None, 1, "lps"),
}


def run_case(make_system, case, kind, coeff):
    model, dx, bw, G0, infl, _ = CASES[case]
    K, G = 1.0, 0.5
    prob = P.unit_cube(model, dx, coeff, kind, K=K, G=G, G0=G0, influence_type=infl)
    sysm = make_system(prob["params"])
    P.setup(sysm, prob, init=False)
    # tstForce.hpp:895-902 initializeForce, then :946-947.
    sysm.compute_weighted_volume()
    sysm.compute_dilatation()
    sysm.compute_force()
    Phi, _ = sysm.compute_energy()
    sysm.compute_stress()  # tstForce.hpp:948
    out = {k: sysm.get(k) for k in ("x", "f", "W", "vol", "theta", "stress")}
    out["Phi"] = Phi
    out["constants"] = sysm.model_constants()
    out["max_neighbors"] = sysm.neighbor_stats()[0]
    return out, prob


def check_case(res, case, kind, coeff, max_checked=None):
    model_id, dx, bw, _, infl, mk = CASES[case]
    K, G = 1.0, 0.5
    m = 3
    horizon = dx * m
    c = res["constants"]
    if mk == "pmb":
        ref = R.PMBRef(c["c"])
    else:
        ref = R.LPSRef(c["theta_coeff"], c["s_coeff"], infl)
    x, f, W, vol, theta = res["x"], res["f"], res["W"], res["vol"], res["theta"]
    sigma = res["stress"]
    lo, hi = -1.0 + horizon * bw, 1.0 - horizon * bw
    interior = np.all((x > lo) & (x < hi), axis=1)
    idx = np.nonzero(interior)[0]
    assert idx.size > 0
    if max_checked is not None:
        idx = idx[:max_checked]
    failures = []
    for p in idx:
        xp = x[p, 0]
        ref_W = R.ref_W(ref, kind, horizon, m, coeff, xp)
        ref_f = R.ref_fx(ref, kind, horizon, m, coeff, xp)
        if kind == "linear":
            if not np.all(np.abs(f[p]) <= 1e-13):
                failures.append(("f", p, f[p]))
            if not R.float_eq(W[p], ref_W):
                failures.append(("W", p, W[p], ref_W))
            aW, band = R.analytic_W(mk, kind, K, G, coeff, horizon, xp)
            if band is None:
                if not R.float_eq(W[p], aW):
                    failures.append(("W_analytic", p, W[p], aW))
            elif abs(W[p] - aW) > band * W[p]:
                failures.append(("W_analytic", p, W[p], aW))
            # tstForce.hpp:744-750: diagonal equal to the reference sum, the
            # other components (xy, xz, yz, yx, zx, zy) <= 1e-13.
            ref_sigma = R.ref_stress(ref, kind, horizon, m, coeff)
            sp = sigma[p]
            for d in range(3):
                if not R.float_eq(sp[d, d], ref_sigma[d]):
                    failures.append(("stress_diag", p, d, sp[d, d], ref_sigma[d]))
            offdiag = [sp[0, 1], sp[0, 2], sp[1, 2], sp[1, 0], sp[2, 0], sp[2, 1]]
            if not all(v <= 1e-13 for v in offdiag):
                failures.append(("stress_offdiag", p, offdiag))
        else:
            if not R.float_eq(f[p, 0], ref_f):
                failures.append(("fx", p, f[p, 0], ref_f))
            af = R.analytic_fx(mk, K, G, coeff)
            if abs(f[p, 0] - af) > abs(0.10 * f[p, 0]):
                failures.append(("fx_analytic", p, f[p, 0], af))
            if not (f[p, 1] <= 1e-13 and f[p, 2] <= 1e-13):
                failures.append(("fyz", p, f[p]))
            if abs(W[p] - ref_W) > 1e-6:
                failures.append(("W", p, W[p], ref_W))
            aW, band = R.analytic_W(mk, kind, K, G, coeff, horizon, xp)
            if abs(W[p] - aW) > band * W[p]:
                failures.append(("W_analytic", p, W[p], aW))
    # tstForce.hpp:863-893 checkAnalyticalDilatation over every particle.
    if kind == "linear":
        if mk == "lps":
            bad = [p for p in range(x.shape[0]) if not R.float_eq(3 * coeff, theta[p])]
            if bad:
                failures.append(("theta", bad[:5]))
    # tstForce.hpp:722 total strain energy vs sum of W_i vol_i.
    ref_Phi = float(np.sum(W * vol))
    if abs(res["Phi"] - ref_Phi) > 1e-5:
        failures.append(("Phi", res["Phi"], ref_Phi))
    assert not failures, failures[:10]
    return idx.size
