"""Pins the CPU oracle against the reference's regression tests
(regression_test/tstKalthoffWinkler.hpp, tstHertz.hpp). CPU only."""
import numpy as np

from cabanapd_b200 import problems as P


def kw_max_crack_y(system, prob):
    """examples/mechanics/kalthoff_winkler.cpp:129-147: OutputTimeSeries with
    a Max reducer of (damage > 0.3 ? y : 0) every output step; the test
    reads the last value."""
    x = prob["x"]
    freq = prob["output_frequency"]
    last = None
    for step in range(1, prob["num_steps"] + 1):
        system.run(1)
        if step % freq == 0:
            system.compute_energy()
            phi = system.get("phi")
            last = max(0.0, float(np.max(np.where(phi > 0.3, x[:, 1], 0.0))))
    return last


def hertz_restitution(system, prob):
    rho, vol = prob["rho"], prob["vol"]

    def ke():
        v = system.get("v")
        return float(np.sum(0.5 * rho * vol * np.sum(v * v, axis=1)))

    ke_i = ke()
    system.run(prob["num_steps"])
    return np.sqrt(ke() / ke_i)


def elastic_wave_profile_errors(golden, xs, us):
    """regression_test/tstElasticWave.hpp:54-96: relative error of each
    profile point against the fitted polynomial (skipping |x| > 0.425 and
    |x| < 0.025) and the l2 norm of the differences."""
    coeff = golden["elastic_wave"]["poly_coeff_descending"]
    rel, total = [], 0.0
    for xx, u in zip(xs, us):
        if xx > 0.425 or xx < -0.425 or (-0.025 < xx < 0.025):
            continue
        fit = 0.0
        for c in coeff:
            fit = fit * xx + c
        rel.append(abs((u - fit) / fit))
        total += (u - fit) ** 2
    return max(rel), total ** 0.5


def test_elastic_wave_profile(oracle, golden):
    """The LinearLPS elastic-wave regression on the oracle (41^3, 60 steps):
    the displacement profile along x within 3.5 % of the fitted polynomial
    and l2 < 3e-5. Passing it needs LinearLPS to compute as LPS."""
    g = golden["elastic_wave"]
    prob = P.elastic_wave_lps(g["input"])
    s = oracle.OracleSystem(prob["params"])
    P.setup(s, prob)
    s.run(prob["num_steps"])
    xs, us = P.displacement_profile(prob, s.get("u"))
    assert len(xs) == 41
    rel, l2 = elastic_wave_profile_errors(golden, xs, us)
    assert rel < g["rel_tol"] and l2 < g["l2_tol"], (rel, l2)


def test_linear_lps_computes_as_lps(oracle):
    """ForceModel<LinearLPS> selects Force<LPS> in the reference, with or
    without fracture: identical fields."""
    prob = P.lps_random_notches(num_cells=(60, 24, 2), steps=5)
    out = []
    for model in (P.PD_LPS, P.PD_LINEAR_LPS):
        s = oracle.OracleSystem(dict(prob["params"], pd_model=model))
        P.setup(s, prob)
        s.run(prob["num_steps"])
        out.append([s.get(f) for f in ("u", "f", "theta", "m")] + [s.compute_energy()])
    for a, b in zip(out[0][:4], out[1][:4]):
        assert np.array_equal(a, b)
    assert out[0][4] == out[1][4]


def test_kalthoff_winkler_crack_extent(oracle, golden):
    g = golden["kalthoff_winkler"]
    prob = P.kalthoff_winkler_regression()
    assert prob["num_steps"] == int(g["input"]["final_time"]["value"] /
                                    g["input"]["timestep"]["value"])
    s = oracle.OracleSystem(prob["params"])
    P.setup(s, prob)
    y = kw_max_crack_y(s, prob)
    assert abs(y - g["max_crack_y"]) <= g["tolerance"], y


def test_hertz_restitution(oracle, golden):
    g = golden["hertz"]
    prob = P.hertz_two_spheres()
    s = oracle.OracleSystem(prob["params"])
    P.setup(s, prob)
    e = g["input"]["restitution"]["value"]
    r = hertz_restitution(s, prob)
    assert abs(r - e) <= g["tolerance"], r


def test_polydisperse_hertz_reduces_to_single_radius(oracle):
    """The per-particle-radius contact extension reproduces the reference's
    single-radius model bit for bit when all radii are equal."""
    prob = P.hertz_two_spheres()
    a = oracle.OracleSystem(prob["params"])
    P.setup(a, prob)
    a.run(400)
    params = dict(prob["params"], per_particle_radius=1)
    b = oracle.OracleSystem(params)
    P.setup(b, dict(prob, radius=np.full(2, 5e-5)))
    b.run(400)
    assert np.array_equal(a.get("u"), b.get("u"))
    assert np.array_equal(a.get("v"), b.get("v"))
