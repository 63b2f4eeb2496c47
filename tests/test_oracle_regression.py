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
