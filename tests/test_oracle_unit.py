"""Pins the CPU oracle against the reference's own unit-test expectations
(unit_test/tstForce.hpp, unit_test/tstIntegrator.hpp). CPU only."""
import math

import numpy as np
import pytest

import force_checks
import reference_sums as R
from cabanapd_b200 import problems as P
from cabanapd_b200.inputs import Inputs, critical_timestep


def _oracle_factory(oracle):
    return lambda params: oracle.OracleSystem(params)


@pytest.mark.parametrize("case,kind,coeff", [
    ("pmb", "linear", 0.1), ("pmb", "quadratic", 0.01),
    ("pmb_damage", "linear", 0.1), ("pmb_damage", "quadratic", 0.01),
    ("linear_pmb", "linear", 0.1),
    ("lps", "linear", 0.1), ("lps", "quadratic", 0.01),
    ("lps_damage", "linear", 0.1), ("lps_damage", "quadratic", 0.01),
    ("linear_lps", "linear", 0.1),
])
def test_force_cases(oracle, case, kind, coeff):
    res, _ = force_checks.run_case(_oracle_factory(oracle), case, kind, coeff)
    # The single-point sums are python loops; check a spread of particles.
    checked = force_checks.check_case(res, case, kind, coeff, max_checked=40)
    assert checked > 0


@pytest.mark.parametrize("m,num,den", [(3, 2.0, 11.0), (6, 2.0, 15.0)])
def test_neighbor_count(oracle, golden, m, num, den):
    """tstForce.hpp:983-1015 test_neighbor: max neighbours == full lattice
    neighbourhood count (122 for m = 3)."""
    assert [m, num, den] in golden["neighbor_cases"]["cases"]
    dx = num / den
    horizon = dx * m
    prob = P.unit_cube(P.PD_PMB, dx, 0.0, "linear")
    prob["params"]["horizon"] = horizon
    s = oracle.OracleSystem(prob["params"])
    P.setup(s, prob, init=False)
    expected = R.ref_neighbors(horizon, m)
    assert s.neighbor_stats()[0] == expected
    if m == 3:
        assert expected == 122


def test_four_spacing_horizon_holds_256_neighbours(oracle):
    """A cubic lattice at a horizon of exactly four spacings (the reference's
    example decks): interior rows hold the 256 lattice offsets within the
    cutoff (horizon + 1e-14, the axis points at 4 spacings included), the
    table size the wide FP64 stencil walk takes."""
    prob = P.plate_impact(num_cells=(24, 12, 12), steps=1, v0=0.0,
                          size=(0.2, 0.1, 0.1), horizon_factor=4.0)
    s = oracle.OracleSystem(prob["params"])
    P.setup(s, prob, init=False)
    assert s.neighbor_stats()[0] == 256
    assert P.plate_impact(num_cells=(24, 12, 12), steps=1, size=(0.2, 0.1, 0.1))[
        "params"]["horizon"] == 3.01 * 0.2 / 24


def test_neighbor_sets_bruteforce(oracle):
    """Every listed pair is within the cutoff and every pair within the cutoff
    is listed (all-pairs check on a jittered cloud)."""
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, size=(600, 3))
    prob = {"params": dict(pd_model=P.PD_PMB, fracture=1, horizon=0.35, K=1.0,
                           G0=1.0, dt=1.0)}
    s = oracle.OracleSystem(prob["params"])
    s.set_particles(x, np.ones(600))
    s.build_neighbors()
    counts, idx, _ = s.neighbors()
    cut2 = (0.35 + 1e-14) ** 2
    for i in range(600):
        d = x - x[i]
        d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
        exp = np.nonzero(d2 <= cut2)[0]
        exp = exp[exp != i]
        assert np.array_equal(idx[i, :counts[i]], exp)


def test_integrator_reversibility(oracle):
    """tstIntegrator.hpp:38-103: 100 velocity-Verlet steps, reverse v, 100
    back. With zero force the reference positions are untouched and the
    displacement returns to zero to rounding."""
    x, vol, _ = P.lattice([-1.0] * 3, [1.0] * 3, [10, 10, 10])
    rng = np.random.default_rng(3)
    v0 = rng.normal(size=x.shape)
    params = dict(pd_model=P.PD_PMB, fracture=0, horizon=1e-3, K=1.0, dt=0.001)
    s = oracle.OracleSystem(params)
    s.set_particles(x, vol)
    s.set_state(None, v0)
    s.build_neighbors()
    assert s.neighbor_stats()[1] == 0
    s.init()
    s.run(100)
    u_mid = s.get("u")
    s.set_state(u_mid, -s.get("v"))
    s.run(100)
    assert np.array_equal(s.get("x"), x)
    assert np.max(np.abs(s.get("u"))) <= 1e-15 * np.max(np.abs(u_mid))


def test_model_constants(oracle):
    """Constructor-derived constants (force_models/*.hpp) for the configs."""
    pr = P.plate_impact(num_cells=(40, 20, 4), steps=1)
    s = oracle.OracleSystem(pr["params"])
    c = s.model_constants()
    h = pr["params"]["horizon"]
    K = pr["params"]["K"]
    assert c["c"] == 18.0 * K / (math.pi * h * h * h * h)
    assert c["s0"] == math.sqrt(5.0 * 22170.0 / 9.0 / K / h)
    assert c["bond_break_coeff"] == (1.0 + c["s0"]) * (1.0 + c["s0"])
    hz = P.hertz_two_spheres()
    c = oracle.OracleSystem(hz["params"]).model_constants()
    ln_e = math.log(0.5)
    assert c["beta"] == -ln_e / math.sqrt(ln_e ** 2 + math.pi ** 2)
    assert c["Rs"] == 0.5 * 5e-5


def test_critical_timestep_matches(oracle):
    """The package's Input.hpp restatement and the oracle's agree exactly,
    and the 41^3 PMB elastic wave's value is 1.7311e-2."""
    dx = 1.0 / 41.0
    h = 3.0 * dx + 0.01 * dx
    a = critical_timestep(dx, dx, dx, 3, h, 1.0, 1.0)
    b = oracle.critical_timestep(dx, dx, dx, 3, h, 1.0, 1.0)
    assert a == b
    assert abs(a - 1.7311e-2) < 1e-6


def test_inputs_semantics(tmp_path):
    """CabanaPD_Input.hpp:30-128: derived keys for a deck."""
    deck = {
        "num_cells": {"value": [75, 151, 7]},
        "system_size": {"value": [0.1, 0.2, 0.009], "unit": "m"},
        "density": {"value": 8000}, "elastic_modulus": {"value": 191e9},
        "horizon": {"value": 0.002}, "final_time": {"value": 70e-6},
        "timestep": {"value": 1e-7}, "output_frequency": {"value": 50},
    }
    inp = Inputs(deck, export_file=str(tmp_path / "cabanaPD.in.json"))
    assert inp["num_steps"] == 700
    assert inp["m"] == 1
    assert inp["low_corner"] == [-0.05, -0.1, -0.0045]
    assert inp["timestep_safety_factor"] == 0.85
    assert inp["output_file"] == "cabanaPD.out"
    with pytest.raises(RuntimeError):
        Inputs(dict(deck, m={"value": 2}))


def _repulsion_pair(oracle, d, radius=0.45e-3, K=130e9, delta=4.17e-3, vol=1e-9):
    """Two particles a distance d apart along (1, 2, 2)/3 under normal
    repulsion alone (the contact-only form of the reference's model)."""
    e = np.array([1.0, 2.0, 2.0]) / 3.0
    x = np.array([[0.0, 0.0, 0.0], d * e])
    params = dict(pd_model=P.PD_NONE, contact_model=P.CONTACT_NORMAL_REPULSION,
                  contact_radius=radius, radius_extend=1e-5, contact_horizon=delta,
                  contact_K=K, dt=1e-9, rebuild_every=0)
    s = oracle.OracleSystem(params)
    s.set_particles(x, np.full(2, vol), np.full(2, 7800.0), np.zeros(2, np.int32), None)
    s.build_neighbors()
    s.init()
    return s, x


def test_normal_repulsion_force_law(oracle):
    """NormalRepulsionModel (force_models/CabanaPD_Contact.hpp:70-88) in
    Force<NormalRepulsionModel>::computeForceFull (force/CabanaPD_Contact.hpp:
    52-92): a pair closer than the contact radius gets ((15 c) sc) vol_j r_d /
    r with sc = (r - radius) / delta, c = 18 K / (pi delta^4), in that
    operation order; a pair inside the search radius but not closer than the
    contact radius gets nothing. The reference's own test of this model
    (unit_test/tstNormalRepulsion.hpp) only constructs it."""
    radius, K, delta, vol = 0.45e-3, 130e9, 4.17e-3, 1e-9
    c = 18.0 * K / (math.pi * delta * delta * delta * delta)
    for d in (0.2e-3, 0.4e-3):
        s, x = _repulsion_pair(oracle, d, radius, K, delta, vol)
        f = s.get("f")
        for i, j in ((0, 1), (1, 0)):
            r_vec = [(x[j, k] - x[i, k]) + (0.0 - 0.0) for k in range(3)]
            r = math.sqrt(r_vec[0] * r_vec[0] + r_vec[1] * r_vec[1] + r_vec[2] * r_vec[2])
            sc = (r - radius) / delta
            coeff = 15.0 * c * sc * vol
            want = [0.0 + coeff * r_vec[k] / r for k in range(3)]
            assert list(f[i]) == want, (d, i, f[i], want)
        # Repulsive: particle 0 is pushed away from particle 1.
        assert np.dot(f[0], x[1] - x[0]) < 0.0
    s, _ = _repulsion_pair(oracle, 0.5e-3, radius, K, delta, vol)
    assert s.neighbors()[0].tolist() == [1, 1]  # listed (search radius 0.91 mm) ...
    assert not np.any(s.get("f"))              # ... but beyond the contact radius


def test_pd_with_normal_repulsion_adds_forces(oracle):
    """Solver with a PD model and a contact model (CabanaPD_Solver.hpp:
    361-363): the contact force is added to the PD force of the same state
    (computeForce with reset = false). On a displaced fragmenting-cylinder
    state the hybrid force equals PD + repulsion within rounding, with the
    repulsion active. In a run at 200 m/s the contact list is rebuilt every
    step (largest displacement above the 0.01 dx search extension)."""
    prob = P.fragmenting_cylinder(num_cells=(40, 40, 20), size=(0.06, 0.06, 0.02),
                                  height=0.015, steps=12)
    rng = np.random.Generator(np.random.PCG64(7))
    u = rng.normal(0.0, 2e-5, size=prob["x"].shape)
    contact_keys = ("contact_model", "contact_horizon", "contact_K", "contact_radius",
                    "radius_extend", "rebuild_every")
    pd_only = {k: val for k, val in prob["params"].items() if k not in contact_keys}
    rep_only = dict(prob["params"], pd_model=P.PD_NONE, fracture=0)
    forces = []
    for params in (prob["params"], pd_only, rep_only):
        s = oracle.OracleSystem(params)
        s.set_particles(prob["x"], prob["vol"], prob["rho"], prob["nofail"], None)
        s.set_state(u, prob["v0"])
        s.build_neighbors()
        s.compute_force()
        forces.append(s.get("f"))
    f, f_pd, f_rep = forces
    assert np.any(f_rep) and np.any(f_pd)
    assert np.linalg.norm(f - (f_pd + f_rep)) <= 1e-13 * np.linalg.norm(f)

    hyb = oracle.OracleSystem(prob["params"])
    P.setup(hyb, prob)
    hyb.run(12)
    assert hyb.contact_rebuilds() == 12  # one per step (set-up's build is not counted)
