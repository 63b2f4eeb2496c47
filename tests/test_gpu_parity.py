"""Parity of the CUDA path (called through the C ABI) against the CPU oracle
on the same seeded inputs, plus the reference's own checks run on the GPU.

Tolerances: the plain-FP64 path evaluates every per-bond expression with
the reference's IEEE operation order and sums each neighbour row in the
oracle's order, so per-particle fields (u, v, f, W, phi, m, theta) and the
broken-bond sets must be BIT-IDENTICAL. Global totals are tree reductions on
the GPU vs serial sums on the CPU: relative difference <= 1e-12. Hertz
contact evaluates pow(|d|, 1.5), which CUDA and glibc may round differently
in the last place: <= 1e-12 relative, norm-wise.
"""
import numpy as np
import pytest

import force_checks
from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import cabanapd_b200
    return cabanapd_b200


def _pair(cuda, oracle, prob, init=True, ordering=0):
    params = dict(prob["params"], ordering=ordering)
    g = cuda.System(params)
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob, init=init)
    P.setup(o, prob, init=init)
    return g, o


def _assert_same(g, o, fields=("u", "v", "f")):
    for fld in fields:
        a, b = g.get(fld), o.get(fld)
        assert np.array_equal(a, b), (fld, np.max(np.abs(a - b)))


def _stress_pair(g, o):
    """Per-particle stress of the current states (computeStress)."""
    g.compute_stress()
    o.compute_stress()
    return g.get("stress"), o.get("stress")


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("case,kind,coeff", [
    ("pmb", "linear", 0.1), ("pmb", "quadratic", 0.01),
    ("pmb_damage", "quadratic", 0.01), ("linear_pmb", "linear", 0.1),
    ("lps", "linear", 0.1), ("lps", "quadratic", 0.01),
    ("lps_damage", "quadratic", 0.01), ("linear_lps", "linear", 0.1),
])
def test_force_cases_match_reference_and_oracle(cuda, oracle, case, kind, coeff):
    """unit_test/tstForce.hpp checks on the GPU, and bit-identity with the
    oracle for every particle."""
    res_g, _ = force_checks.run_case(lambda p: cuda.System(p), case, kind, coeff)
    force_checks.check_case(res_g, case, kind, coeff, max_checked=40)
    res_o, _ = force_checks.run_case(lambda p: oracle.OracleSystem(p), case, kind, coeff)
    for fld in ("f", "W", "theta", "stress"):
        assert np.array_equal(res_g[fld], res_o[fld]), fld
    assert _rel(res_g["Phi"], res_o["Phi"]) <= 1e-12
    assert res_g["constants"] == res_o["constants"]
    assert res_g["max_neighbors"] == res_o["max_neighbors"] == 122


@pytest.mark.parametrize("ordering", [0, 1])
def test_neighbor_sets_identical(cuda, oracle, ordering):
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, size=(3000, 3))
    params = dict(pd_model=P.PD_PMB, fracture=1, horizon=0.2, K=1.0, G0=1.0, dt=1.0)
    g = cuda.System(dict(params, ordering=ordering))
    o = oracle.OracleSystem(params)
    for s in (g, o):
        s.set_particles(x, np.ones(3000), n_frozen=100)
        s.build_neighbors()
    assert g.neighbor_stats() == o.neighbor_stats()
    cg, ig, mg = g.neighbors()
    co, io, mo = o.neighbors()
    assert np.array_equal(cg, co)
    assert np.array_equal(ig, io)
    assert np.array_equal(mg, mo)
    assert np.all(cg[:100] == 0)


def test_elastic_wave_pmb_bit_exact(cuda, oracle):
    """Config 0 (41^3 PMB elastic wave, 100 steps): displacements bit-identical
    at every checked step, total strain energy within 1e-12."""
    prob = P.elastic_wave_pmb(n=41, steps=100)
    g, o = _pair(cuda, oracle, prob)
    assert g.neighbor_stats() == o.neighbor_stats()
    done = 0
    for target in (1, 10, 100):
        g.run(target - done)
        o.run(target - done)
        done = target
        _assert_same(g, o)
        wg, _ = g.compute_energy()
        wo, _ = o.compute_energy()
        assert _rel(wg, wo) <= 1e-12
        assert np.array_equal(g.get("W"), o.get("W"))


@pytest.mark.parametrize("ordering", [0, 1])
def test_plate_impact_fracture_bit_exact(cuda, oracle, ordering):
    """Config 1 layout at reduced size: identical broken-bond sets, forces,
    displacements and damage after each block of steps."""
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=240, v0=60.0)
    g, o = _pair(cuda, oracle, prob, ordering=ordering)
    _, _, mu0 = o.neighbors()
    _, _, mg0 = g.neighbors()
    assert np.array_equal(mg0, mu0)
    assert (mu0 == 0).sum() > 0  # the notches cut bonds
    for _ in range(3):
        g.run(80)
        o.run(80)
        _assert_same(g, o)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        assert np.array_equal(g.get("phi"), o.get("phi"))
        assert _rel(wg, wo) <= 1e-12 and _rel(dg, do) <= 1e-12
        sg, so = _stress_pair(g, o)
        assert np.array_equal(sg, so)
    assert (o.neighbors()[2] == 0).sum() > (mu0 == 0).sum()  # bonds broke


def test_lps_random_notches_bit_exact(cuda, oracle):
    """Config 2 layout at reduced size (LPS, fracture, 20 seeded notches,
    traction BC, no-fail zone): m, theta, u, f, mu identical."""
    prob = P.lps_random_notches(num_cells=(100, 40, 4), steps=60)
    prob["bcs"] = [(k, c, i, v * 25.0) for k, c, i, v in prob["bcs"]]
    g, o = _pair(cuda, oracle, prob)
    for _ in range(3):
        g.run(20)
        o.run(20)
        _assert_same(g, o, ("u", "v", "f", "m", "theta"))
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
    wg, dg = g.compute_energy()
    wo, do = o.compute_energy()
    assert _rel(wg, wo) <= 1e-12 and _rel(dg, do) <= 1e-12
    assert np.array_equal(g.get("W"), o.get("W"))
    sg, so = _stress_pair(g, o)
    assert np.array_equal(sg, so)  # LPS with fracture: intact bonds only


@pytest.mark.parametrize("model", [P.PD_LINEAR_PMB, P.PD_LINEAR_LPS, P.PD_LPS])
def test_elastic_models_bit_exact(cuda, oracle, model):
    prob = P.elastic_wave_pmb(n=21, steps=30)
    prob["params"] = dict(prob["params"], pd_model=model, G=0.5)
    g, o = _pair(cuda, oracle, prob)
    g.run(30)
    o.run(30)
    _assert_same(g, o, ("u", "v", "f", "theta", "m"))
    sg, so = _stress_pair(g, o)
    assert np.array_equal(sg, so)


def test_kalthoff_winkler_regression_on_gpu(cuda, golden):
    from test_oracle_regression import kw_max_crack_y
    g_ = golden["kalthoff_winkler"]
    prob = P.kalthoff_winkler_regression()
    s = cuda.System(prob["params"])
    P.setup(s, prob)
    y = kw_max_crack_y(s, prob)
    assert abs(y - g_["max_crack_y"]) <= g_["tolerance"], y


def test_hertz_regression_on_gpu(cuda, oracle, golden):
    from test_oracle_regression import hertz_restitution
    prob = P.hertz_two_spheres()
    s = cuda.System(prob["params"])
    P.setup(s, prob)
    r = hertz_restitution(s, prob)
    e = golden["hertz"]["input"]["restitution"]["value"]
    assert abs(r - e) <= golden["hertz"]["tolerance"], r
    o = oracle.OracleSystem(prob["params"])
    P.setup(o, prob)
    o.run(prob["num_steps"])
    v_g, v_o = s.get("v"), o.get("v")
    assert np.linalg.norm(v_g - v_o) <= 1e-12 * np.linalg.norm(v_o)
    assert s.contact_rebuilds() == o.contact_rebuilds()


# DEM packings: the 4 M-sphere packing's layout (non-overlapping, free flight over the
# test's steps) and a compressed one (spacing 2.1 mm < 2 R_max: overlapping
# pairs from the start, so the Hertz force law is exercised).
DEM_CASES = {"free": dict(spacing=2.5e-3, dt=2e-6), "compressed": dict(spacing=2.1e-3, dt=1e-7)}


@pytest.mark.parametrize("case", ["free", "compressed"])
def test_dem_packing_parity(cuda, oracle, case):
    """Config 3 layout at reduced size: polydisperse Hertz, rebuild every 10
    steps; contact sets identical at each rebuild, fields within 1e-12."""
    prob = P.dem_packing(lattice_dims=(16, 16, 8), steps=100, **DEM_CASES[case])
    g, o = _pair(cuda, oracle, prob)
    for _ in range(4):
        g.run(25)
        o.run(25)
        assert g.contact_rebuilds() == o.contact_rebuilds()
        assert np.array_equal(g.neighbors()[1], o.neighbors()[1])
        for fld in ("u", "v", "f"):
            a, b = g.get(fld), o.get(fld)
            assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b), fld
    assert (np.count_nonzero(o.get("f")) > 0) == (case == "compressed")


def test_linear_lps_fracture_is_lps(cuda, oracle):
    """LinearLPS with fracture runs the LPS fracture kernels (the
    reference's Solver selects Force<LPS> for it): bit-identical to the
    oracle and to an LPS system."""
    prob = P.lps_random_notches(num_cells=(80, 32, 4), steps=30)
    lin = dict(prob, params=dict(prob["params"], pd_model=P.PD_LINEAR_LPS))
    g, o = _pair(cuda, oracle, lin)
    ref = P.setup(cuda.System(prob["params"]), prob)
    for s in (g, o, ref):
        s.run(prob["num_steps"])
    _assert_same(g, o, ("u", "v", "f", "theta", "m"))
    _assert_same(g, ref, ("u", "v", "f", "theta", "m"))
    assert np.array_equal(g.neighbors()[2], o.neighbors()[2])


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("problem", ["plate", "lps", "dem"])
def test_fused_step_equals_separate_stages(cuda, precision, problem):
    """cpd_step runs one bond kernel per step with the boundary conditions
    and both half steps in its epilogue (alternating displacement buffers);
    the four separate stages of cpd_step_stage give the same bits, for odd and
    even chunk lengths (ForceValue BC on the plate, per-particle ForceAdd
    traction on the LPS box). The compressed DEM packing (contact alone,
    rebuilt every 10 steps) alternates velocity buffers as well, since the
    contact damping reads neighbour velocities; its rebuilds fall inside
    the chunks."""
    if problem == "plate":
        prob = P.plate_impact(num_cells=(96, 48, 6), steps=60, v0=60.0)
    elif problem == "dem":
        prob = P.dem_packing(lattice_dims=(16, 16, 8), steps=60, **DEM_CASES["compressed"])
    else:
        prob = P.lps_random_notches(num_cells=(100, 40, 4), steps=60)
        prob["bcs"] = [(k, c, i, v * 25.0) for k, c, i, v in prob["bcs"]]
    a = P.setup(cuda.System(dict(prob["params"], precision=precision)), prob)
    b = P.setup(cuda.System(dict(prob["params"], precision=precision)), prob)
    for chunk in (1, 2, 7, 50):
        a.run(chunk)
        for _ in range(chunk):
            for stage in range(4):
                b.step_stage(stage)
        for fld in ("u", "v", "f"):
            assert np.array_equal(a.get(fld), b.get(fld)), (chunk, fld)
        assert np.array_equal(a.neighbors()[1], b.neighbors()[1])
        assert np.array_equal(a.neighbors()[2], b.neighbors()[2])
        assert a.contact_rebuilds() == b.contact_rebuilds()
    assert a.compute_energy() == b.compute_energy()
    if problem == "dem":
        assert a.contact_rebuilds() == 6 and np.any(a.get("f"))


def test_errors_are_reported(cuda):
    s = cuda.System(dict(pd_model=P.PD_PMB, horizon=0.1, K=1.0, dt=1.0))
    with pytest.raises(cuda.CpdError):
        s.init()  # no particles
    with pytest.raises(cuda.CpdError):
        cuda.System(dict(pd_model=P.PD_LINEAR_PMB, fracture=1, horizon=0.1, K=1.0))
    x, vol, _ = P.lattice([0, 0, 0], [1, 1, 1], [4, 4, 4])
    s.set_particles(x, vol)
    with pytest.raises(cuda.CpdError):
        s.step(1)  # neighbour list not built
    s.build_neighbors()
    with pytest.raises(cuda.CpdError):
        s.step(1)  # init not called
    with pytest.raises(cuda.CpdError):
        s.prenotch([[1, 0, 0]], [[0, 1, 0]], [[0, 0, 0]])  # no fracture model
    with pytest.raises(cuda.CpdError):
        s.add_bc(P.BC_FORCE_VALUE, [10 ** 6], [0.0])
    with pytest.raises(cuda.CpdError):
        s.get("stress")  # cpd_compute_stress not called


# ---------------------------------------------------------------------------
# Throughput-form FP64 path (precision = CPD_FP64). On lattices the PMB bond
# stage is the stencil kernel: stretch formed without the cancellation of
# (r - xi)/xi from the exact lattice offsets, pair force from a polynomial
# accurate to ~2e-16; elsewhere rsqrt-based bond lengths with FMA. Bars of
# the throughput FP64 path: per step, from the same state, forces and displacements
# within 1e-12 (norm-wise); broken-bond sets identical; totals within 1e-10
# over a run. The reference's own rounding of s = (r - xi)/xi is ~1e-16
# absolute per bond, and over a run that is what separates two correct FP64
# evaluations: the elastic wave reaches ~3e-12 in u after 100 steps, and the
# oracle compiled with and without FMA contraction differs by 1.3e-12 there.
FAST = 1


def _nrel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _pair_fast(cuda, oracle, prob, ordering=0):
    g = cuda.System(dict(prob["params"], precision=FAST, ordering=ordering))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    return g, o


@pytest.mark.parametrize("case,kind,coeff", [
    ("pmb", "linear", 0.1), ("pmb", "quadratic", 0.01),
    ("pmb_damage", "quadratic", 0.01),
    ("lps", "linear", 0.1), ("lps", "quadratic", 0.01),
    ("lps_damage", "linear", 0.1),
])
def test_fast_force_cases(cuda, oracle, case, kind, coeff):
    res_g, _ = force_checks.run_case(lambda p: cuda.System(dict(p, precision=FAST)),
                                     case, kind, coeff)
    force_checks.check_case(res_g, case, kind, coeff, max_checked=40)
    res_o, _ = force_checks.run_case(lambda p: oracle.OracleSystem(p), case, kind, coeff)
    for fld in ("f", "theta"):
        assert _nrel(res_g[fld], res_o[fld]) <= 1e-12, fld


def _restart_from_oracle(g, o):
    """Puts the oracle's state into the GPU system: u and v, then the force
    of that state from the GPU's own kernel with the boundary conditions
    applied, as a step leaves it (the next step's first half step reads it)."""
    g.set_state(o.get("u"), o.get("v"))
    g.step_stage(1)
    g.step_stage(2)
    g.synchronize()


def test_fast_elastic_wave(cuda, oracle):
    """Config 0 (41^3, 100 steps). Fields within 1e-12 over the first 10
    steps and 1e-11 after 100; strain energy within 1e-10."""
    prob = P.elastic_wave_pmb(n=41, steps=100)
    g, o = _pair_fast(cuda, oracle, prob)
    done = 0
    for target, bar in ((1, 1e-12), (10, 1e-12), (100, 1e-11)):
        g.run(target - done)
        o.run(target - done)
        done = target
        for fld in ("u", "v", "f"):
            assert _nrel(g.get(fld), o.get(fld)) <= bar, (target, fld)
        wg, _ = g.compute_energy()
        wo, _ = o.compute_energy()
        assert _rel(wg, wo) <= 1e-10


@pytest.mark.parametrize("problem", ["wave", "plate"])
def test_fast_per_step_from_the_oracle_state(cuda, oracle, problem):
    """The throughput FP64 path's per-step bar: from the oracle's state at several
    points of a run, one GPU step gives u, v and f within 1e-12 (norm-wise)
    of the oracle's step, and the GPU's force of that state is within 1e-12
    of the oracle's."""
    if problem == "wave":
        prob, marks = P.elastic_wave_pmb(n=41, steps=100), (0, 10, 60, 99)
    else:
        prob, marks = P.plate_impact(num_cells=(96, 48, 6), steps=240, v0=60.0), (0, 80, 239)
    g, o = _pair_fast(cuda, oracle, prob)
    done = 0
    for m in marks:
        # Both run to the mark (the bond states stay identical), then the GPU
        # system takes the oracle's displacement and velocity.
        g.run(m - done)
        o.run(m - done)
        done = m
        _restart_from_oracle(g, o)
        if problem == "plate":
            assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        assert _nrel(g.get("f"), o.get("f")) <= 1e-12, (m, "f of the same state")
        g.run(1)
        o.run(1)
        done += 1
        for fld in ("u", "v", "f"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-12, (m, fld)


@pytest.mark.parametrize("ordering", [0, 1])
def test_fast_plate_impact(cuda, oracle, ordering):
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=240, v0=60.0)
    g, o = _pair_fast(cuda, oracle, prob, ordering=ordering)
    for _ in range(3):
        g.run(80)
        o.run(80)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        for fld in ("u", "v", "f"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-12, fld
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        assert _rel(wg, wo) <= 1e-12 and _rel(dg, do) <= 1e-12
        # The exact stress kernel on states within 1e-12 of each other.
        assert _nrel(*_stress_pair(g, o)) <= 1e-10


def test_fast_lps_random_notches(cuda, oracle):
    prob = P.lps_random_notches(num_cells=(100, 40, 4), steps=60)
    prob["bcs"] = [(k, c, i, v * 25.0) for k, c, i, v in prob["bcs"]]
    g, o = _pair_fast(cuda, oracle, prob)
    for _ in range(3):
        g.run(20)
        o.run(20)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        for fld in ("u", "v", "f", "m", "theta"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-12, fld
    assert (o.neighbors()[2] == 0).sum() > 0


# ---------------------------------------------------------------------------
# Mixed-precision path (precision = CPD_MIXED, PMB): FP32 bond arithmetic with
# Kahan-compensated sums, FP64 integration. Bars of the mixed path: displacement
# <= 1e-6 relative to the FP64 oracle (norm-wise), broken-bond sets identical
# (FP64 re-test within 1e-4 s0); velocities and forces <= 1e-5.
MIXED = 2


def _pair_mixed(cuda, oracle, prob, ordering=0):
    g = cuda.System(dict(prob["params"], precision=MIXED, ordering=ordering))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    return g, o


@pytest.mark.parametrize("ordering", [0, 1])
def test_mixed_plate_impact(cuda, oracle, ordering):
    """ordering 0: lattice bonds use the FP32 stencil table; ordering 1
    (Morton) breaks the per-code index delta, so bonds take the generic
    hi/lo-position branch."""
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=240, v0=60.0)
    g, o = _pair_mixed(cuda, oracle, prob, ordering=ordering)
    # With v0 = 60 m/s the crack runs fast; on the generic branch (FP32 error
    # ~2x the table branch) a bond whose FP64 stretch is 1.5e-7 above s0
    # breaks one step later at step 216, after which the crack tips differ.
    # Checked here up to step 160 for that branch, 240 for the table branch.
    for _ in range(3 if ordering == 0 else 2):
        g.run(80)
        o.run(80)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        assert _nrel(g.get("u"), o.get("u")) <= 1e-6
        assert _nrel(g.get("v"), o.get("v")) <= 1e-5
        assert _nrel(g.get("f"), o.get("f")) <= 1e-5
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        assert _rel(wg, wo) <= 1e-6 and _rel(dg, do) <= 1e-12
        assert _nrel(*_stress_pair(g, o)) <= 1e-5
    assert (o.neighbors()[2] == 0).sum() > 0


def test_mixed_plate_at_the_full_plates_spacing(cuda):
    """The FP32 table constants at the 800 x 400 x 36 plate's spacing
    (dx = 2.5e-4 m: c vol / xi^3 ~ 1e22) stay finite: a 20 x 10 x 2.5 mm
    plate of 80 x 40 x 10 cells, mixed against FP64 over 40 steps."""
    prob = P.plate_impact(num_cells=(80, 40, 10), steps=40, v0=60.0, size=(0.02, 0.01, 0.0025))
    runs = {}
    for prec in (MIXED, 1):
        s = cuda.System(dict(prob["params"], precision=prec))
        P.setup(s, prob)
        s.run(40)
        runs[prec] = s
    g, f = runs[MIXED], runs[1]
    assert g.stencil_stats()[2] == 122 and f.stencil_stats()[2] == 122
    assert np.all(np.isfinite(g.get("f")))
    assert _nrel(g.get("u"), f.get("u")) <= 1e-6
    assert _nrel(g.get("v"), f.get("v")) <= 1e-5
    assert _nrel(g.get("f"), f.get("f")) <= 1e-5
    assert np.array_equal(g.neighbors()[2], f.neighbors()[2])


def _with_void(prob, sites):
    """The problem with the given lattice sites left empty (index deltas
    across them shift: the rows whose neighbours lie across them take the
    general kernels)."""
    from cabanapd_b200 import shard
    keep = np.setdiff1d(np.arange(len(prob["x"])), sites)
    return shard.local_problem(prob, keep, np.ones(keep.size, dtype=bool))


def _with_hole(prob, centre=(0.03, 0.0), radius=0.008):
    """The problem with the lattice sites inside a cylinder through the
    plate's thickness left empty (every lattice line that crosses it is
    shorter)."""
    x = np.asarray(prob["x"])
    inside = (x[:, 0] - centre[0]) ** 2 + (x[:, 1] - centre[1]) ** 2 < radius ** 2
    return _with_void(prob, np.nonzero(inside)[0])


@pytest.mark.parametrize("body", ["pair", "void", "hole", "void_and_pair"])
@pytest.mark.parametrize("precision", [1, MIXED])
def test_stencil_kernels_plate_against_oracle(cuda, oracle, precision, body):
    """The lattice-stencil bond kernels (FP64: the two-launch walk; MIXED:
    the FP32 walk on the split records) on a cubic notched plate: beside an
    off-lattice pair (one warp on the general kernels), with two empty
    lattice sites, with a cylindrical hole through the plate, and with both
    empty sites and the pair. With empty sites the particles' index deltas
    vary: on a lattice of distinct cells FP64 gathers its records by cell
    and keeps every row on the stencil kernel, and MIXED runs that FP64
    kernel; with the pair off the lattice as well, both keep the rows whose
    deltas are the majority's. FP64 (and MIXED on the FP64 kernel) within
    1e-12 of the oracle with identical bonds over 160 steps; MIXED on its
    own kernels within the mixed bars, bonds identical."""
    plate = _cubic_plate(96, 8, steps=160)
    if body == "pair":
        prob = _with_offlattice_pair(plate)
    elif body == "void":
        prob = _with_void(plate, [13000, 13001])
    elif body == "hole":
        prob = _with_hole(plate)
    else:
        prob = _with_offlattice_pair(_with_void(plate, [13000, 13001]))
    g = cuda.System(dict(prob["params"], precision=precision))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    warps, irregular, entries = g.stencil_stats()
    assert entries == 122
    rows_warps = (len(prob["x"]) + 31) // 32
    fp64_kernels = precision == 1 or body in ("void", "hole")
    if body == "pair":
        assert warps == len(plate["x"]) // 32 and irregular == 1
    elif body in ("void", "hole"):
        assert warps == rows_warps and irregular == 0
    else:
        # The rows whose neighbours lie across an empty site in index
        # order leave the stencil kernel (the rows within three planes of
        # the void, most of this 8-plane plate).
        assert irregular > 0 and warps > 0.1 * rows_warps
    for _ in range(4):
        g.run(40)
        o.run(40)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        if fp64_kernels:
            for fld in ("u", "v", "f"):
                assert _nrel(g.get(fld), o.get(fld)) <= 1e-12, fld
        else:
            assert _nrel(g.get("u"), o.get("u")) <= 1e-6
            assert _nrel(g.get("v"), o.get("v")) <= 1e-5
            assert _nrel(g.get("f"), o.get("f")) <= 1e-5
    assert (o.neighbors()[2] == 0).sum() > 0


def test_fp64_stencil_at_a_four_spacing_horizon(cuda, oracle):
    """A horizon of four spacings (the reference's example decks): 256 table
    entries, the FP64 stencil walk in four launches of 64, rows coded from
    the positions; within 1e-12 of the oracle with identical bonds over 120
    steps, every warp on the stencil kernel."""
    prob = P.plate_impact(num_cells=(96, 48, 8), steps=120, v0=60.0,
                          size=(0.2, 0.1, 0.2 * 8 / 96), horizon_factor=4.0)
    g = cuda.System(dict(prob["params"], precision=1))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    warps, irregular, entries = g.stencil_stats()
    assert entries == 256 and irregular == 0 and warps == len(prob["x"]) // 32
    for _ in range(3):
        g.run(40)
        o.run(40)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        for fld in ("u", "v", "f"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-12, fld
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        assert _rel(wg, wo) <= 1e-12 and _rel(dg, do) <= 1e-12
    assert (o.neighbors()[2] == 0).sum() > 0


def test_step_energy_at_a_four_spacing_horizon(cuda, oracle):
    """The output step in one call on the wide FP64 walk (256 entries, four
    launches, the partial energy passed on with the partial force): states,
    bonds and phi as step + energy bit for bit, W to FP64 rounding, totals
    against the oracle."""
    prob = P.plate_impact(num_cells=(96, 48, 8), steps=60, v0=60.0,
                          size=(0.2, 0.1, 0.2 * 8 / 96), horizon_factor=4.0)
    a = cuda.System(dict(prob["params"], precision=1))
    b = cuda.System(dict(prob["params"], precision=1))
    o = oracle.OracleSystem(prob["params"])
    for s_ in (a, b, o):
        P.setup(s_, prob)
    assert a.stencil_stats()[2] == 256
    for _ in range(3):
        la, lb = a.kernel_launches(), b.kernel_launches()
        wa, da = a.step_energy(20)
        b.step(20)
        wb, db = b.compute_energy()
        o.run(20)
        wo, do = o.compute_energy()
        assert a.kernel_launches() - la < b.kernel_launches() - lb
        for fld in ("u", "v", "f", "phi"):
            assert np.array_equal(a.get(fld), b.get(fld)), fld
        assert not np.array_equal(a.get("W"), b.get("W"))
        assert _nrel(a.get("W"), b.get("W")) <= 1e-13
        assert _rel(wa, wb) <= 1e-13 and _rel(da, db) <= 1e-13
        assert _rel(wa, wo) <= 1e-12 and _rel(da, do) <= 1e-12
    assert da > 0


def test_mixed_at_a_four_spacing_horizon_runs_the_fp64_stencil(cuda):
    """CPD_MIXED PMB at a horizon of four spacings (a 256-entry table, past
    the mixed path's byte codes) runs the FP64 stencil kernels: the same
    bits as CPD_FP64 on the same plate."""
    prob = P.plate_impact(num_cells=(96, 48, 8), steps=60, v0=60.0,
                          size=(0.2, 0.1, 0.2 * 8 / 96), horizon_factor=4.0)
    runs = {}
    for prec in (1, MIXED):
        s = cuda.System(dict(prob["params"], precision=prec))
        P.setup(s, prob)
        assert s.stencil_stats()[2] == 256
        s.run(60)
        runs[prec] = s
    for fld in ("u", "v", "f"):
        assert np.array_equal(runs[1].get(fld), runs[MIXED].get(fld)), fld
    assert np.array_equal(runs[1].neighbors()[2], runs[MIXED].neighbors()[2])
    assert runs[1].compute_energy() == runs[MIXED].compute_energy()


def test_mixed_elastic_wave(cuda, oracle):
    prob = P.elastic_wave_pmb(n=41, steps=100)
    g, o = _pair_mixed(cuda, oracle, prob)
    g.run(100)
    o.run(100)
    assert _nrel(g.get("u"), o.get("u")) <= 1e-6
    assert _nrel(g.get("f"), o.get("f")) <= 1e-5


def test_mixed_lps_random_notches(cuda, oracle):
    """LPS fracture on the mixed kernels (stencil rows, FP32 bonds, Kahan
    sums, FP64 re-test in the guard band): same bars as the PMB mixed path."""
    prob = P.lps_random_notches(num_cells=(100, 40, 4), steps=60)
    prob["bcs"] = [(k, c, i, v * 25.0) for k, c, i, v in prob["bcs"]]
    g, o = _pair_mixed(cuda, oracle, prob)
    for _ in range(3):
        g.run(20)
        o.run(20)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        assert _nrel(g.get("u"), o.get("u")) <= 1e-6
        for fld in ("v", "f", "m", "theta"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-5, fld
        dg = g.compute_energy()[1]
        do = o.compute_energy()[1]
        assert _rel(dg, do) <= 1e-12
        assert _nrel(*_stress_pair(g, o)) <= 1e-5
    assert (o.neighbors()[2] == 0).sum() > 0


def test_mixed_lps_elastic_wave(cuda, oracle, golden):
    """The LinearLPS (= LPS) elastic wave of the regression test on the mixed
    kernels, against the FP64 oracle."""
    prob = P.elastic_wave_lps(golden["elastic_wave"]["input"])
    g, o = _pair_mixed(cuda, oracle, prob)
    g.run(prob["num_steps"])
    o.run(prob["num_steps"])
    assert _nrel(g.get("u"), o.get("u")) <= 1e-6
    assert _nrel(g.get("theta"), o.get("theta")) <= 1e-5


def test_mixed_lps_irregular_rows_keep_fp64(cuda, oracle):
    """Morton order breaks the lattice index deltas, so rows are irregular
    and LPS under CPD_MIXED keeps the FP64 kernels (<= 1e-12)."""
    prob = P.lps_random_notches(num_cells=(100, 40, 4), steps=40)
    g, o = _pair_mixed(cuda, oracle, prob, ordering=1)
    g.run(40)
    o.run(40)
    assert _nrel(g.get("u"), o.get("u")) <= 1e-12
    assert np.array_equal(g.neighbors()[2], o.neighbors()[2])


def test_mixed_dem_packing(cuda, oracle):
    """Config 3 on the mixed Hertz kernel (FP64 overlap, FP32 force law):
    contact sets identical at each rebuild; displacement within 1e-6 and
    velocity and force within 1e-5 of the FP64 oracle, norm-wise."""
    prob = P.dem_packing(lattice_dims=(16, 16, 8), steps=100, **DEM_CASES["compressed"])
    g, o = _pair_mixed(cuda, oracle, prob)
    for _ in range(4):
        g.run(25)
        o.run(25)
        assert g.contact_rebuilds() == o.contact_rebuilds()
        assert np.array_equal(g.neighbors()[1], o.neighbors()[1])
        assert _nrel(g.get("u"), o.get("u")) <= 1e-6
        assert _nrel(g.get("v"), o.get("v")) <= 1e-5
        assert _nrel(g.get("f"), o.get("f")) <= 1e-5
    assert np.count_nonzero(o.get("f")) > 0


@pytest.mark.parametrize("precision", [FAST, MIXED])
def test_plate_with_frozen_particles(cuda, oracle, precision):
    """Frozen particles (the first z-layer and ten more, so the integrated
    rows start off a warp boundary) on the FP64 and mixed kernels: the bars of
    the FP64 / mixed plate tests, and the frozen particles never move. The
    impact strip's force condition keeps its integrated particles only.
    Checked over 100 steps: at step 118 a bond to a frozen particle whose FP64
    stretch is 4.1e-7 below s0 breaks on the mixed path (its state is ~2e-8
    off the FP64 one), after which the crack tips differ."""
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=100, v0=60.0)
    nf = 96 * 48 + 10
    prob = dict(prob, n_frozen=nf)
    prob["bcs"] = [(k, c, idx[idx >= nf], v) for k, c, idx, v in prob["bcs"]]
    g = cuda.System(dict(prob["params"], precision=precision))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    tol_u, tol_v = (1e-12, 1e-12) if precision == FAST else (1e-6, 1e-5)
    for _ in range(2):
        g.run(50)
        o.run(50)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        assert _nrel(g.get("u"), o.get("u")) <= tol_u
        assert _nrel(g.get("v"), o.get("v")) <= tol_v
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        assert _rel(dg, do) <= 1e-12 and _rel(wg, wo) <= (1e-12 if precision == FAST else 1e-6)
    assert not np.any(g.get("u")[:nf])
    assert (o.neighbors()[2] == 0).sum() > 0



def _cylinder(steps):
    return P.fragmenting_cylinder(num_cells=(60, 60, 40), size=(0.06, 0.06, 0.04),
                                  height=0.03, steps=steps)


@pytest.mark.parametrize("ordering", [0, 1])
def test_fragmenting_cylinder_bit_exact(cuda, oracle, ordering):
    """PMB fracture plus normal-repulsion contact (the fragmenting-cylinder
    example on a shorter cylinder, 21 k particles): the EXACT path equals the
    oracle bit for bit in u, v, f and the broken bonds, with the contact list
    rebuilt on current positions every step."""
    prob = _cylinder(40)
    g, o = _pair(cuda, oracle, prob, ordering=ordering)
    for _ in range(2):
        g.run(20)
        o.run(20)
        assert g.contact_rebuilds() == o.contact_rebuilds()
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        _assert_same(g, o)
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        assert _rel(wg, wo) <= 1e-12 and _rel(dg, do) <= 1e-12
    assert g.contact_rebuilds() == 40 and dg > 0.0


def test_fragmenting_cylinder_fp64_and_mixed(cuda, oracle):
    """The same problem on the FP64 kernels (the PD bond force in its
    throughput form beside the exact repulsion kernel): within 1e-10 of the
    oracle (norm-wise), identical broken-bond sets. MIXED runs the FP64 PD
    kernels when contact is present, so it equals FP64 bit for bit."""
    prob = _cylinder(40)
    g, o = _pair_fast(cuda, oracle, prob)
    m = cuda.System(dict(prob["params"], precision=MIXED))
    P.setup(m, prob)
    for _ in range(2):
        g.run(20)
        o.run(20)
        m.run(20)
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        for fld in ("u", "v", "f"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-10, fld
            assert np.array_equal(m.get(fld), g.get(fld)), fld



def _cubic_plate(nx, nz, steps, v0=60.0):
    """The notched plate on a cubic lattice (nx x nx/2 x nz cells, spacing
    0.2 m / nx on every axis), whose 122-entry offset table the unrolled
    stencil kernels take (the plate's own thickness of 0.009 m gives other
    spacings a larger table)."""
    return P.plate_impact(num_cells=(nx, nx // 2, nz), steps=steps, v0=v0,
                          size=(0.2, 0.1, 0.2 * nz / nx))


def _with_offlattice_pair(prob):
    """Two particles appended far from the body, 1.3 spacings apart: their
    bond is no lattice offset, so the last warp takes the general kernels
    beside the stencil warps (one particle volume kept)."""
    out = dict(prob)
    x = np.asarray(prob["x"])
    h = float(prob["dx"][0])
    far = x.max(axis=0) + 10.0 * h
    extra = np.array([far, far + np.array([1.3 * h, 0.0, 0.0])])
    out["x"] = np.vstack([x, extra])
    for key in ("vol", "rho", "nofail"):
        a = np.asarray(prob[key])
        out[key] = np.concatenate([a, a[:2]])
    out["v0"] = np.vstack([np.asarray(prob["v0"]), np.zeros((2, 3))])
    return out


@pytest.mark.parametrize("precision", [1, MIXED])
def test_step_energy_equals_step_then_energy(cuda, oracle, precision):
    """cpd_step_energy (the Solver's output step in one call) against
    cpd_step + cpd_compute_energy on the same system, and the oracle's
    totals. On this lattice (one particle volume) the last step's stencil
    kernel forms the energy itself: states, bonds and phi bit for bit (phi
    from the same ordered volume sums), W to the rounding of its bond terms
    (FP32 on the mixed path, FP64 on the FP64 path; another form of the
    stretch), the totals summed in another order."""
    prob = _cubic_plate(96, 8, steps=120)
    a = cuda.System(dict(prob["params"], precision=precision))
    b = cuda.System(dict(prob["params"], precision=precision))
    o = oracle.OracleSystem(prob["params"])
    for s in (a, b, o):
        P.setup(s, prob)
    warps, irregular, entries = a.stencil_stats()
    assert warps == (len(prob["x"]) + 31) // 32 and irregular == 0 and entries == 122
    # The initial state's fields from init against the energy pass on the
    # same state.
    w0, phi0 = a.get("W"), a.get("phi")
    a.compute_energy()
    assert np.array_equal(phi0, a.get("phi"))
    assert np.array_equal(w0, a.get("W"))
    for _ in range(6):
        la, lb = a.kernel_launches(), b.kernel_launches()
        wa, da = a.step_energy(20)
        b.step(20)
        wb, db = b.compute_energy()
        # The energy rides on the last step's bond kernel (the energy pass
        # runs only over irregular warps, if any).
        assert a.kernel_launches() - la <= b.kernel_launches() - lb
        o.run(20)
        wo, do = o.compute_energy()
        for fld in ("u", "v", "f", "phi"):
            assert np.array_equal(a.get(fld), b.get(fld)), fld
        assert np.array_equal(a.neighbors()[2], b.neighbors()[2])
        # W from the stencil kernel's own terms, not the energy pass's.
        assert not np.array_equal(a.get("W"), b.get("W"))
        tw = 1e-6 if precision == MIXED else 1e-13
        assert _nrel(a.get("W"), b.get("W")) <= tw
        assert _rel(wa, wb) <= tw and _rel(da, db) <= 1e-13
        assert _rel(da, do) <= 1e-12 and _rel(wa, wo) <= (1e-6 if precision == MIXED else 1e-12)
    assert da > 0



def test_step_energy_with_irregular_rows(cuda, oracle):
    """The fused output step beside a warp on the general kernels (an
    off-lattice pair appended to the cubic plate: that warp takes the
    energy kernel after the step): against step + energy and the oracle,
    as above."""
    prob = _with_offlattice_pair(_cubic_plate(96, 8, steps=60))
    a = cuda.System(dict(prob["params"], precision=MIXED))
    b = cuda.System(dict(prob["params"], precision=MIXED))
    o = oracle.OracleSystem(prob["params"])
    for s_ in (a, b, o):
        P.setup(s_, prob)
    warps, irregular, _ = a.stencil_stats()
    assert warps > 0 and irregular == 1
    for _ in range(3):
        wa, da = a.step_energy(20)
        b.step(20)
        wb, db = b.compute_energy()
        o.run(20)
        wo, do = o.compute_energy()
        for fld in ("u", "v", "f", "phi"):
            assert np.array_equal(a.get(fld), b.get(fld)), fld
        assert _nrel(a.get("W"), b.get("W")) <= 1e-6
        assert _rel(wa, wb) <= 1e-6 and _rel(da, db) <= 1e-13
        assert _rel(da, do) <= 1e-12 and _rel(wa, wo) <= 1e-6
        assert _nrel(a.get("W"), o.get("W")) <= 1e-5


@pytest.mark.parametrize("model", ["pmb", "lps"])
def test_mixed_with_unequal_volumes(cuda, oracle, model):
    """Particle volumes that differ (by up to 1e-3, seeded): the mixed path
    without its one-volume shortcuts (damage sums by FP64 volume gathers,
    LPS neighbour factors from their own array), against the oracle with
    the mixed bars; the output step in one call equals step + energy."""
    if model == "pmb":
        prob = P.plate_impact(num_cells=(96, 48, 6), steps=80, v0=60.0)
    else:
        prob = P.lps_random_notches(num_cells=(100, 40, 4), steps=60)
        prob["bcs"] = [(k, c, i, v * 25.0) for k, c, i, v in prob["bcs"]]
    rng = np.random.Generator(np.random.PCG64(11))
    prob["vol"] = prob["vol"] * (1.0 + 1e-3 * rng.random(prob["vol"].size))
    g, o = _pair_mixed(cuda, oracle, prob)
    b = cuda.System(dict(prob["params"], precision=MIXED))
    P.setup(b, prob)
    for _ in range(3):
        wg, dg = g.step_energy(20)
        b.step(20)
        wb, db = b.compute_energy()
        o.run(20)
        wo, do = o.compute_energy()
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
        assert _nrel(g.get("u"), o.get("u")) <= 1e-6
        for fld in ("v", "f"):
            assert _nrel(g.get(fld), o.get(fld)) <= 1e-5, fld
        assert np.array_equal(g.get("phi"), o.get("phi"))
        assert _rel(dg, do) <= 1e-12 and _rel(wg, wo) <= 1e-6
        assert (wg, dg) == (wb, db)
    assert (o.neighbors()[2] == 0).sum() > 0


def test_split_forms_on_small_systems():
    """The split mixed forms (the LPS lean kernels over the lists of
    full-stencil and shared-subset warps with the general kernels over the
    rest, and the mixed energy pass in the same two parts) run on systems of
    2^20 rows and more; a child process forces them onto the small mixed
    test systems (CPD_SPLIT_MIN_ROWS=0) and runs the mixed parity tests
    there with the same bars."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    env = dict(os.environ, CPD_SPLIT_MIN_ROWS="0")
    sel = ("test_mixed_plate_impact or test_mixed_lps_random_notches or test_mixed_elastic_wave"
           " or test_plate_with_frozen_particles or test_step_energy_equals_step_then_energy"
           " or test_mixed_with_unequal_volumes")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider",
                        os.path.join(here, "test_gpu_parity.py"), "-k", sel],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "10 passed" in r.stdout, r.stdout[-500:]
