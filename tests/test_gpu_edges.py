"""Edge cases of the CUDA path against the oracle: a lone particle, isolated
particles beside a body, row counts that are not multiples of a warp, a
body with every bond cut, most particles frozen, zero steps, and a horizon
of five spacings (rows past four bond words, a stencil too large for the
lean forms). EXACT must equal the oracle bit for bit, FP64 within 1e-12,
MIXED within the mixed bars (u 1e-6, v and f 1e-5), with identical bonds.
"""
import numpy as np
import pytest

from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu

EXACT, FAST, MIXED = 0, 1, 2
TOL = {EXACT: (0.0, 0.0), FAST: (1e-12, 1e-12), MIXED: (1e-6, 1e-5)}


@pytest.fixture(scope="module")
def cuda():
    import cabanapd_b200
    return cabanapd_b200


def _nrel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _check(g, o, precision, tol_fields=None):
    tu, tf = TOL[precision]
    tols = {"u": tu, "v": tf, "f": tf}
    tols.update(tol_fields or {})
    for fld in ("u", "v", "f"):
        a, b, tol = g.get(fld), o.get(fld), tols[fld]
        if tol == 0.0:
            assert np.array_equal(a, b), fld
        else:
            assert _nrel(a, b) <= tol, (fld, _nrel(a, b))
    if g.neighbor_stats()[1] > 0:
        assert np.array_equal(g.neighbors()[2], o.neighbors()[2])
    wg, dg = g.compute_energy()
    wo, do = o.compute_energy()
    assert np.array_equal(g.get("phi"), o.get("phi"), equal_nan=True)
    assert (np.isnan(dg) and np.isnan(do)) or abs(dg - do) <= 1e-12 * max(abs(do), 1.0)
    assert abs(wg - wo) <= max(tu, 1e-12) * max(abs(wo), 1e-300) or wg == wo


def _run(cuda, oracle, prob, precision, steps):
    g = cuda.System(dict(prob["params"], precision=precision))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    g.run(steps)
    o.run(steps)
    return g, o


def _plate(num_cells, steps=30, v0=60.0):
    return P.plate_impact(num_cells=num_cells, steps=steps, v0=v0)


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_lone_particle(cuda, oracle, precision):
    """One particle, no neighbours: no force, and the damage of an empty
    row is 1 - 0/0 (NaN) on every path, as in the oracle."""
    prob = _plate((20, 10, 4))
    keep = np.array([0])
    prob.update(x=prob["x"][keep], vol=prob["vol"][keep], rho=prob["rho"][keep],
                nofail=prob["nofail"][keep], v0=prob["v0"][keep], bcs=[], notches=None)
    g, o = _run(cuda, oracle, prob, precision, 5)
    assert g.n == 1 and not np.any(g.get("f"))
    _check(g, o, precision)


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_isolated_particles_beside_a_body(cuda, oracle, precision):
    """Three particles far outside the plate (empty rows) appended to it:
    the plate's rows and the isolated ones follow the oracle."""
    prob = _plate((33, 17, 5))
    far = prob["x"][:3] + np.eye(3)  # a metre away from the plate and each other
    n = prob["x"].shape[0]
    prob.update(x=np.ascontiguousarray(np.vstack([prob["x"], far])),
                vol=np.concatenate([prob["vol"], prob["vol"][:3]]),
                rho=np.concatenate([prob["rho"], prob["rho"][:3]]),
                nofail=np.concatenate([prob["nofail"], np.zeros(3, np.int32)]),
                v0=np.ascontiguousarray(np.vstack([prob["v0"], np.zeros((3, 3))])))
    g, o = _run(cuda, oracle, prob, precision, 30)
    assert g.n == n + 3
    assert np.all(g.neighbors()[0][n:] == 0)
    _check(g, o, precision)


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_ragged_row_counts(cuda, oracle, precision):
    """Particle counts of 37 x 19 x 3 (not a multiple of a warp or block)."""
    g, o = _run(cuda, oracle, _plate((37, 19, 3)), precision, 40)
    _check(g, o, precision)


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_every_bond_cut(cuda, oracle, precision):
    """Pre-notches on the mid-planes between all neighbouring x, y and z
    layers: every bond crosses one, so every bond is cut, no force acts
    and every particle's damage is 1."""
    prob = _plate((12, 8, 3), v0=10.0)
    x = prob["x"]
    lo, hi = x.min(axis=0) - 1e-3, x.max(axis=0) + 1e-3
    p0, v1, v2 = [], [], []
    for d in range(3):
        a, b = (d + 1) % 3, (d + 2) % 3
        layers = np.unique(x[:, d])
        for g in 0.5 * (layers[1:] + layers[:-1]):
            corner = lo.copy()
            corner[d] = g
            e1, e2 = np.zeros(3), np.zeros(3)
            e1[a] = hi[a] - lo[a]
            e2[b] = hi[b] - lo[b]
            p0.append(corner)
            v1.append(e1)
            v2.append(e2)
    prob["notches"] = (np.array(v1), np.array(v2), np.array(p0))
    g, o = _run(cuda, oracle, prob, precision, 10)
    assert not np.any(g.neighbors()[2]) and not np.any(o.neighbors()[2])
    assert not np.any(g.get("f"))
    _check(g, o, precision)
    assert np.all(g.get("phi") == 1.0)


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_most_particles_frozen(cuda, oracle, precision):
    """All but the last 24 particles frozen: rows only for those, which
    still see the frozen particles as neighbours."""
    prob = _plate((16, 8, 3))
    prob["n_frozen"] = prob["x"].shape[0] - 8 * 3
    prob["bcs"] = [bc for bc in prob["bcs"]
                   if np.all(np.asarray(bc[2]) >= prob["n_frozen"])]
    g, o = _run(cuda, oracle, prob, precision, 20)
    _check(g, o, precision)


def test_zero_steps_change_nothing(cuda):
    prob = _plate((20, 10, 4))
    g = cuda.System(dict(prob["params"], precision=MIXED))
    P.setup(g, prob)
    before = [g.get(f) for f in ("u", "v", "f")]
    g.run(0)
    assert g.step_energy(0) == g.compute_energy()
    for a, f in zip(before, ("u", "v", "f")):
        assert np.array_equal(a, g.get(f))


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_five_spacing_horizon(cuda, oracle, precision):
    """delta = 5.01 dx: ~515 neighbours per row (17 bond words) and a stencil
    table of over 500 entries, past the shared memory of the lean forms, so
    the mixed path takes its general kernel."""
    from cabanapd_b200.inputs import critical_timestep
    prob = _plate((24, 14, 12), v0=40.0)
    h = prob["dx"][0]
    horizon = 5.01 * h
    dt = 0.5 * critical_timestep(h, h, h, 5, horizon, prob["params"]["K"], 8000.0)
    prob["params"] = dict(prob["params"], horizon=horizon, dt=dt)
    g, o = _run(cuda, oracle, prob, precision, 20)
    assert g.neighbor_stats()[0] > 500
    _check(g, o, precision)


@pytest.mark.parametrize("precision", [FAST, MIXED])
def test_thin_plate_with_stencil_entries_no_row_holds(cuda, oracle, precision):
    """Two cell layers: the stencil table (built from the horizon) has
    entries two and three layers apart that no row holds. The stencil
    kernels walk every entry; those read the row's own record and add
    nothing (they once carried an unset index delta)."""
    prob = _plate((40, 20, 2))
    g, o = _run(cuda, oracle, prob, precision, 30)
    _check(g, o, precision)


@pytest.mark.parametrize("precision", [FAST, MIXED])
def test_count_pass_spacing_equals_list_spacing(cuda, precision, monkeypatch):
    """The stencil set-up takes the lattice spacing from the neighbour
    build's count pass; with CPD_CHECK_SPACING=1 it also walks the list and
    fails the set-up if the two differ in any bit. A notched plate and an
    LPS box whose first layer (and a few more rows) is frozen."""
    monkeypatch.setenv("CPD_CHECK_SPACING", "1")
    plate = P.plate_impact(num_cells=(60, 30, 4), steps=4, v0=60.0)
    box = P.lps_random_notches(num_cells=(80, 32, 4), steps=4)
    nf = 80 * 32 + 7
    box = dict(box, n_frozen=nf)
    box["bcs"] = [(k, c, idx[idx >= nf], v) for k, c, idx, v in box["bcs"]]
    for prob in (plate, box):
        s = cuda.System(dict(prob["params"], precision=precision))
        P.setup(s, prob)
        s.run(prob["num_steps"])
        assert np.all(np.isfinite(s.get("u")))


@pytest.mark.parametrize("precision", [FAST, MIXED])
@pytest.mark.parametrize("model", ["lps", "pmb"])
def test_notched_two_layer_bodies(cuda, oracle, precision, model):
    """Two lattice layers (rows hold part of the stencil table and fewer
    bond-state words than the table has) with notches cutting bonds: the
    stencil kernels read only the list's words. LPS box 102 x 41 x 2 with
    20 random notches (a slightly non-cubic lattice), PMB plate 60 x 30 x 2
    on a cubic lattice (the plate 6.7 mm thick) with its two notches; 30
    steps against the oracle.

    The LPS forces of a two-layer body cancel far more than a bulk body's
    (every row is a surface row): the oracle itself, started from positions
    moved by one ulp, ends 30 steps later ~1e-11 away in f and ~2e-12 in v.
    FP64 is held to that spread (measured here, and at least 1e-12) in v
    and f, and to 1e-12 in u."""
    if model == "lps":
        prob = P.lps_random_notches(num_cells=(102, 41, 2), steps=30, seed=20261209)
    else:
        prob = P.plate_impact(num_cells=(60, 30, 2), steps=30, v0=60.0,
                              size=(0.2, 0.1, 0.2 * 2 / 60))
    g = cuda.System(dict(prob["params"], precision=precision))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    tu = TOL[precision][0]
    if model == "pmb":
        # A cubic lattice: the stencil kernels hold the rows.
        assert g.stencil_stats()[0] > 0
    if model == "lps":
        assert _nrel(g.get("m"), o.get("m")) <= (1e-13 if precision == FAST else 1e-6)
    g.run(prob["num_steps"])
    o.run(prob["num_steps"])
    tol_fields = None
    if model == "lps" and precision == FAST:
        moved = dict(prob)
        rng = np.random.default_rng(5)
        x = np.asarray(prob["x"], dtype=np.float64)
        moved["x"] = np.nextafter(x, np.where(rng.random(x.shape) < 0.5, -np.inf, np.inf))
        o2 = oracle.OracleSystem(prob["params"])
        P.setup(o2, moved)
        o2.run(prob["num_steps"])
        tol_fields = {fld: max(1e-12, _nrel(o2.get(fld), o.get(fld))) for fld in ("v", "f")}
    _check(g, o, precision, tol_fields)
    assert (o.neighbors()[2] == 0).sum() > 0
    assert _nrel(g.get("u"), o.get("u")) <= tu
