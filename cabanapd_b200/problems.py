"""Problem builders: particle lattices, initial conditions, pre-notches and
boundary conditions for the workloads this package runs.

Everything here is host-side numpy set-up that mirrors what the reference's
example programs do through ``Particles::domain/create/update``,
``Prenotch``, ``Region`` and ``createBoundaryCondition`` before the solver
starts. A problem is a plain dict consumed by :func:`setup`, which drives
any backend with the System call surface (the CUDA system, or the CPU
oracle in the tests).

Particle order: one particle per cell at the cell centre, x index fastest,
then y, then z (the order Cabana::Grid::createParticles assigns to owned
cells); volume = dx*dy*dz, rho = 1, nofail = 0 (CabanaPD_Particles.hpp:
242-307).
"""
import math

import numpy as np

from .inputs import PI, critical_timestep

# Model / BC numbering shared with the C ABI (include/cabanapd_b200.h).
PD_NONE, PD_PMB, PD_LPS, PD_LINEAR_PMB, PD_LINEAR_LPS = 0, 1, 2, 3, 4
CONTACT_NONE, CONTACT_HERTZ, CONTACT_NORMAL_REPULSION = 0, 1, 2
BC_FORCE_VALUE, BC_FORCE_UPDATE, BC_FORCE_ADD = 0, 1, 2


def lattice(low, high, num_cells):
    """Cell-centre particles of a uniform grid (x fastest).

    Returns (x [n,3], vol [n], dx [3]). Node coordinates are low + i*h and
    the particle sits half a cell above its low node, as Cabana's uniform
    particle initialisation computes them.
    """
    low = [float(v) for v in low]
    high = [float(v) for v in high]
    nc = [int(v) for v in num_cells]
    h = [(high[d] - low[d]) / nc[d] for d in range(3)]
    axes = []
    for d in range(3):
        i = np.arange(nc[d], dtype=np.float64)
        lo_node = low[d] + i * h[d]
        hi_node = low[d] + (i + 1.0) * h[d]
        axes.append(lo_node + 0.5 * (hi_node - lo_node))
    zz, yy, xx = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    x = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    vol = np.full(x.shape[0], h[0] * h[1] * h[2])
    return np.ascontiguousarray(x), vol, h


def in_prism(x, low, high):
    """Region<RectangularPrism>::inside (CabanaPD_Geometry.hpp:80-94):
    closed box test on each axis."""
    return ((x[:, 0] >= low[0]) & (x[:, 0] <= high[0]) & (x[:, 1] >= low[1]) &
            (x[:, 1] <= high[1]) & (x[:, 2] >= low[2]) & (x[:, 2] <= high[2]))


def pmb_s0(G0, K, horizon, influence_type=1):
    """CabanaPD_ForceModels.hpp:93-102."""
    if influence_type == 0:
        return math.sqrt(8.0 * G0 / 15.0 / K / horizon)
    return math.sqrt(5.0 * G0 / 9.0 / K / horizon)


def _problem(name, params, x, vol, **kw):
    n = x.shape[0]
    p = {
        "name": name,
        "params": params,
        "x": x,
        "vol": vol,
        "rho": kw.pop("rho", np.ones(n)),
        "nofail": kw.pop("nofail", np.zeros(n, dtype=np.int32)),
        "radius": kw.pop("radius", None),
        "u0": kw.pop("u0", None),
        "v0": kw.pop("v0", None),
        "notches": kw.pop("notches", None),
        "bcs": kw.pop("bcs", []),
        "num_steps": kw.pop("num_steps", 0),
        "n_frozen": kw.pop("n_frozen", 0),
    }
    p.update(kw)
    return p


def setup(system, problem, init=True):
    """Load a problem into a backend and run the Solver's init sequence."""
    system.set_particles(problem["x"], problem["vol"], problem["rho"],
                         problem["nofail"], problem["radius"],
                         n_frozen=problem["n_frozen"])
    if problem["u0"] is not None or problem["v0"] is not None:
        system.set_state(problem["u0"], problem["v0"])
    system.build_neighbors()
    if problem["notches"] is not None:
        system.prenotch(*problem["notches"])
    for kind, comp, idx, vals in problem["bcs"]:
        system.add_bc(kind, idx, vals, component=comp)
    if init:
        system.init()
    return system


# ---------------------------------------------------------------------------
# Workloads.

def elastic_wave_pmb(n=41, steps=100):
    """PMB elastic wave on [-0.5, 0.5]^3: n^3 particles, delta = 3.01 dx,
    K = 1, rho = 1, no fracture, u0 = 1e-4 exp(-(|x|/0.1)^2) x/|x|,
    dt = 0.5 * the PMB stable step."""
    x, vol, h = lattice([-0.5] * 3, [0.5] * 3, [n] * 3)
    m = 3
    horizon = float(m) * h[0] + 0.01 * h[0]
    K, rho0 = 1.0, 1.0
    dt = 0.5 * critical_timestep(h[0], h[1], h[2], m, horizon, K, rho0)
    r = np.sqrt(x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1] + x[:, 2] * x[:, 2])
    amp = 1e-4 * np.exp(-(r / 0.1) ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        comp = np.where(r[:, None] > 0.0, x / r[:, None], 0.0)
    u0 = amp[:, None] * comp
    params = dict(pd_model=PD_PMB, fracture=0, horizon=horizon, K=K, dt=dt)
    return _problem("elastic_wave_pmb", params, x, vol, u0=u0, num_steps=steps,
                    dx=h)


def elastic_wave_lps(deck):
    """The LinearLPS spherical-wave program of the reference's
    examples/mechanics/elastic_wave.cpp:57-100 for an input deck (dict in
    the JSON input format): cell-centre lattice from system_size and
    num_cells, horizon + 1e-10, u0 = 1e-3 exp(-((|x| - 0.25) / 0.07)^2) x/|x|
    (exp from the C library, through math.exp), v0 = 0, num_steps =
    int(final_time / timestep)."""
    n = deck["num_cells"]["value"]
    size = deck["system_size"]["value"]
    low = [-0.5 * s for s in size]
    high = [0.5 * s for s in size]
    x, vol, h = lattice(low, high, n)
    u0 = np.zeros_like(x)
    for p in range(x.shape[0]):
        r = math.sqrt(x[p, 0] * x[p, 0] + x[p, 1] * x[p, 1] + x[p, 2] * x[p, 2])
        d = r - 0.25
        arg = d * d / 0.07 / 0.07
        for c in range(3):
            direction = x[p, c] / r if r > 0.0 else 0.0
            u0[p, c] = 0.001 * math.exp(-arg) * direction
    dt = deck["timestep"]["value"]
    steps = int(deck["final_time"]["value"] / dt)
    params = dict(pd_model=PD_LINEAR_LPS, fracture=0,
                  horizon=deck["horizon"]["value"] + 1e-10,
                  K=deck["bulk_modulus"]["value"], G=deck["shear_modulus"]["value"], dt=dt)
    return _problem("elastic_wave_lps", params, x, vol,
                    rho=np.full(x.shape[0], float(deck["density"]["value"])), u0=u0,
                    num_steps=steps, dx=h,
                    output_frequency=int(deck["output_frequency"]["value"]))


def displacement_profile(prob, u, profile_dim=0, displacement_dim=None):
    """createDisplacementProfile (CabanaPD_OutputProfiles.hpp:27-84): the
    particles strictly within half a cell of the line through the origin
    along profile_dim, in index order, as (x[profile_dim], u[disp_dim])."""
    if displacement_dim is None:
        displacement_dim = profile_dim
    x, h = prob["x"], prob["dx"]
    d1, d2 = (profile_dim + 1) % 3, (profile_dim + 2) % 3
    on = np.nonzero((x[:, d1] < h[d1] / 2) & (x[:, d1] > -h[d1] / 2) &
                    (x[:, d2] < h[d2] / 2) & (x[:, d2] > -h[d2] / 2))[0]
    return x[on, profile_dim], u[on, displacement_dim]


def plate_impact(num_cells=(800, 400, 36), steps=2000, v0=16.5, size=(0.2, 0.1, 0.009),
                 horizon_factor=3.01):
    """PMB brittle fracture, double-notched plate impact (Kalthoff-Winkler
    layout of examples/mechanics/kalthoff_winkler.cpp): plate
    0.2 x 0.1 x 0.009 m, delta = 3.01 dx, E = 191 GPa, nu = 0.25,
    rho = 8000, G0 = 22170, two 0.05 m notches from the left edge at
    y = +-0.025, v_x = v0 on the strip between them held by a zero-force BC.
    `size` scales the plate (notches and strip in proportion), e.g. for a
    small plate at the full plate's spacing; `horizon_factor` is delta / dx
    (the reference's example decks use 4).
    """
    size = [float(s) for s in size]
    low = [-0.5 * s for s in size]
    high = [0.5 * s for s in size]
    x, vol, h = lattice(low, high, num_cells)
    horizon = horizon_factor * h[0]
    E, nu, rho0, G0 = 191e9, 0.25, 8000.0, 22170.0
    K = E / (3.0 * (1.0 - 2.0 * nu))
    dt = 0.5 * critical_timestep(h[0], h[1], h[2], int(math.floor(horizon / h[0])),
                                 horizon, K, rho0)
    length, width, thick = size
    y1, y2 = -width / 4.0, width / 4.0
    p0 = np.array([[low[0], y1, low[2]], [low[0], y2, low[2]]])
    v1 = np.array([[length / 4.0, 0.0, 0.0]] * 2)
    v2 = np.array([[0.0, 0.0, thick]] * 2)
    rho = np.full(x.shape[0], rho0)
    v = np.zeros_like(x)
    strip = (x[:, 1] > y1) & (x[:, 1] < y2) & (x[:, 0] < low[0] + h[0])
    v[strip, 0] = v0
    x_bc = low[0]
    bc_mask = in_prism(x, [x_bc - h[0], y1 - 0.25 * h[0], -thick],
                       [x_bc + h[0], y2 + 0.25 * h[0], thick])
    bcs = [(BC_FORCE_VALUE, 0, np.nonzero(bc_mask)[0], np.array([0.0]))]
    params = dict(pd_model=PD_PMB, fracture=1, horizon=horizon, K=K, G0=G0,
                  dt=dt)
    s0 = pmb_s0(G0, K, horizon, 1)
    return _problem("plate_impact", params, x, vol, rho=rho, v0=v,
                    notches=(v1, v2, p0), bcs=bcs, num_steps=steps, dx=h, s0=s0)


class _StdMt19937Uniform:
    """std::uniform_real_distribution<double>(0, 1) over std::mt19937(seed),
    as libstdc++ evaluates it (generate_canonical with two 32-bit draws)."""

    def __init__(self, seed):
        self._bg = np.random.MT19937()
        self._bg._legacy_seeding(int(seed))

    def __call__(self):
        lo, hi = (int(v) for v in self._bg.random_raw(2))
        r = (float(lo) + float(hi) * 4294967296.0) / 18446744073709551616.0
        if r >= 1.0:
            r = math.nextafter(1.0, 0.0)
        return r


def random_notches(seed, count, low, high, min_len, max_len):
    """Pre-notches drawn as examples/mechanics/random_cracks.cpp:66-114."""
    dis = _StdMt19937Uniform(seed)
    thick = high[2] - low[2]
    p0s, v1s, v2s = [], [], []
    for _ in range(count):
        rx, ry = dis(), dis()
        xc = (low[0] + max_len) + ((high[0] - max_len) - (low[0] + max_len)) * rx
        yc = (low[1] + max_len) + ((high[1] - max_len) - (low[1] + max_len)) * ry
        p0s.append([xc, yc, low[2]])
        rl = dis()
        length = min_len + (max_len - min_len) * rl
        th = PI * dis()
        v1s.append([length * math.cos(th), length * math.sin(th), 0.0])
        rv = dis()
        v2s.append([0.0, (-1.0 + 2.0 * rv) * thick, thick])
    return np.array(v1s), np.array(v2s), np.array(p0s)


def lps_random_notches(num_cells=(1000, 400, 20), steps=1000, seed=44758454,
                       count=20):
    """LPS fracture with random pre-notches (random_cracks.cpp layout):
    box 0.1 x 0.04 x 0.002 m, delta = 3.01 dx, K = 14.9 GPa, G = 8.9 GPa,
    rho = 2440, G0 = 3.8, influence type 0; traction 2 MPa on the y faces
    (f_y += +-sigma0/dy on slabs within +-dy of each face), no-fail zone
    within delta of the y faces; notch length U(0.002, 0.01)."""
    size = [0.1, 0.04, 0.002]
    low = [-0.5 * s for s in size]
    high = [0.5 * s for s in size]
    x, vol, h = lattice(low, high, num_cells)
    horizon = 3.01 * h[0]
    K, G, rho0, G0 = 14.9e9, 8.9e9, 2440.0, 3.8
    dt = 0.5 * critical_timestep(h[0], h[1], h[2], int(math.floor(horizon / h[0])),
                                 horizon, K, rho0)
    v1, v2, p0 = random_notches(seed, count, low, high, 0.002, 0.01)
    dy = h[1]
    plane1_lo = [low[0], low[1] - dy, low[2]]
    plane1_hi = [high[0], low[1] + dy, high[2]]
    plane2_lo = [low[0], high[1] - dy, low[2]]
    plane2_hi = [high[0], high[1] + dy, high[2]]
    nofail = ((x[:, 1] <= plane1_lo[1] + horizon + 1e-10) |
              (x[:, 1] >= plane2_hi[1] - horizon - 1e-10)).astype(np.int32)
    sigma0 = 2e6
    b0 = sigma0 / dy
    idx = np.concatenate([np.nonzero(in_prism(x, plane1_lo, plane1_hi))[0],
                          np.nonzero(in_prism(x, plane2_lo, plane2_hi))[0]])
    ypos = x[idx, 1]
    vals = b0 * (np.abs(ypos) / ypos)
    bcs = [(BC_FORCE_ADD, 1, idx, vals)]
    params = dict(pd_model=PD_LPS, fracture=1, influence_type=0,
                  horizon=horizon, K=K, G=G, G0=G0, dt=dt)
    rho = np.full(x.shape[0], rho0)
    return _problem("lps_random_notches", params, x, vol, rho=rho,
                    nofail=nofail, notches=(v1, v2, p0), bcs=bcs,
                    num_steps=steps, dx=h, s0=pmb_s0(G0, K, horizon, 0))


def dem_packing(lattice_dims=(200, 200, 100), spacing=2.5e-3, steps=5000,
                seed=20241203, dt=1e-7, rebuild_every=10):
    """Hertzian DEM packing: spheres on a jittered lattice (jitter
    U(+-1.4e-4) per axis, strictly non-overlapping for R <= 1.1e-3), radii
    U(0.9, 1.1) mm, velocities N(0, 0.1) m/s per component, E = 70 GPa,
    nu = 0.3, rho = 2500, e = 0.8, contact list rebuilt every
    ``rebuild_every`` steps with skin 0.2 R_max."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nx_, ny_, nz_ = lattice_dims
    size = [nx_ * spacing, ny_ * spacing, nz_ * spacing]
    low = [-0.5 * s for s in size]
    high = [0.5 * s for s in size]
    x, _, _ = lattice(low, high, lattice_dims)
    n = x.shape[0]
    x = x + rng.uniform(-1.4e-4, 1.4e-4, size=(n, 3))
    radius = rng.uniform(0.9e-3, 1.1e-3, size=n)
    v = rng.normal(0.0, 0.1, size=(n, 3))
    vol = 4.0 / 3.0 * PI * radius ** 3
    r_max = 1.1e-3
    params = dict(pd_model=PD_NONE, contact_model=CONTACT_HERTZ,
                  contact_radius=r_max, radius_extend=0.2 * r_max, nu=0.3,
                  E=70e9, restitution=0.8, dt=dt, rebuild_every=rebuild_every,
                  per_particle_radius=1)
    rho = np.full(n, 2500.0)
    return _problem("dem_packing", params, np.ascontiguousarray(x), vol, rho=rho,
                    radius=radius, v0=v, num_steps=steps)


def hertz_two_spheres():
    """regression_test/tstHertz.hpp:40-136 with inputs/hertzian_contact.json:
    two spheres at x = +-5.1e-5 approaching at 1 m/s each."""
    x = np.array([[5.1e-5, 0.0, 0.0], [-5.1e-5, 0.0, 0.0]])
    vol = np.full(2, 5.236e-13)
    rho = np.full(2, 7.95e3)
    v = np.array([[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]])
    dt = 0.8e-8
    steps = int(1e-5 / dt)
    params = dict(pd_model=PD_NONE, contact_model=CONTACT_HERTZ,
                  contact_radius=5e-5, radius_extend=1e-8, nu=0.25,
                  E=195.6e9, restitution=0.5, dt=dt, rebuild_every=0)
    return _problem("hertz_two_spheres", params, x, vol, rho=rho, v0=v,
                    num_steps=steps)


def kalthoff_winkler_regression():
    """regression_test/tstKalthoffWinkler.hpp with
    regression_test/inputs/kalthoff_winkler.json driven the way
    examples/mechanics/kalthoff_winkler.cpp does: 75 x 151 x 7 cells,
    nu = 1/3, horizon = 0.002 + 1e-10, G0 = 42408, v0 = 16 m/s,
    output every 50 steps."""
    num_cells = [75, 151, 7]
    size = [0.1, 0.2, 0.009]
    low = [-0.5 * s for s in size]
    high = [0.5 * s for s in size]
    x, vol, h = lattice(low, high, num_cells)
    rho0, E, G0 = 8000.0, 191e9, 42408.0
    nu = 1.0 / 3.0
    K = E / (3.0 * (1.0 - 2.0 * nu))
    horizon = 0.002 + 1e-10
    height, width, thick = size
    y1, y2 = -width / 8.0, width / 8.0
    p0 = np.array([[low[0], y1, low[2]], [low[0], y2, low[2]]])
    v1 = np.array([[height / 2.0, 0.0, 0.0]] * 2)
    v2 = np.array([[0.0, 0.0, thick]] * 2)
    dx = h[0]
    v = np.zeros_like(x)
    strip = (x[:, 1] > y1) & (x[:, 1] < y2) & (x[:, 0] < -0.5 * height + dx)
    v[strip, 0] = 16.0
    x_bc = -0.5 * height
    bc_mask = in_prism(x, [x_bc - dx, y1 - 0.25 * dx, -thick],
                       [x_bc + dx, y2 + 0.25 * dx, thick])
    bcs = [(BC_FORCE_VALUE, 0, np.nonzero(bc_mask)[0], np.array([0.0]))]
    dt = 1e-7
    steps = int(70e-6 / dt)
    params = dict(pd_model=PD_PMB, fracture=1, horizon=horizon, K=K, G0=G0, dt=dt)
    return _problem("kalthoff_winkler", params, x, vol,
                    rho=np.full(x.shape[0], rho0), v0=v, notches=(v1, v2, p0),
                    bcs=bcs, num_steps=steps, output_frequency=50, dx=h)


def random_in_cells(low, high, num_cells, rng):
    """One particle per cell at a uniform random point of the cell (x index
    fastest), the placement Cabana::InitRandom makes; the reference's own
    random stream is not reproduced. Returns (x [n,3], vol [n], dx [3])."""
    low = [float(v) for v in low]
    high = [float(v) for v in high]
    nc = [int(v) for v in num_cells]
    h = [(high[d] - low[d]) / nc[d] for d in range(3)]
    lo_nodes = [low[d] + np.arange(nc[d], dtype=np.float64) * h[d] for d in range(3)]
    hi_nodes = [low[d] + (np.arange(nc[d], dtype=np.float64) + 1.0) * h[d] for d in range(3)]
    zz, yy, xx = np.meshgrid(lo_nodes[2], lo_nodes[1], lo_nodes[0], indexing="ij")
    lo = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    zz, yy, xx = np.meshgrid(hi_nodes[2], hi_nodes[1], hi_nodes[0], indexing="ij")
    hi = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1)
    t = rng.random(lo.shape)
    x = lo + t * (hi - lo)
    return np.ascontiguousarray(x), np.full(x.shape[0], h[0] * h[1] * h[2]), h


def fragmenting_cylinder(num_cells=(200, 200, 300), size=(0.2, 0.2, 0.3), height=0.1,
                         outer=0.025, inner=0.02, steps=None, seed=20261204, contact=True,
                         x=None):
    """examples/mechanics/fragmenting_cylinder.cpp with its input deck
    (examples/mechanics/inputs/fragmenting_cylinder.json): a hollow steel
    cylinder, PMB with fracture (K = 130 GPa, rho = 7800, critical stretch
    0.02, horizon 0.00417462 + 1e-10 m, G0 = 9 K delta sc^2 / 5), thrown
    outward by v_r = 200 - 50 z'^2 and v_z = 100 z' m/s, z' = (z - z_min) /
    (H / 2) - 1. With ``contact`` the fragments repel through normal
    repulsion (the PD delta and K, radius 0.9 dx / 2, search extension
    0.01 dx). Particles sit at a seeded random point of their cell and are
    kept inside the shell (``x`` overrides the placement with given
    positions, before the shell filter). dt = 1.7e-7 s; the deck's final
    time 2.4e-4 s gives 1411 steps."""
    low = [-0.5 * s for s in size]
    high = [0.5 * s for s in size]
    if x is None:
        rng = np.random.Generator(np.random.PCG64(seed))
        x, vol, h = random_in_cells(low, high, num_cells, rng)
    else:
        h = [(high[d] - low[d]) / num_cells[d] for d in range(3)]
        x = np.ascontiguousarray(x, dtype=np.float64)
        vol = np.full(x.shape[0], h[0] * h[1] * h[2])
    center = [0.5 * (low[d] + high[d]) for d in range(3)]
    rsq = (x[:, 0] - center[0]) ** 2 + (x[:, 1] - center[1]) ** 2
    keep = ~((rsq < inner * inner) | (rsq > outer * outer) |
             (x[:, 2] > center[2] + 0.5 * height) | (x[:, 2] < center[2] - 0.5 * height))
    x = np.ascontiguousarray(x[keep])
    vol = vol[keep]
    rho0, K, sc = 7800.0, 130e9, 0.02
    horizon = 0.00417462 + 1e-10
    G0 = 9 * K * horizon * (sc * sc) / 5
    z_min = center[2] - 0.5 * height
    zf = ((x[:, 2] - z_min) / (0.5 * height)) - 1
    vr = 200.0 - 50.0 * zf * zf
    ang = np.arctan2(x[:, 1], x[:, 0])
    v = np.stack([vr * np.cos(ang), vr * np.sin(ang), 100.0 * zf], axis=1)
    dt = 1.7e-7
    if steps is None:
        steps = int(2.4e-4 / dt)
    params = dict(pd_model=PD_PMB, fracture=1, horizon=horizon, K=K, G0=G0, dt=dt)
    if contact:
        params.update(contact_model=CONTACT_NORMAL_REPULSION, contact_horizon=horizon,
                      contact_K=K, contact_radius=0.9 * h[0] / 2.0,
                      radius_extend=0.01 * h[0], rebuild_every=0)
    return _problem("fragmenting_cylinder", params, x, vol, rho=np.full(x.shape[0], rho0),
                    v0=np.ascontiguousarray(v), num_steps=steps, output_frequency=50, dx=h)


def unit_cube(model, dx, s0, kind, K=1.0, G=0.5, G0=None, influence_type=None):
    """unit_test/tstForce.hpp:593-661 createParticles: [-1, 1]^3 lattice,
    m = 3, horizon = 3 dx; ``kind`` 'linear' sets u = s0 x (all
    components), 'quadratic' sets u_x = s0 x^2."""
    nc = int(2.0 / dx)
    x, vol, h = lattice([-1.0] * 3, [1.0] * 3, [nc] * 3)
    if kind == "linear":
        u0 = s0 * x
    else:
        u0 = np.zeros_like(x)
        u0[:, 0] = s0 * x[:, 0] * x[:, 0]
    horizon = dx * 3
    params = dict(pd_model=model, fracture=0 if G0 is None else 1,
                  horizon=horizon, K=K, G=G, G0=G0 or 0.0, dt=1.0)
    if influence_type is not None:
        params["influence_type"] = influence_type
    return _problem("unit_cube", params, x, vol, u0=u0, dx=h)


# ---------------------------------------------------------------------------
# Served stream of independent jobs.

def served_jobs(count=512, n_range=(1e3, 2e6), steps_range=(200, 2000), seed=20261203):
    """Independent jobs for the job server: half PMB (alternately the
    elastic-wave cube and the double-notched plate), half LPS (random-notch
    box), particle counts log-uniform in n_range (grids keep each geometry's
    aspect ratio), step counts uniform in steps_range, all seeded.
    Returns a list of problem dicts (see setup())."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi = math.log(n_range[0]), math.log(n_range[1])
    jobs = []
    for k in range(count):
        target = math.exp(rng.uniform(lo, hi))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        kind = ("wave", "plate", "lps", "lps")[k % 4]
        if kind == "wave":
            side = max(8, int(round(target ** (1.0 / 3.0))))
            prob = elastic_wave_pmb(n=side, steps=steps)
        elif kind == "plate":
            a = max(16, int(round((target / (0.5 * 0.045)) ** (1.0 / 3.0))))
            cells = (a, max(8, a // 2), max(1, int(round(0.045 * a))))
            prob = plate_impact(num_cells=cells, steps=steps)
        else:
            a = max(30, int(round((target / (0.4 * 0.02)) ** (1.0 / 3.0))))
            cells = (a, max(12, int(round(0.4 * a))), max(1, int(round(0.02 * a))))
            prob = lps_random_notches(num_cells=cells, steps=steps, seed=seed + k)
        prob["kind"] = kind
        jobs.append(prob)
    return jobs
