"""The CabanaPD-API front end (include/CabanaPD.hpp): programs written
against the reference's Inputs / ForceModel / Particles / Solver /
Prenotch / createBoundaryCondition / OutputTimeSeries API (examples/*.cpp,
built by examples/Makefile) run on the GPU library.

CPU tests: the front end compiles as plain C++, and its Inputs derive the
same keys and critical time step as the Python Inputs.
GPU tests: each example reproduces the reference's regression check for its
program, and, in EXACT precision, gives bit-identical results to the same
problem driven through the Python binding of the C ABI (same kernels, same
order), which the parity tests tie to the oracle.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from cabanapd_b200 import problems as P
from cabanapd_b200.inputs import Inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXAMPLES = os.path.join(ROOT, "examples")
BUILD = os.path.join(EXAMPLES, "_build")
INCLUDE = os.path.join(ROOT, "include")


def _gxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    pytest.skip("no host C++ compiler")


# ---------------------------------------------------------------------------
# CPU


@pytest.mark.parametrize("name", ["kalthoff_winkler", "elastic_wave", "random_cracks",
                                  "hertz_spheres", "stress_cube", "fragmenting_cylinder"])
def test_examples_compile_as_host_cpp(name):
    """The front end is plain C++17 outside nvcc (KOKKOS_LAMBDA = [=])."""
    r = subprocess.run([_gxx(), "-std=c++17", "-fsyntax-only", "-Wall", "-I", INCLUDE,
                        os.path.join(EXAMPLES, name + ".cpp")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr


DECKS = {
    "kw": {"num_cells": {"value": [75, 151, 7]},
           "system_size": {"value": [0.1, 0.2, 0.009]},
           "density": {"value": 8000}, "elastic_modulus": {"value": 191e9},
           "horizon": {"value": 0.002}, "final_time": {"value": 70e-6},
           "timestep": {"value": 1e-7}, "output_frequency": {"value": 50}},
    "m_and_corners": {"low_corner": {"value": [-1.0, -0.5, 0.0]},
                      "high_corner": {"value": [1.0, 0.5, 0.25]},
                      "dx": {"value": [0.05, 0.05, 0.05]}, "m": {"value": 3},
                      "density": {"value": [2.0, 3.0]},
                      "bulk_modulus": {"value": [1.0, 2.0]},
                      "final_time": {"value": 1.0}, "timestep": {"value": 0.0125},
                      "timestep_safety_factor": {"value": 0.5}},
    "mass_scaling": {"num_cells": {"value": [20, 10, 4]},
                     "system_size": {"value": [2.0, 1.0, 0.4]},
                     "density": {"value": 100.0}, "elastic_modulus": {"value": 3.0},
                     "horizon": {"value": 0.31}, "final_time": {"value": 2.0},
                     "timestep": {"value": 0.01}, "mass_scaling_factor": {"value": 4.0}},
}

_PROBE = r"""
#include <cstdio>
#include "cabanapd_shim/inputs.hpp"
int main(int, char** argv)
{
    CabanaPD::Inputs in(argv[1]);
    const double dt_crit = in.computeCriticalTimeStep();
    std::array<double, 3> lo = in["low_corner"], hi = in["high_corner"], dx = in["dx"];
    std::array<int, 3> nc = in["num_cells"];
    std::printf("%.17g %.17g %.17g %.17g %.17g %.17g\n", lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
    std::printf("%.17g %.17g %.17g %d %d %d\n", dx[0], dx[1], dx[2], nc[0], nc[1], nc[2]);
    std::printf("%d %.17g %d %.17g %.17g\n", (int)in["m"], (double)in["horizon"],
                (int)in["num_steps"], (double)in["timestep"], in.getVector("density")[0]);
    std::printf("%.17g %.17g\n", dt_crit, (double)in["critical_timestep_mechanics"]);
    return 0;
}
"""


@pytest.fixture(scope="module")
def inputs_probe(tmp_path_factory):
    d = tmp_path_factory.mktemp("probe")
    src = d / "probe.cpp"
    src.write_text(_PROBE)
    exe = d / "probe"
    r = subprocess.run([_gxx(), "-std=c++17", "-O1", "-ffp-contract=off", "-I", INCLUDE,
                        str(src), "-o", str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return str(exe)


@pytest.mark.parametrize("deck", sorted(DECKS))
def test_cpp_inputs_match_python_inputs(inputs_probe, tmp_path, deck):
    """CabanaPD_Input.hpp:30-301 derived keys and dt_crit, C++ front end vs
    the Python Inputs, bit for bit."""
    path = tmp_path / "deck.json"
    path.write_text(json.dumps(DECKS[deck]))
    r = subprocess.run([inputs_probe, str(path)], cwd=tmp_path, capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    got = [float(t) for t in r.stdout.split()]
    py = Inputs(str(path))
    dt_crit = py.compute_critical_timestep()
    want = (list(py["low_corner"]) + list(py["high_corner"]) + list(py["dx"]) +
            list(py["num_cells"]) +
            [py["m"], py["horizon"], py["num_steps"], py["timestep"],
             (py["density"] if not isinstance(py["density"], list) else py["density"][0])] +
            [dt_crit, py["critical_timestep_mechanics"]])
    assert len(got) == len(want)
    for a, b in zip(got, want):
        assert a == float(b), (got, want)


_XDMF_PROBE = r"""
#include <CabanaPD.hpp>
int main()
{
    using CabanaPD::detail::OutputField;
    const int64_t n = 5;
    OutputField pos{"reference_positions", 3, {}, {}};
    OutputField f{"forces", 3, {}, {}}, w{"damage", 1, {}, {}}, s{"stress", 9, {}, {}};
    OutputField t{"type", 1, {}, std::vector<int32_t>(n, 0)};
    for (int64_t i = 0; i < n; i++) {
        for (int c = 0; c < 3; c++) {
            pos.values.push_back(i + 0.25 * c);
            f.values.push_back(-1.5 * i + c);
        }
        w.values.push_back(0.125 * i);
        t.ints[i] = static_cast<int32_t>(i % 2);
        for (int c = 0; c < 9; c++) s.values.push_back(10.0 * i + c);
    }
    CabanaPD::detail::write_xdmf_particles("particles", 3, 2.5e-6, n, pos, {f, t, w, s});
    return 0;
}
"""


def read_xdmf_particles(path):
    """Parse a particle XDMF file: (time, {name: array}) with the geometry
    under the name of the first DataItem's role, "positions"."""
    import xml.etree.ElementTree as ET
    root = ET.parse(path).getroot()
    grid = root.find("Domain/Grid")
    time = float(grid.find("Time").get("Value"))

    def load(item):
        dims = [int(v) for v in item.get("Dimensions").split()]
        dtype = {("Float", "8"): "<f8", ("Int", "4"): "<i4"}[(item.get("NumberType"),
                                                               item.get("Precision"))]
        assert item.get("Endian") == "Little" and item.get("Format") == "Binary"
        data = np.fromfile(os.path.join(os.path.dirname(path), item.text.strip()), dtype=dtype,
                           count=int(np.prod(dims)), offset=int(item.get("Seek")))
        return data.reshape(dims)

    out = {"positions": load(grid.find("Geometry/DataItem"))}
    for att in grid.findall("Attribute"):
        out[att.get("Name")] = load(att.find("DataItem"))
    return time, out


def test_xdmf_particle_writer(tmp_path):
    """The particle output format of the front end: an XDMF polyvertex grid
    whose heavy data (doubles and int32, [n][components]) sit back to back
    in one binary file, read back exactly."""
    src = tmp_path / "probe.cpp"
    src.write_text(_XDMF_PROBE)
    exe = tmp_path / "probe"
    r = subprocess.run([_gxx(), "-std=c++17", "-O1", "-I", INCLUDE, str(src), "-o", str(exe)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    time, fields = read_xdmf_particles(str(tmp_path / "particles_3.xmf"))
    assert time == 2.5e-6
    i = np.arange(5.0)
    assert np.array_equal(fields["positions"], i[:, None] + 0.25 * np.arange(3.0)[None, :])
    assert np.array_equal(fields["forces"], -1.5 * i[:, None] + np.arange(3.0)[None, :])
    assert np.array_equal(fields["type"], (np.arange(5) % 2).astype(np.int32))
    assert np.array_equal(fields["damage"], 0.125 * i)
    assert np.array_equal(fields["stress"], 10.0 * i[:, None] + np.arange(9.0)[None, :])


# ---------------------------------------------------------------------------
# GPU


def _run_example(name, deck, workdir, precision="exact", args=(), env_extra=None):
    exe = os.path.join(BUILD, name)
    if not os.path.exists(exe):
        raise RuntimeError(f"{exe} is missing: build the examples (make -C examples)")
    path = os.path.join(workdir, name + ".json")
    with open(path, "w") as fh:
        json.dump(deck, fh)
    env = dict(os.environ, CABANAPD_B200_PRECISION=precision, **(env_extra or {}))
    r = subprocess.run([exe, path, *args], cwd=workdir, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def _printed(stdout, key):
    for line in stdout.splitlines():
        if line.startswith(key + ":"):
            return [float(t) for t in line.split(":", 1)[1].replace("damage:", "").split()]
    raise AssertionError(f"{key} not printed: {stdout}")


@pytest.fixture(scope="module")
def lib():
    import cabanapd_b200
    return cabanapd_b200


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["exact", "fp64"])
def test_kalthoff_winkler_program(lib, golden, tmp_path, precision):
    """regression_test/tstKalthoffWinkler.hpp:53 on the example program; in
    EXACT precision the crack extent equals the Python-driven GPU run's."""
    from test_oracle_regression import kw_max_crack_y
    g = golden["kalthoff_winkler"]
    out = _run_example("kalthoff_winkler", g["input"], str(tmp_path), precision)
    y = _printed(out, "max crack y")[0]
    assert abs(y - g["max_crack_y"]) <= g["tolerance"], y
    series = np.loadtxt(tmp_path / "output_kw_crack_y.txt")
    assert series.shape[0] == 14 and series[-1, 0] == pytest.approx(y, abs=1e-15)
    if precision == "exact":
        prob = P.kalthoff_winkler_regression()
        s = lib.System(dict(prob["params"], precision=lib.system.FP64_EXACT))
        P.setup(s, prob)
        assert kw_max_crack_y(s, prob) == y


@pytest.mark.gpu
def test_elastic_wave_program(lib, golden, tmp_path):
    """regression_test/tstElasticWave.hpp:54-96 on the example program's
    displacement profile (LinearLPS, 41^3), and bit-identity of that profile
    with the Python-driven GPU run."""
    from test_oracle_regression import elastic_wave_profile_errors
    g = golden["elastic_wave"]
    _run_example("elastic_wave", g["input"], str(tmp_path), "exact")
    prof = np.loadtxt(tmp_path / "displacement_profile.txt", ndmin=2)
    assert prof.shape[0] == 41
    rel, l2 = elastic_wave_profile_errors(golden, prof[:, 1], prof[:, 2])
    assert rel < g["rel_tol"] and l2 < g["l2_tol"], (rel, l2)

    prob = P.elastic_wave_lps(g["input"])
    s = lib.System(prob["params"])
    P.setup(s, prob)
    s.run(prob["num_steps"])
    xs, us = P.displacement_profile(prob, s.get("u"))
    assert np.array_equal(prof[:, 1], xs)
    assert np.array_equal(prof[:, 2], us)


def _random_cracks_deck(num_cells, steps):
    prob = P.lps_random_notches(num_cells=num_cells, steps=steps)
    dt = prob["params"]["dt"]
    deck = {
        "num_cells": {"value": list(num_cells)},
        "system_size": {"value": [0.1, 0.04, 0.002]},
        "density": {"value": 2440.0}, "bulk_modulus": {"value": 14.9e9},
        "shear_modulus": {"value": 8.9e9}, "fracture_energy": {"value": 3.8},
        "horizon": {"value": prob["params"]["horizon"]}, "traction": {"value": 2e6},
        "minimum_prenotch_length": {"value": 0.002},
        "maximum_prenotch_length": {"value": 0.01},
        "final_time": {"value": (steps + 0.5) * dt}, "timestep": {"value": dt},
        "output_frequency": {"value": steps},
    }
    return prob, deck


@pytest.mark.gpu
def test_random_cracks_program_custom_traction(lib, tmp_path):
    """LPS fracture with 20 seeded notches and the traction as a device
    functor f(p, 1) += b0 * sign(y): totals at the last step equal the
    Python-driven run that applies the same traction as a per-particle
    force boundary condition."""
    prob, deck = _random_cracks_deck((200, 80, 4), 60)
    out = _run_example("random_cracks", deck, str(tmp_path), "exact")
    W, D = _printed(out, "strain energy")
    s = lib.System(dict(prob["params"], precision=lib.system.FP64_EXACT))
    P.setup(s, prob)
    s.run(prob["num_steps"])
    Wp, Dp = s.compute_energy()
    assert Dp > 0.0
    assert (W, D) == (Wp, Dp)


def _hertz_deck(golden):
    g = dict(golden["hertz"]["input"])
    g.pop("system_size", None)
    g.pop("num_cells", None)
    r = 5.1e-5
    g["low_corner"] = {"value": [-2 * r, -r, -r]}
    g["high_corner"] = {"value": [2 * r, r, r]}
    g["num_cells"] = {"value": [2, 1, 1]}
    g["impact_speed"] = {"value": 1.0}
    steps = int(g["final_time"]["value"] / g["timestep"]["value"])
    g["output_frequency"] = {"value": steps}
    return g, steps


@pytest.mark.gpu
def test_hertz_program_restitution(lib, golden, tmp_path):
    """regression_test/tstHertz.hpp:135 (restitution within 1e-3 of the
    input) on the HertzianModel program, equal to the Python-driven run."""
    from test_oracle_regression import hertz_restitution
    deck, steps = _hertz_deck(golden)
    out = _run_example("hertz_spheres", deck, str(tmp_path), "exact")
    e = _printed(out, "restitution")[0]
    want = deck["restitution"]["value"]
    assert abs(e - want) <= golden["hertz"]["tolerance"], e

    lo, hi = deck["low_corner"]["value"], deck["high_corner"]["value"]
    x, _, _ = P.lattice(lo, hi, [2, 1, 1])
    v = np.zeros_like(x)
    v[:, 0] = np.where(x[:, 0] > 0.0, -1.0, 1.0)
    prob = P.hertz_two_spheres()
    prob.update(x=x, v0=v, vol=np.full(2, deck["volume"]["value"]), num_steps=steps)
    s = lib.System(prob["params"])
    P.setup(s, prob)
    assert hertz_restitution(s, prob) == pytest.approx(e, rel=1e-14, abs=0)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["pmb", "lps"])
def test_stress_cube_program(lib, tmp_path, case):
    """EnergyStressOutput particles through the CabanaPD API (stress_cube.cpp):
    the stress the solver computes at init meets the reference's stress
    checks (unit_test/tstForce.hpp:744-750: diagonal FLOAT_EQ the single-point
    sum, other components <= 1e-13) at interior particles, and equals bit for
    bit the stress of the same problem driven through the Python binding."""
    import force_checks
    import reference_sums as R
    model_id, dx, bw, _, infl, _ = force_checks.CASES[case]
    nc = int(2.0 / dx)
    s0 = 0.1
    deck = {"low_corner": {"value": [-1.0, -1.0, -1.0]},
            "high_corner": {"value": [1.0, 1.0, 1.0]},
            "num_cells": {"value": [nc, nc, nc]}, "horizon": {"value": dx * 3},
            "density": {"value": 1.0}, "bulk_modulus": {"value": 1.0},
            "shear_modulus": {"value": 0.5}, "stretch": {"value": s0},
            "timestep": {"value": 1e-3}, "final_time": {"value": 4.5e-3},
            "output_frequency": {"value": 2}}
    _run_example("stress_cube", deck, str(tmp_path), "exact", args=(case,))
    init = np.loadtxt(tmp_path / "stress_init.txt")
    final = np.loadtxt(tmp_path / "stress_final.txt")
    assert np.all(np.isfinite(final)) and final.shape == init.shape
    x, sigma = init[:, :3], init[:, 3:].reshape(-1, 3, 3)

    prob = P.unit_cube(model_id, dx, s0, "linear", K=1.0, G=0.5, influence_type=infl)
    s = lib.System(dict(prob["params"], precision=0))
    P.setup(s, prob)
    s.compute_stress()
    assert np.array_equal(x, s.get("x"))
    assert np.array_equal(sigma, s.get("stress"))

    c = s.model_constants()
    ref = R.PMBRef(c["c"]) if case == "pmb" else R.LPSRef(c["theta_coeff"], c["s_coeff"], infl)
    horizon = dx * 3
    ref_sigma = R.ref_stress(ref, "linear", horizon, 3, s0)
    lo, hi = -1.0 + horizon * bw, 1.0 - horizon * bw
    interior = np.nonzero(np.all((x > lo) & (x < hi), axis=1))[0]
    assert interior.size > 0
    for p in interior:
        for d in range(3):
            assert R.float_eq(sigma[p, d, d], ref_sigma[d]), (p, d, sigma[p, d, d], ref_sigma[d])
        off = sigma[p][~np.eye(3, dtype=bool)]
        assert np.all(off <= 1e-13), (p, off)


def _cylinder_deck(steps, use_contact=True):
    """The fragmenting-cylinder deck (examples/mechanics/inputs/
    fragmenting_cylinder.json) on a shorter cylinder in a smaller box."""
    dt = 1.7e-7
    return {
        "dx": {"value": [0.001, 0.001, 0.001]},
        "system_size": {"value": [0.06, 0.06, 0.04]},
        "density": {"value": 7800}, "bulk_modulus": {"value": 130e9},
        "shear_modulus": {"value": 78e9}, "critical_stretch": {"value": 0.02},
        "horizon": {"value": 0.00417462}, "use_contact": {"value": use_contact},
        "contact_horizon_factor": {"value": 0.9},
        "contact_horizon_extend_factor": {"value": 0.01},
        "cylinder_outer_radius": {"value": 0.025}, "cylinder_inner_radius": {"value": 0.02},
        "cylinder_height": {"value": 0.03}, "max_radial_velocity": {"value": 200},
        "min_radial_velocity": {"value": 50}, "max_vertical_velocity": {"value": 100},
        "final_time": {"value": (steps + 0.5) * dt}, "timestep": {"value": dt},
        "timestep_safety_factor": {"value": 0.70}, "output_frequency": {"value": steps},
        "output_reference": {"value": False},
    }


@pytest.mark.gpu
@pytest.mark.parametrize("use_contact", [True, False])
def test_fragmenting_cylinder_program(lib, tmp_path, use_contact):
    """PMB fracture with normal-repulsion contact through the CabanaPD API
    (Solver(inputs, particles, model, contact)): final totals equal the
    Python-driven run of the same particles bit for bit and fragmentation
    has started; with contact the list is rebuilt every step (200 m/s)."""
    steps = 40
    deck = _cylinder_deck(steps, use_contact)
    out = _run_example("fragmenting_cylinder", deck, str(tmp_path), "exact")
    W, D = _printed(out, "strain energy")
    n = int(_printed(out, "particles")[0])
    init = np.loadtxt(tmp_path / "cylinder_initial.txt", ndmin=2)
    assert init.shape == (n, 6)
    nc = Inputs(str(tmp_path / "fragmenting_cylinder.json"))["num_cells"]
    prob = P.fragmenting_cylinder(num_cells=nc, size=(0.06, 0.06, 0.04), height=0.03,
                                  steps=steps, contact=use_contact, x=init[:, :3])
    assert prob["x"].shape[0] == n
    prob["v0"] = np.ascontiguousarray(init[:, 3:])
    s = lib.System(dict(prob["params"], precision=lib.system.FP64_EXACT))
    P.setup(s, prob)
    s.run(steps)
    assert s.compute_energy() == (W, D)
    assert D > 0.0
    if use_contact:
        assert s.contact_rebuilds() == steps


@pytest.mark.gpu
def test_particle_output_files(lib, tmp_path):
    """Particles::output through the Solver (initial output and each output
    step) with CABANAPD_B200_PARTICLE_OUTPUT set: the LPS program's last
    output holds the displacements, velocities, forces, damage, weighted
    volume and dilatation of the Python-driven run bit for bit, at the
    reference positions (output_reference defaults to true)."""
    prob, deck = _random_cracks_deck((200, 80, 4), 60)
    deck["output_frequency"] = {"value": 30}
    _run_example("random_cracks", deck, str(tmp_path), "exact",
                 env_extra={"CABANAPD_B200_PARTICLE_OUTPUT": "1"})
    names = sorted(p.name for p in tmp_path.glob("particles_*.xmf"))
    assert names == ["particles_0.xmf", "particles_1.xmf", "particles_2.xmf"]
    t0, first = read_xdmf_particles(str(tmp_path / "particles_0.xmf"))
    t2, last = read_xdmf_particles(str(tmp_path / "particles_2.xmf"))
    dt = prob["params"]["dt"]
    assert t0 == 0.0 and t2 == 60 * dt
    s = lib.System(dict(prob["params"], precision=lib.system.FP64_EXACT))
    P.setup(s, prob)
    assert np.array_equal(first["positions"], s.get("x"))
    assert not np.any(first["displacements"])
    s.run(prob["num_steps"])
    s.compute_energy()
    assert np.array_equal(last["positions"], s.get("x"))
    for name, field in (("displacements", "u"), ("velocities", "v"), ("damage", "phi"),
                        ("weighted_volume", "m"), ("dilatation", "theta"),
                        ("strain_energy", "W")):
        assert np.array_equal(last[name], s.get(field)), name
    assert np.any(last["damage"] > 0)
    # The program's traction is a device functor added after the library's
    # force; the Python run applies it as a force BC, so forces agree to
    # rounding of that sum only.
    f = s.get("f")
    assert np.linalg.norm(last["forces"] - f) <= 1e-14 * np.linalg.norm(f)
