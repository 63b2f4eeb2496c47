"""The reference's own example programs, unchanged, on the B200 path.

oracle/reference_programs.mk compiles CabanaPD's examples/mechanics/
kalthoff_winkler.cpp, examples/mechanics/elastic_wave.cpp and
examples/dem/powder_fill.cpp from the CabanaPD tree, without edits, against
include/CabanaPD.hpp (with include/cabanapd_shim/compat standing in for
<mpi.h> and <Kokkos_Core.hpp>) into oracle/_ref/. That is the drop-in claim:
an existing CabanaPD program and input deck drive the GPU library.

GPU tests run the binaries with the reference's regression decks (from
tests/golden/reference_expectations.json) and apply the reference's own
regression checks:
- regression_test/tstKalthoffWinkler.hpp:53, max crack y 7.42e-2 +- 1.1e-4,
  read from the last line of output_kw_crack_y.txt as that test reads it;
- regression_test/tstElasticWave.hpp:54-96, the displacement profile against
  the fitted polynomial.
Each result also equals, bit for bit, the same deck run through this
repository's own example program (examples/*.cpp), which tests/test_shim.py
ties to the Python-driven run and so to the oracle.

The powder fill has no regression check in the reference; a shortened deck
(200 steps) must run, keep the container frozen, and move the powder down
under gravity.
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_BIN = os.path.join(ROOT, "oracle", "_ref")
OWN_BIN = os.path.join(ROOT, "examples", "_build")
PROGRAMS = ("kalthoff_winkler", "elastic_wave", "powder_fill")


def _exe(name, own=False):
    exe = os.path.join(OWN_BIN if own else REF_BIN, name)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} is not built (oracle/reference_programs.mk needs the CabanaPD tree)")
    return exe


def _run(exe, deck, workdir, precision="fp64", env_extra=None):
    os.makedirs(workdir, exist_ok=True)
    path = os.path.join(workdir, "deck.json")
    with open(path, "w") as fh:
        json.dump(deck, fh)
    env = dict(os.environ, CABANAPD_B200_PRECISION=precision, **(env_extra or {}))
    r = subprocess.run([exe, path], cwd=workdir, env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


# ---------------------------------------------------------------------------
# CPU


@pytest.mark.parametrize("name", PROGRAMS)
def test_reference_program_links_the_library(name):
    """A built reference program is linked against this repository's C ABI
    library (and against no Kokkos, Cabana or MPI library)."""
    exe = _exe(name)
    r = subprocess.run(["ldd", exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    assert "libcabanapd_b200.so" in r.stdout
    for other in ("kokkos", "cabana.so", "libmpi"):
        assert other not in r.stdout.lower()


# ---------------------------------------------------------------------------
# GPU


def _last_value(path):
    last = None
    with open(path) as fh:
        for line in fh:
            if line.strip():
                last = float(line.split()[0])
    return last


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["exact", "fp64", "mixed"])
def test_kalthoff_winkler_reference_program(golden, tmp_path, precision):
    """tstKalthoffWinkler's check on the reference's own program, and the
    same output series as this repository's example program."""
    g = golden["kalthoff_winkler"]
    _run(_exe("kalthoff_winkler"), g["input"], str(tmp_path / "ref"), precision)
    y = _last_value(tmp_path / "ref" / "output_kw_crack_y.txt")
    assert abs(y - g["max_crack_y"]) <= g["tolerance"], y
    _run(_exe("kalthoff_winkler", own=True), g["input"], str(tmp_path / "own"), precision)
    a = np.loadtxt(tmp_path / "ref" / "output_kw_crack_y.txt", ndmin=2)
    b = np.loadtxt(tmp_path / "own" / "output_kw_crack_y.txt", ndmin=2)
    assert np.array_equal(a, b)


@pytest.mark.gpu
def test_elastic_wave_reference_program(golden, tmp_path):
    """tstElasticWave's profile check on the reference's own program
    (LinearLPS, 41^3), equal to this repository's example program."""
    from test_oracle_regression import elastic_wave_profile_errors
    g = golden["elastic_wave"]
    _run(_exe("elastic_wave"), g["input"], str(tmp_path / "ref"), "exact")
    prof = np.loadtxt(tmp_path / "ref" / "displacement_profile.txt", ndmin=2)
    assert prof.shape[0] == 41
    rel, l2 = elastic_wave_profile_errors(golden, prof[:, 1], prof[:, 2])
    assert rel < g["rel_tol"] and l2 < g["l2_tol"], (rel, l2)
    _run(_exe("elastic_wave", own=True), g["input"], str(tmp_path / "own"), "exact")
    own = np.loadtxt(tmp_path / "own" / "displacement_profile.txt", ndmin=2)
    assert np.array_equal(prof, own)


def _powder_deck(steps):
    # examples/dem/inputs/powder_fill.json, shortened to `steps` steps.
    dt = 2e-6
    return {
        "num_cells": {"value": [50, 50, 25]},
        "system_size": {"value": [0.25, 0.25, 0.125]},
        "density": {"value": 2.0e3}, "volume": {"value": 6.544985e-8},
        "elastic_modulus": {"value": 1.0e5}, "poisson_ratio": {"value": 0.25},
        "restitution": {"value": 0.5}, "radius": {"value": 2.5e-3},
        "radius_extend": {"value": 2.5e-3}, "cylinder_diameter": {"value": 0.25},
        "wall_thickness": {"value": 0.0045}, "min_height": {"value": 0.01},
        "final_time": {"value": (steps + 0.5) * dt}, "timestep": {"value": dt},
        "timestep_safety_factor": {"value": 0.9}, "output_frequency": {"value": steps},
        "output_reference": {"value": False},
    }


@pytest.mark.gpu
def test_powder_fill_reference_program(tmp_path):
    """The reference's powder fill (Hertzian contact, frozen container,
    gravity body term, Solver::remove) runs 200 steps on the GPU: the
    container stays put and the powder falls."""
    from test_shim import read_xdmf_particles
    steps = 200
    _run(_exe("powder_fill"), _powder_deck(steps), str(tmp_path), "fp64",
         env_extra={"CABANAPD_B200_PARTICLE_OUTPUT": "1"})
    outs = sorted((f for f in os.listdir(tmp_path) if f.endswith(".xmf")),
                  key=lambda f: int(f.split("_")[1].split(".")[0]))
    assert outs, os.listdir(tmp_path)
    _, fields = read_xdmf_particles(str(tmp_path / outs[-1]))
    u = fields["displacements"]
    v = fields["velocities"]
    assert np.all(np.isfinite(u)) and np.all(np.isfinite(v))
    moving = np.any(v != 0.0, axis=1)
    assert 0 < moving.sum() < u.shape[0]          # frozen container, moving powder
    assert np.all(u[~moving] == 0.0)
    t = steps * 2e-6
    # Free fall over t: v_z = -g t for a powder particle out of contact.
    assert np.median(v[moving, 2]) == pytest.approx(-9.8 * t, rel=1e-2)
