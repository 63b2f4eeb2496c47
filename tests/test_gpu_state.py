"""State snapshots (cpd_save_state / cpd_load_state): a run stopped, saved,
restored into a freshly set-up system and continued equals the
uninterrupted run bit for bit, on every precision path and with contact
lists rebuilt inside the interval.
"""
import numpy as np
import pytest

from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda():
    import cabanapd_b200
    return cabanapd_b200


def _system(cuda, prob, precision, ordering=0):
    s = cuda.System(dict(prob["params"], precision=precision, ordering=ordering))
    return P.setup(s, prob)


def _state(s):
    return [s.get(f) for f in ("u", "v", "f")] + [s.neighbors()[2]]


CASES = {
    "plate": (lambda: P.plate_impact(num_cells=(96, 48, 6), steps=120, v0=60.0), 60, 60),
    "lps": (lambda: P.lps_random_notches(num_cells=(100, 40, 4), steps=60), 30, 30),
    "cylinder": (lambda: P.fragmenting_cylinder(num_cells=(60, 60, 40), size=(0.06, 0.06, 0.04),
                                                height=0.03, steps=30), 15, 15),
    "dem": (lambda: P.dem_packing(lattice_dims=(16, 16, 8), steps=60, spacing=2.1e-3, dt=1e-7),
            25, 35),
}


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("case", sorted(CASES))
def test_restart_equals_uninterrupted_run(cuda, case, precision):
    make, first, second = CASES[case]
    prob = make()
    whole = _system(cuda, prob, precision)
    whole.run(first + second)
    part = _system(cuda, prob, precision)
    part.run(first)
    snap = part.save_state()
    rebuilds = part.contact_rebuilds()
    part.close()
    resumed = _system(cuda, prob, precision)
    resumed.load_state(snap)
    assert resumed.contact_rebuilds() == rebuilds
    resumed.run(second)
    for a, b in zip(_state(resumed), _state(whole)):
        assert np.array_equal(a, b)
    assert resumed.contact_rebuilds() == whole.contact_rebuilds()
    if prob["params"].get("pd_model", 0):
        assert resumed.compute_energy() == whole.compute_energy()


def test_restart_with_morton_order(cuda):
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=80, v0=60.0)
    whole = _system(cuda, prob, 2, ordering=1)
    whole.run(80)
    part = _system(cuda, prob, 2, ordering=1)
    part.run(40)
    resumed = _system(cuda, prob, 2, ordering=1)
    resumed.load_state(part.save_state())
    resumed.run(40)
    for a, b in zip(_state(resumed), _state(whole)):
        assert np.array_equal(a, b)


def test_snapshot_of_another_system_is_rejected(cuda):
    prob = P.plate_impact(num_cells=(48, 24, 4), steps=10, v0=60.0)
    s = _system(cuda, prob, 2)
    s.run(5)
    snap = s.save_state()
    other = _system(cuda, P.plate_impact(num_cells=(40, 24, 4), steps=10, v0=60.0), 2)
    with pytest.raises(cuda.CpdError, match="set up differently"):
        other.load_state(snap)
    with pytest.raises(cuda.CpdError, match="not a state snapshot"):
        s.load_state(np.zeros_like(snap))
    with pytest.raises(cuda.CpdError, match="truncated"):
        s.load_state(snap[:-8])
