"""GPU test of cpd_compute_energy_noalloc, the energy/damage entry point for
callers that may not allocate device memory once a run has started (a job
server that reserved each job's memory at admission, or a framework that
owns all device memory through its own pool).

The test plays such a caller: its output buffers come from its own pool
(torch), and it checks the entry point against cpd_compute_energy on two
calls in a row, at two different states of a notched-plate run, on every
arithmetic path (bit-exact FP64, throughput FP64 and mixed precision, the
last also in its split form on a plate of over 2^20 rows), with frozen
rows, and checks that a system above the fixed scratch limit is refused.
Named to be collected last, and self-contained so it passes alone in a
fresh process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu

EXACT, FAST, MIXED = 0, 1, 2


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def _check_noalloc(prob, precision, step_blocks):
    import torch

    import cabanapd_b200
    lib = cabanapd_b200.load_library()
    sysm = cabanapd_b200.System(dict(prob["params"], device=0, precision=precision))
    P.setup(sysm, prob)
    _, stride = sysm.device_field("W")
    n, frozen = sysm.n, prob["n_frozen"]
    # NaN-filled caller buffers: every row the entry point leaves unwritten
    # would show up as NaN below.
    W_dev = torch.full((stride,), float("nan"), dtype=torch.float64, device="cuda:0")
    phi_dev = torch.full((stride,), float("nan"), dtype=torch.float64, device="cuda:0")
    totals = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()

    def noalloc():
        rc = lib.cpd_compute_energy_noalloc(sysm.handle, ctypes.c_void_p(W_dev.data_ptr()),
                                            ctypes.c_void_p(phi_dev.data_ptr()),
                                            ctypes.c_void_p(totals.data_ptr()))
        assert rc == 0, lib.cpd_last_error().decode()
        sysm.synchronize()
        return totals.cpu().numpy().copy(), W_dev.cpu().numpy()[:n], phi_dev.cpu().numpy()[:n]

    D_ref = 0.0
    for steps in step_blocks:
        sysm.run(steps)
        # Two calls in a row on the same state, then the allocating entry point.
        t1, w1, p1 = noalloc()
        t2, w2, p2 = noalloc()
        W_ref, D_ref = sysm.compute_energy()
        w_ref, phi_ref = sysm.get("W"), sysm.get("phi")
        for t, w, p in ((t1, w1, p1), (t2, w2, p2)):
            assert _rel(t[0], W_ref) <= 1e-12
            assert _rel(t[1], D_ref) <= 1e-12
            assert np.array_equal(w, w_ref)
            assert np.array_equal(p, phi_ref)
            if frozen:
                assert not np.any(w[:frozen]) and not np.any(p[:frozen])
    return D_ref


@pytest.mark.parametrize("precision", [EXACT, FAST, MIXED])
def test_energy_noalloc_matches_allocating_entry_point(precision):
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=120, v0=60.0)
    D = _check_noalloc(prob, precision, (0, 60))
    assert D > 0  # bonds were cut and broke, so damage is non-trivial


@pytest.mark.parametrize("precision", [FAST, MIXED])
def test_energy_noalloc_with_frozen_rows(precision):
    """The first 600 particles frozen: their W and phi rows read 0."""
    prob = P.plate_impact(num_cells=(48, 24, 6), steps=40, v0=60.0)
    prob["n_frozen"] = 600
    prob["bcs"] = [bc for bc in prob["bcs"] if np.all(np.asarray(bc[2]) >= 600)]
    _check_noalloc(prob, precision, (0, 20))


def test_energy_noalloc_mixed_split_form():
    """2^20 rows: the mixed energy pass runs as two launches (the lean warps,
    then the rest) whose partial rows both land in the fixed scratch."""
    prob = P.plate_impact(num_cells=(256, 128, 32), steps=4, v0=60.0)
    assert prob["x"].shape[0] >= 1 << 20
    _check_noalloc(prob, MIXED, (0, 2))


def test_energy_noalloc_rejects_missing_outputs():
    import cabanapd_b200
    lib = cabanapd_b200.load_library()
    prob = P.plate_impact(num_cells=(24, 12, 4), steps=1)
    sysm = cabanapd_b200.System(prob["params"])
    P.setup(sysm, prob)
    rc = lib.cpd_compute_energy_noalloc(sysm.handle, None, None, None)
    assert rc == 1  # CPD_ERR_INVALID_ARGUMENT
    assert b"device pointers" in lib.cpd_last_error()


def test_energy_noalloc_rejects_rows_above_the_limit():
    """4,194,305 rows (one past the scratch limit) are refused before any
    work is queued; a horizon below the spacing keeps the list empty."""
    import torch

    import cabanapd_b200
    lib = cabanapd_b200.load_library()
    n = 4194304 + 1
    x = np.zeros((n, 3))
    x[:, 0] = np.arange(n, dtype=np.float64)
    params = dict(pd_model=P.PD_PMB, fracture=1, horizon=0.5, K=1.0, G0=1.0, dt=1.0)
    sysm = cabanapd_b200.System(dict(params, device=0))
    sysm.set_particles(x, np.ones(n))
    sysm.build_neighbors()
    buf = torch.zeros((n + 256,), dtype=torch.float64, device="cuda:0")
    tot = torch.zeros((2,), dtype=torch.float64, device="cuda:0")
    rc = lib.cpd_compute_energy_noalloc(sysm.handle, ctypes.c_void_p(buf.data_ptr()),
                                        ctypes.c_void_p(buf.data_ptr()),
                                        ctypes.c_void_p(tot.data_ptr()))
    assert rc == 1  # CPD_ERR_INVALID_ARGUMENT
    assert b"4194304" in lib.cpd_last_error()
