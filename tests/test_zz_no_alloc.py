"""GPU test of cpd_compute_energy_noalloc, the energy/damage entry point for
callers that may not allocate device memory once a run has started (a job
server that reserved each job's memory at admission, or a framework that
owns all device memory through its own pool).

The test plays such a caller: its output buffers come from its own pool
(torch), and it checks the entry point against cpd_compute_energy on two
calls in a row, at two different states of a notched-plate run. Named to
be collected last, and self-contained so it passes alone in a fresh process
as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_energy_noalloc_matches_allocating_entry_point():
    import torch

    import cabanapd_b200
    lib = cabanapd_b200.load_library()
    prob = P.plate_impact(num_cells=(96, 48, 6), steps=120, v0=60.0)
    sysm = cabanapd_b200.System(dict(prob["params"], device=0))
    P.setup(sysm, prob)
    _, stride = sysm.device_field("W")
    n = sysm.n
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

    for steps in (0, 60):
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
    assert D_ref > 0  # bonds were cut and broke, so damage is non-trivial


def test_energy_noalloc_rejects_missing_outputs():
    import cabanapd_b200
    lib = cabanapd_b200.load_library()
    prob = P.plate_impact(num_cells=(24, 12, 4), steps=1)
    sysm = cabanapd_b200.System(prob["params"])
    P.setup(sysm, prob)
    rc = lib.cpd_compute_energy_noalloc(sysm.handle, None, None, None)
    assert rc == 1  # CPD_ERR_INVALID_ARGUMENT
    assert b"device pointers" in lib.cpd_last_error()
