"""The job server (cpd_server_*): continuous batching of independent
simulations on one GPU.

The acceptance test of serving: every job's result is the same alone and in
the mix. Jobs own their arrays and streams and every kernel is
deterministic, so the tolerance is zero: a job's final displacement and
velocity fields and its energy/damage totals computed by the server while
other jobs run are bit-identical to a plain System running that job alone,
in every precision mode. Further tests: admission respects the device-memory
budget, graph replay equals direct stepping, and failures stay confined to
their job. The host-side job description needs no GPU (CPU test).
"""
import ctypes
import time

import numpy as np
import pytest

from cabanapd_b200 import problems as P


def _solo(lib, prob, precision):
    s = lib.System(dict(prob["params"], precision=precision))
    P.setup(s, prob)
    s.run(prob["num_steps"])
    W, D = s.compute_energy()
    return s.get("u"), s.get("v"), W, D


def test_job_description_needs_no_gpu():
    """cpd_job_* only copy host arrays; submitting needs a server, and
    creating a server without a CUDA device fails cleanly."""
    import torch
    from cabanapd_b200 import system
    lib = system.load()
    prob = P.plate_impact(num_cells=(24, 12, 2), steps=5)
    p = system._params_struct(prob["params"])
    job = ctypes.c_void_p()
    assert lib.cpd_job_create(ctypes.byref(p), 5, ctypes.byref(job)) == 0
    x = np.ascontiguousarray(prob["x"])
    assert lib.cpd_job_set_particles(job, x.shape[0], 0, x.ctypes.data,
                                     prob["vol"].ctypes.data, None, None, None) == 0
    assert lib.cpd_job_keep_fields(job, 1 << 20) != 0  # unknown field bit
    assert lib.cpd_job_keep_fields(job, (1 << system.FIELDS["u"]) |
                                   (1 << system.FIELDS["phi"])) == 0
    assert lib.cpd_job_destroy(job) == 0
    if not torch.cuda.is_available():
        with pytest.raises(system.CpdError):
            system.Server()


@pytest.fixture(scope="module")
def lib():
    import cabanapd_b200
    return cabanapd_b200


def _mix(count=8, seed=7):
    return P.served_jobs(count=count, n_range=(1.5e3, 6e4), steps_range=(20, 90), seed=seed)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_each_job_same_alone_and_in_the_mix(lib, precision):
    jobs = _mix()
    srv = lib.Server(max_active=8, steps_per_launch=16)
    ids = [srv.submit(j, precision=precision, keep=("u", "v")) for j in jobs]
    srv.drain(timeout=600)
    stats = srv.stats()
    assert stats["done"] == len(jobs) and stats["failed"] == 0
    for jid, prob in zip(ids, jobs):
        st = srv.status(jid)
        assert st["state"] == lib.system.JOB_DONE and st["steps_done"] == prob["num_steps"]
        u, v, W, D = _solo(lib, prob, precision)
        assert np.array_equal(srv.get(jid, "u"), u), prob["kind"]
        assert np.array_equal(srv.get(jid, "v"), v), prob["kind"]
        assert (st["total_strain_energy"], st["total_damage"]) == (W, D)
    srv.close()


def _solo_batch(lib, prob, precision, chunk=16):
    s = lib.System(dict(prob["params"], precision=precision))
    P.setup(s, prob)
    b = lib.Batch([s], [prob["num_steps"]])
    b.run(chunk_steps=chunk)
    b.close()
    W, D = s.compute_energy()
    return s.get("u"), s.get("v"), W, D


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [1, 2])
def test_batched_jobs_same_alone_and_in_the_mix(lib, precision):
    """Batch groups on (every job small enough): jobs set up together share
    one batch, and each job's fields and totals equal the same job advanced
    alone in a batch of its own, bit for bit."""
    jobs = _mix(count=10, seed=13)
    srv = lib.Server(max_active=10, steps_per_launch=16, batch_max_particles=10**6)
    ids = [srv.submit(j, precision=precision, keep=("u", "v")) for j in jobs]
    srv.drain(timeout=600)
    stats = srv.stats()
    assert stats["done"] == len(jobs) and stats["failed"] == 0
    for jid, prob in zip(ids, jobs):
        st = srv.status(jid)
        assert st["state"] == lib.system.JOB_DONE and st["steps_done"] == prob["num_steps"]
        u, v, W, D = _solo_batch(lib, prob, precision)
        assert np.array_equal(srv.get(jid, "u"), u), prob["kind"]
        assert np.array_equal(srv.get(jid, "v"), v), prob["kind"]
        assert (st["total_strain_energy"], st["total_damage"]) == (W, D)
    srv.close()


@pytest.mark.gpu
def test_jobs_admitted_while_others_run(lib):
    """Continuous batching: short jobs submitted after a long one are
    admitted and finish while the long one is still on the GPU."""
    long_job = P.plate_impact(num_cells=(200, 100, 9), steps=1500)
    short = P.served_jobs(count=4, n_range=(2e3, 2e4), steps_range=(50, 100), seed=9)
    srv = lib.Server(max_active=8, steps_per_launch=32)
    first = srv.submit(long_job, precision=2)
    t_end = time.time() + 120
    while srv.status(first)["state"] == lib.system.JOB_QUEUED and time.time() < t_end:
        time.sleep(0.001)
    assert srv.status(first)["state"] == lib.system.JOB_RUNNING
    rest = [srv.submit(j, precision=2) for j in short]
    srv.drain(timeout=600)
    lf = srv.status(first)
    for jid in rest:
        st = srv.status(jid)
        assert st["state"] == lib.system.JOB_DONE
        assert lf["start_time"] < st["start_time"] and st["finish_time"] < lf["finish_time"]
    srv.close()


@pytest.mark.gpu
def test_admission_respects_the_memory_budget(lib):
    jobs = _mix(count=6, seed=11)
    probe = lib.Server(max_active=1)
    sizes = []
    for j in jobs:
        jid = probe.submit(j, precision=2)
        sizes.append(probe.wait(jid)["device_bytes"])
    probe.close()
    budget = int(1.6 * max(sizes))
    srv = lib.Server(max_active=6, steps_per_launch=16, hbm_budget_bytes=budget)
    ids = [srv.submit(j, precision=2) for j in jobs]
    srv.drain(timeout=600)
    st = srv.stats()
    assert st["done"] == len(jobs)
    assert st["peak_resident_bytes"] <= budget
    for jid, prob in zip(ids, jobs):
        u, _, _, _ = _solo(lib, prob, 2)
        assert np.array_equal(srv.get(jid, "u"), u)
    srv.close()


@pytest.mark.gpu
def test_graph_replay_equals_direct_steps(lib):
    jobs = _mix(count=4, seed=3)
    out = []
    for graphs in (True, False):
        srv = lib.Server(max_active=4, steps_per_launch=8, use_graphs=graphs)
        ids = [srv.submit(j, precision=2) for j in jobs]
        srv.drain(timeout=600)
        out.append([srv.get(i, "u") for i in ids])
        srv.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_failures_stay_with_their_job(lib):
    good = _mix(count=2, seed=5)
    bad = dict(good[0], params=dict(good[0]["params"], pd_model=P.PD_LINEAR_PMB, fracture=1))
    srv = lib.Server(max_active=4, hbm_budget_bytes=2 * 10**8)
    big = P.plate_impact(num_cells=(400, 200, 18), steps=10)
    ids = [srv.submit(good[0], precision=2), srv.submit(bad, precision=2),
           srv.submit(big, precision=2), srv.submit(good[1], precision=2)]
    srv.drain(timeout=600)
    states = [srv.status(i)["state"] for i in ids]
    assert states == [lib.system.JOB_DONE, lib.system.JOB_FAILED, lib.system.JOB_FAILED,
                      lib.system.JOB_DONE]
    assert "fracture" in srv.error(ids[1])
    assert "budget" in srv.error(ids[2])
    with pytest.raises(lib.CpdError):
        srv.get(ids[1], "u")
    srv.release(ids[1])
    with pytest.raises(lib.CpdError):
        srv.status(ids[1])
    srv.close()


def _wait_steps(srv, jid, steps, timeout=120.0):
    t_end = time.time() + timeout
    while srv.status(jid)["steps_done"] < steps and time.time() < t_end:
        time.sleep(0.002)
    return srv.status(jid)


@pytest.mark.gpu
def test_evicted_job_resumes_bit_identical(lib):
    """A running job evicted on request (its state saved to the host, its
    device memory freed) is set up again and resumes from the snapshot: its
    fields and totals equal the uninterrupted run bit for bit."""
    prob = P.plate_impact(num_cells=(120, 60, 6), steps=600)
    srv = lib.Server(max_active=2, steps_per_launch=16)
    jid = srv.submit(prob, precision=1, keep=("u", "v"))
    st = _wait_steps(srv, jid, 64)
    assert st["state"] == lib.system.JOB_RUNNING and st["steps_done"] < prob["num_steps"]
    srv.evict(jid)
    srv.drain(timeout=600)
    st = srv.status(jid)
    assert st["state"] == lib.system.JOB_DONE and st["steps_done"] == prob["num_steps"]
    assert st["evictions"] == 1
    u, v, W, D = _solo(lib, prob, 1)
    assert np.array_equal(srv.get(jid, "u"), u)
    assert np.array_equal(srv.get(jid, "v"), v)
    assert (st["total_strain_energy"], st["total_damage"]) == (W, D)
    srv.close()


@pytest.mark.gpu
def test_budget_pressure_evicts_the_long_job(lib):
    """A budget that holds one of two jobs: the short job that arrives while
    the long one runs waits evict_after_s, then the long job is evicted,
    the short one runs and finishes first, and the long one resumes; both
    equal their uninterrupted runs bit for bit."""
    long_job = P.plate_impact(num_cells=(200, 100, 9), steps=2000)
    short = P.plate_impact(num_cells=(80, 40, 4), steps=100)
    probe = lib.Server(max_active=1)
    sizes = [probe.wait(probe.submit(j, precision=2))["device_bytes"] for j in (long_job, short)]
    probe.close()
    budget = sizes[0] + sizes[1] // 2
    srv = lib.Server(max_active=4, steps_per_launch=16, hbm_budget_bytes=budget,
                     evict_after_s=0.05)
    a = srv.submit(long_job, precision=2, keep=("u",))
    _wait_steps(srv, a, 64)
    b = srv.submit(short, precision=2, keep=("u",))
    srv.drain(timeout=600)
    sa, sb = srv.status(a), srv.status(b)
    assert sa["state"] == sb["state"] == lib.system.JOB_DONE
    assert sa["evictions"] == 1 and sb["evictions"] == 0
    assert sb["finish_time"] < sa["finish_time"]
    assert srv.stats()["peak_resident_bytes"] <= budget
    for jid, prob in ((a, long_job), (b, short)):
        u, _, _, _ = _solo(lib, prob, 2)
        assert np.array_equal(srv.get(jid, "u"), u)
    srv.close()
