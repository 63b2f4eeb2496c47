"""Batched step (cpd_batch_*): many systems advanced by one persistent-block
launch per time step, k-step chunks replayed from CUDA graphs, launch shape
picked by the autotuner.

The checks:
- an instance's results do not depend on the batch it runs in, its place
  in the batch or the launch shape: bit-identical alone, beside other
  instances of other models and sizes, and under every autotuner candidate,
  in both precisions;
- the FP64 instances run the FP64 throughput kernels' arithmetic: bit for
  bit the per-system cpd_step on the systems whose per-system path is those
  kernels (LPS, and PMB off a lattice), whatever the chunk length; and the
  FP64 plate against the oracle (identical broken-bond bits, fields within
  1e-12);
- mixed instances within the mixed tolerance of FP64 with the same broken
  bonds;
- frozen particles and boundary conditions; state changes refused while a
  system is batched; the tuner's record.
"""
import numpy as np
import pytest

from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu

FP64, MIXED = 1, 2


@pytest.fixture(scope="module")
def cuda():
    import cabanapd_b200
    return cabanapd_b200


def _nrel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _system(cuda, prob, precision):
    s = cuda.System(dict(prob["params"], precision=precision))
    P.setup(s, prob)
    return s


def _state(s):
    return {f: s.get(f) for f in ("u", "v", "f")} | {"bits": s.neighbors()[2]}


def _same(a, b):
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def _plate(steps=40):
    return P.plate_impact(num_cells=(48, 24, 4), steps=steps, v0=60.0)


def _lps(steps=30):
    return P.lps_random_notches(num_cells=(100, 40, 4), steps=steps)


def _jittered_wave(n=14, steps=30, seed=3):
    """The PMB elastic wave with positions moved off the lattice by up to
    1e-3 of a spacing: no stencil rows, so the per-system FP64 path runs the
    FP64 throughput kernel on every row."""
    prob = P.elastic_wave_pmb(n=n, steps=steps)
    rng = np.random.default_rng(seed)
    h = prob["dx"][0]
    prob["x"] = prob["x"] + (rng.random(prob["x"].shape) - 0.5) * 2e-3 * h
    return prob


def _frozen_plate(steps=40):
    prob = _plate(steps)
    nf = 48 * 24 + 10
    prob = dict(prob, n_frozen=nf)
    prob["bcs"] = [(k, c, idx[idx >= nf], v) for k, c, idx, v in prob["bcs"]]
    return prob


@pytest.mark.parametrize("make", [_lps, _jittered_wave, _frozen_plate])
def test_fp64_instance_equals_system_step(cuda, make):
    """LPS with fracture and traction, PMB off the lattice and a plate with
    frozen rows: a batched FP64 instance equals the per-system cpd_step bit
    for bit (where the per-system path is the FP64 throughput kernel), with
    chunks shorter than the run and a last partial chunk."""
    prob = make()
    steps = 37
    ref = _system(cuda, prob, FP64)
    ref.run(steps)
    s = _system(cuda, prob, FP64)
    b = cuda.Batch([s], [steps])
    b.run(chunk_steps=16)
    assert b.remaining(0) == 0
    b.close()
    if make is _frozen_plate:
        # The plate's per-system FP64 path is the lattice-stencil kernel, whose
        # rounding differs: the FP64 bar instead of bits.
        assert np.array_equal(s.neighbors()[2], ref.neighbors()[2])
        for f in ("u", "v", "f"):
            assert _nrel(s.get(f), ref.get(f)) <= 1e-12, f
        assert not np.any(s.get("u")[:prob["n_frozen"]])
    else:
        _same(_state(s), _state(ref))
    wb, db = s.compute_energy()
    wr, dr = ref.compute_energy()
    assert abs(wb - wr) <= 1e-12 * abs(wr) and abs(db - dr) <= 1e-12 * max(abs(dr), 1.0)


def test_fp64_plate_batch_matches_oracle(cuda, oracle):
    """PMB fracture plate in a batch beside an LPS box: against the oracle,
    identical broken-bond bits and fields within 1e-12 norm-wise."""
    prob = _plate(40)
    s = _system(cuda, prob, FP64)
    other = _system(cuda, _lps(), FP64)
    o = oracle.OracleSystem(prob["params"])
    P.setup(o, prob)
    b = cuda.Batch([other, s], [40, 40])
    b.run(chunk_steps=8)
    b.close()
    o.run(40)
    assert np.array_equal(s.neighbors()[2], o.neighbors()[2])
    assert (o.neighbors()[2] == 0).sum() > 0
    for f in ("u", "v", "f"):
        assert _nrel(s.get(f), o.get(f)) <= 1e-12, f


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_instance_independent_of_batch_and_launch_shape(cuda, precision):
    """The same plate and LPS box alone, in a batch with other instances of
    other sizes and models (in both orders), and under every launch-shape
    candidate: identical bits."""

    def run(probs, steps, candidate=-1, chunk=16):
        systems = [_system(cuda, p, precision) for p in probs]
        b = cuda.Batch(systems, steps)
        if candidate >= 0:
            b.set_candidate(candidate)
        b.run(chunk_steps=chunk)
        ncand = len(b.tuning()[1])
        b.close()
        return systems, ncand

    plate, lps = _plate(40), _lps(30)
    (alone_p,), ncand = run([plate], [40])
    (alone_l,), _ = run([lps], [30])
    ref_p, ref_l = _state(alone_p), _state(alone_l)
    mix, _ = run([_jittered_wave(n=10), lps, plate, _plate(40)], [25, 30, 40, 12], chunk=8)
    _same(_state(mix[2]), ref_p)
    _same(_state(mix[1]), ref_l)
    for cand in range(ncand):
        (sp, sl), _ = run([plate, lps], [40, 30], candidate=cand)
        _same(_state(sp), ref_p)
        _same(_state(sl), ref_l)


def test_mixed_batch_close_to_fp64(cuda):
    """Mixed plate and LPS box in one batch: within the mixed path's
    tolerance of the per-system FP64 runs, with the same broken bonds."""
    probs = [(_plate(40), 40), (_lps(30), 30)]
    systems = [_system(cuda, p, MIXED) for p, _ in probs]
    b = cuda.Batch(systems, [k for _, k in probs])
    b.run(chunk_steps=16)
    b.close()
    for s, (p, k) in zip(systems, probs):
        ref = _system(cuda, p, FP64)
        ref.run(k)
        assert np.array_equal(s.neighbors()[2], ref.neighbors()[2])
        assert _nrel(s.get("u"), ref.get("u")) <= 1e-6
        assert _nrel(s.get("v"), ref.get("v")) <= 1e-5


def test_batched_system_refuses_state_changes(cuda):
    """While batched, a system refuses steps and state changes but serves
    reads; closing the batch releases it. Exact-precision and contact
    systems are not batched."""
    s = _system(cuda, _plate(10), FP64)
    b = cuda.Batch([s], [10])
    b.step(4)
    with pytest.raises(cuda.CpdError):
        s.step(1)
    with pytest.raises(cuda.CpdError):
        s.set_state(np.zeros((s.n, 3)), None)
    with pytest.raises(cuda.CpdError):
        cuda.Batch([s], [5])
    w, _ = s.compute_energy()
    assert np.isfinite(w)
    b.close()
    s.step(1)
    exact = _system(cuda, _plate(10), 0)
    with pytest.raises(cuda.CpdError):
        cuda.Batch([exact], [5])
    dem = _system(cuda, P.hertz_two_spheres(), FP64)
    with pytest.raises(cuda.CpdError):
        cuda.Batch([dem], [5])


def test_autotuner_times_each_candidate_then_keeps_the_fastest(cuda):
    systems = [_system(cuda, p, MIXED) for p in (_plate(400), _lps(400))]
    b = cuda.Batch(systems, [400, 400])
    chosen, cands = b.tuning()
    assert chosen == -1 and len(cands) >= 4
    for _ in range(len(cands)):
        b.step(16)
        b.synchronize()
    chosen, cands = b.tuning()
    assert 0 <= chosen < len(cands)
    rates = [t for _, _, t in cands]
    assert all(r > 0 for r in rates)
    assert rates[chosen] == max(rates)
    kernels_per_chunk = 2 + 16 * 3 + 1  # half steps, LPS + bond passes, advance
    assert b.launches() <= len(cands) * kernels_per_chunk
    b.close()


def test_release_finished_instance_while_the_batch_runs(cuda):
    """An instance with fewer steps is handed back once done (then it steps
    and is destroyed on its own) while the others run on, unchanged."""
    lps, plate = _lps(30), _plate(40)
    (ref,) = [_system(cuda, plate, FP64)]
    rb = cuda.Batch([ref], [40])
    rb.run(chunk_steps=8)
    rb.close()
    short = _system(cuda, lps, FP64)
    s = _system(cuda, plate, FP64)
    b = cuda.Batch([short, s], [12, 40])
    with pytest.raises(cuda.CpdError):
        b.release(0)
    b.step(8)
    b.step(8)
    assert b.remaining(0) == 0
    b.release(0)
    short.step(3)
    short.close()
    while b.remaining(1) > 0:
        b.step(8)
    b.close()
    _same(_state(s), _state(ref))
