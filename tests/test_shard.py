"""Single-job sharding (cabanapd_b200.shard): slabs with ghost rows, one
(u, v, f) exchange per step.

CPU: two gloo ranks (torch.distributed point-to-point, as between GPUs with
NCCL), each advancing its slab on the oracle as the rank-local engine, must
give the single-system run bit for bit (owned rows keep their global
neighbour order, and the oracle's arithmetic is the reference's), with the
same broken bonds; the PMB plate (halo delta) and the LPS box (halo
2 delta). Three shards in one process as well.
GPU: two shards on one device in one process (no kernel waits on another)
against the single CUDA system, EXACT and FP64.
"""
import os
import socket

import numpy as np
import pytest

from cabanapd_b200 import problems as P
from cabanapd_b200 import shard


def _plate():
    return P.plate_impact(num_cells=(40, 24, 4), steps=30, v0=60.0)


def _lps():
    return P.lps_random_notches(num_cells=(60, 30, 3), steps=20)


def _single(oracle, prob):
    o = oracle.OracleSystem(prob["params"])
    P.setup(o, prob)
    o.run(prob["num_steps"])
    return o


def _global_bonds(system, rows, owned):
    """Owned rows' neighbours (global indices) and bond states."""
    counts, idx, mu = system.neighbors()
    out = {}
    for k in np.nonzero(owned)[0]:
        c = counts[k]
        out[int(rows[k])] = (tuple(rows[idx[k, :c]]), tuple(mu[k, :c]))
    return out


def _check_against_single(oracle, prob, u, v, f, totals, bonds):
    o = _single(oracle, prob)
    assert np.array_equal(u, o.get("u"))
    assert np.array_equal(v, o.get("v"))
    assert np.array_equal(f, o.get("f"))
    w, d = o.compute_energy()
    assert abs(totals[0] - w) <= 1e-12 * abs(w) and abs(totals[1] - d) <= 1e-12 * max(abs(d), 1)
    counts, idx, mu = o.neighbors()
    for g, (nbrs, states) in bonds.items():
        c = counts[g]
        assert nbrs == tuple(idx[g, :c]) and states == tuple(mu[g, :c]), g
    return o


def test_slab_partition_owns_every_particle_once():
    x, _, _ = P.lattice([0, 0, 0], [1, 1, 1], [7, 11, 5])
    part = shard.SlabPartition(x, 3, 1, 0.2)
    per = np.bincount(part.owner, minlength=3)
    assert per.sum() == len(x) and per.min() > 0
    assert per.max() - per.min() <= 7 * 5          # whole planes of 7 x 5 particles
    for r in range(3):
        loc = part.local[r]
        assert np.all(np.diff(loc) > 0)
        assert set(np.nonzero(part.owner == r)[0]) <= set(loc)
    send, recv = part.plan(1)
    assert set(send) == set(recv) == {0, 2}


@pytest.mark.parametrize("make", [_plate, _lps])
def test_three_shards_in_process_equal_the_single_run(oracle, make):
    prob = make()
    shards = [shard.ShardedSystem(prob, r, 3, oracle.OracleSystem) for r in range(3)]
    shard.step_in_process(shards, prob["num_steps"])
    u = shard.gather_in_process(shards, "u")
    v = shard.gather_in_process(shards, "v")
    f = shard.gather_in_process(shards, "f")
    parts = [s.owned_totals() for s in shards]
    totals = (sum(p[0] for p in parts), sum(p[1] for p in parts))
    bonds = {}
    for s in shards:
        bonds.update(_global_bonds(s.system, s.rows, s.owned))
    o = _check_against_single(oracle, prob, u, v, f, totals, bonds)
    if prob["params"].get("fracture"):
        assert (o.neighbors()[2] == 0).sum() > 0


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, which, outdir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import pyoracle
        pyoracle.load()
        prob = _plate() if which == "plate" else _lps()
        s = shard.ShardedSystem(prob, rank, world, pyoracle.OracleSystem)
        ex = shard.DistExchange()
        s.step(prob["num_steps"], ex)
        fields = {k: ex.gather(s, k) for k in ("u", "v", "f")}
        totals = ex.totals(s)
        bonds = _global_bonds(s.system, s.rows, s.owned)
        parts = [None] * world
        dist.all_gather_object(parts, bonds)
        if rank == 0:
            merged = {}
            for p in parts:
                merged.update(p)
            np.savez(os.path.join(outdir, "out.npz"), u=fields["u"], v=fields["v"],
                     f=fields["f"], totals=np.array(totals))
            import pickle
            with open(os.path.join(outdir, "bonds.pkl"), "wb") as fh:
                pickle.dump(merged, fh)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("which", ["plate", "lps"])
def test_two_gloo_ranks_equal_the_single_run(oracle, tmp_path, which):
    import pickle

    import torch.multiprocessing as mp
    mp.start_processes(_rank_main, args=(2, _free_port(), which, str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    out = np.load(tmp_path / "out.npz")
    with open(tmp_path / "bonds.pkl", "rb") as fh:
        bonds = pickle.load(fh)
    prob = _plate() if which == "plate" else _lps()
    _check_against_single(oracle, prob, out["u"], out["v"], out["f"], tuple(out["totals"]),
                          bonds)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_two_shards_on_one_gpu_equal_the_single_system(precision):
    import cabanapd_b200
    prob = _plate()

    def make(params):
        return cabanapd_b200.System(dict(params, precision=precision))

    shards = [shard.ShardedSystem(prob, r, 2, make) for r in range(2)]
    shard.step_in_process(shards, prob["num_steps"])
    single = make(prob["params"])
    P.setup(single, prob)
    single.run(prob["num_steps"])
    for fld in ("u", "v", "f"):
        assert np.array_equal(shard.gather_in_process(shards, fld), single.get(fld)), fld
    parts = [s.owned_totals() for s in shards]
    w, d = single.compute_energy()
    assert abs(sum(p[0] for p in parts) - w) <= 1e-12 * abs(w)
    assert abs(sum(p[1] for p in parts) - d) <= 1e-12 * max(abs(d), 1)
