"""One simulation split across ranks (one GPU each): slab decomposition with
ghost particles, the single-job form of the reference's halo exchange
(src/CabanaPD_Comm.hpp:233-438: a persistent Cabana::Gather of u, and m /
theta for LPS, to the neighbouring ranks every step, called from
src/CabanaPD_Solver.hpp:466-473).

Layout. The particles are cut into slabs along one axis (whole lattice
planes, about the same number of particles per slab). A rank's system holds
its own particles and, as ghosts, every particle of another slab within a
halo of its slab along that axis: delta for PMB, 2 delta for LPS. Local rows
keep the global particle order (ascending global index), so every owned
row sees the neighbours it has in the whole system, in the same order, and
its bond terms are summed in the same order: the owned rows' results are the
single-system results (bit for bit where the arithmetic is EXACT).

Ghosts are ordinary rows of the local system: each rank integrates them
itself. Their own forces come from incomplete neighbourhoods and are
discarded: after every step the owners send (u, v, f) of the ghost rows, and
the next first half step then moves every ghost exactly as its owner moves
it. With the LPS halo of 2 delta, the ghosts within delta of the slab have
complete neighbourhoods, so their dilatation, which the owned rows' forces
read, is the owner's. One exchange per step (72 bytes per ghost); the step
itself stays the fused cpd_step (first half step, then one bond launch that
also applies the boundary conditions and the second half step). Broken-bond
decisions depend on positions only, so every copy of a bond decides alike.

Transport: torch.distributed point-to-point (NCCL between GPUs, gloo on the
CPU) through DistExchange, or in one process for several shards
(step_in_process). The rank-local engine is any object with the System
call surface (cabanapd_b200.System on the GPU).

Not sharded: contact models (their lists follow current positions).
"""
import numpy as np

from . import problems as P


class SlabPartition:
    """Slabs of whole lattice planes along `axis` for `world` ranks, and each
    rank's local particle set (owned + ghosts within `halo`)."""

    def __init__(self, x, world, axis, halo):
        coord = np.asarray(x)[:, axis]
        planes, counts = np.unique(coord, return_counts=True)
        if len(planes) < world:
            raise ValueError(f"{len(planes)} planes along axis {axis} for {world} ranks")
        cum = np.cumsum(counts)
        n = int(cum[-1])
        bounds = [0]
        for r in range(1, world):
            k = int(np.searchsorted(cum, r * n / world)) + 1
            k = max(bounds[-1] + 1, min(k, len(planes) - (world - r)))
            bounds.append(k)
        bounds.append(len(planes))
        plane = np.searchsorted(planes, coord)
        self.owner = (np.searchsorted(np.asarray(bounds[1:-1]), plane, side="right")
                      .astype(np.int64))
        self.world = world
        self.local = []
        for r in range(world):
            lo = planes[bounds[r]] - halo
            hi = planes[bounds[r + 1] - 1] + halo
            self.local.append(np.nonzero((coord >= lo) & (coord <= hi))[0].astype(np.int64))

    def plan(self, rank):
        """Local rows to send to / receive from every other rank: rank q
        needs, for its ghosts owned here, their current state."""
        send, recv = {}, {}
        mine = self.local[rank]
        own = self.owner[mine]
        for q in range(self.world):
            if q == rank:
                continue
            theirs = self.local[q]
            need = theirs[self.owner[theirs] == rank]       # q's ghosts owned here
            if need.size:
                send[q] = np.searchsorted(mine, need)
            ghosts = np.nonzero(own == q)[0]                 # my ghosts owned by q
            if ghosts.size:
                recv[q] = ghosts
        return send, recv


def _halo(params):
    if params.get("contact_model", P.CONTACT_NONE) != P.CONTACT_NONE:
        raise ValueError("contact models are not sharded")
    delta = float(params["horizon"])
    lps = params.get("pd_model") in (P.PD_LPS, P.PD_LINEAR_LPS)
    return (2.0 if lps else 1.0) * delta * (1.0 + 1e-9)


def local_problem(prob, rows, owned_mask):
    """The sub-problem of the given global rows (ascending): particle arrays,
    initial state, frozen count, notches, and the force boundary conditions
    of the owned rows (ghost rows take their state from their owners)."""
    rows = np.asarray(rows)
    sub = dict(prob)
    for key in ("x", "vol", "rho", "nofail", "radius", "u0", "v0"):
        if prob.get(key) is not None:
            sub[key] = np.ascontiguousarray(np.asarray(prob[key])[rows])
    sub["n_frozen"] = int(np.count_nonzero(rows < int(prob.get("n_frozen", 0))))
    pos = {int(g): k for k, g in enumerate(rows)}
    bcs = []
    for kind, comp, idx, vals in prob.get("bcs", []):
        idx = np.asarray(idx)
        vals = np.atleast_1d(np.asarray(vals, dtype=np.float64))
        keep = [k for k, g in enumerate(idx) if int(g) in pos and owned_mask[pos[int(g)]]]
        local_idx = np.array([pos[int(idx[k])] for k in keep], dtype=np.int64)
        if kind == P.BC_FORCE_ADD:
            local_vals = vals[keep] if len(keep) else np.zeros(0)
        else:
            local_vals = vals
        bcs.append((kind, comp, local_idx, local_vals))
    sub["bcs"] = bcs
    return sub


class _DeviceRows:
    """(u, v, f) rows of a CUDA system, read and written in place on the
    device (cpd_device_field: component-major [3][stride] in the caller's
    order)."""

    def __init__(self, system):
        import torch
        self._views = {}
        for name in ("u", "v", "f"):
            ptr, stride = system.device_field(name)
            holder = type("DevArray", (), {})()
            holder.__cuda_array_interface__ = {
                "shape": (3, stride), "typestr": "<f8", "data": (ptr, False),
                "version": 3, "strides": None}
            self._views[name] = torch.as_tensor(holder, device="cuda")
        self._torch = torch

    def read(self, rows):
        idx = self._torch.as_tensor(rows, device="cuda")
        return self._torch.cat([self._views[k][:, idx] for k in ("u", "v", "f")], dim=0)

    def write(self, rows, data):
        idx = self._torch.as_tensor(rows, device="cuda")
        for c, k in enumerate(("u", "v", "f")):
            self._views[k][:, idx] = data[3 * c:3 * c + 3].to(self._views[k].dtype)
        # The system's own stream does not order against torch's: the next
        # step must see these rows.
        self._torch.cuda.current_stream().synchronize()


class _HostRows:
    """(u, v, f) rows of a host engine with get / set_field."""

    def __init__(self, system):
        self._s = system

    def read(self, rows):
        import torch
        return torch.as_tensor(np.concatenate([self._s.get(k)[rows].T for k in ("u", "v", "f")]))

    def write(self, rows, data):
        data = data.cpu().numpy()
        for c, k in enumerate(("u", "v", "f")):
            a = self._s.get(k)
            a[rows] = data[3 * c:3 * c + 3].T
            self._s.set_field(k, a)


class ShardedSystem:
    """Rank `rank` of `world` of one simulation. make_system(params) returns
    the rank-local engine (cabanapd_b200.System, or any object with its call
    surface); prob is the whole problem (every rank builds it alike)."""

    def __init__(self, prob, rank, world, make_system, axis=1):
        self.rank, self.world = rank, world
        part = SlabPartition(prob["x"], world, axis, _halo(prob["params"]))
        self.rows = part.local[rank]                     # local row -> global index
        self.owned = part.owner[self.rows] == rank       # local rows owned here
        self.send, self.recv = part.plan(rank)
        self.n_global = len(prob["x"])
        self.system = make_system(dict(prob["params"]))
        P.setup(self.system, local_problem(prob, self.rows, self.owned))
        self._io = (_DeviceRows(self.system) if hasattr(self.system, "device_field")
                    else _HostRows(self.system))

    # -- one step and its exchange, in parts (step_in_process drives them) --
    def advance(self):
        self.system.run(1)

    def pack(self):
        return {q: self._io.read(rows) for q, rows in self.send.items()}

    def unpack(self, received):
        for q, rows in self.recv.items():
            self._io.write(rows, received[q])

    def recv_shapes(self):
        return {q: (9, len(rows)) for q, rows in self.recv.items()}

    # -- with torch.distributed ----------------------------------------------
    def step(self, num_steps, exchange):
        for _ in range(num_steps):
            self.advance()
            self.unpack(exchange.exchange(self.pack(), self.recv_shapes()))

    def owned_totals(self):
        """This rank's share of (total strain energy, total damage): the
        reference's sums over its owned rows (strain energy density times
        volume, and damage)."""
        self.system.compute_energy()
        W = self.system.get("W")[self.owned]
        vol = self.system.get("vol")[self.owned]
        phi = self.system.get("phi")[self.owned]
        return float(np.sum(W * vol)), float(np.sum(phi))

    def owned_field(self, field):
        """(global indices, values) of the owned rows."""
        return self.rows[self.owned], self.system.get(field)[self.owned]


class DistExchange:
    """Ghost-state exchange over torch.distributed point-to-point operations
    (NCCL with CUDA tensors, gloo with CPU tensors)."""

    def __init__(self, group=None, device="cpu"):
        import torch.distributed as dist
        self.dist, self.group, self.device = dist, group, device

    def exchange(self, sends, recv_shapes):
        import torch
        ops, out = [], {}
        for q, shape in sorted(recv_shapes.items()):
            out[q] = torch.empty(shape, dtype=torch.float64, device=self.device)
            ops.append(self.dist.P2POp(self.dist.irecv, out[q], q, self.group))
        for q, data in sorted(sends.items()):
            ops.append(self.dist.P2POp(self.dist.isend,
                                       data.to(self.device).contiguous(), q, self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        return out

    def totals(self, shard):
        import torch
        w, d = shard.owned_totals()
        t = torch.tensor([w, d], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return float(t[0]), float(t[1])

    def gather(self, shard, field):
        """The whole field in global order on every rank."""
        idx, vals = shard.owned_field(field)
        parts = [None] * shard.world
        self.dist.all_gather_object(parts, (idx, vals), group=self.group)
        out = np.zeros((shard.n_global,) + vals.shape[1:])
        for i, v in parts:
            out[i] = v
        return out


def step_in_process(shards, num_steps):
    """Advance shards of one simulation held in one process in lockstep
    (the exchange passes the packed tensors directly)."""
    for _ in range(num_steps):
        for s in shards:
            s.advance()
        packs = [s.pack() for s in shards]
        for s in shards:
            s.unpack({q: packs[q][s.rank] for q in s.recv})


def gather_in_process(shards, field):
    out = None
    for s in shards:
        idx, vals = s.owned_field(field)
        if out is None:
            out = np.zeros((s.n_global,) + vals.shape[1:])
        out[idx] = vals
    return out
