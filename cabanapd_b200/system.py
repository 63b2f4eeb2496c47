"""Python binding of the C ABI (include/cabanapd_b200.h) via ctypes.

The CUDA library is the only compute path: if libcabanapd_b200.so is
missing, or no CUDA device is present, System() raises. There is no CPU
fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcabanapd_b200.so")

FIELDS = {"x": 0, "u": 1, "v": 2, "f": 3, "vol": 4, "rho": 5, "m": 6,
          "theta": 7, "W": 8, "phi": 9, "radius": 10, "stress": 11}
VECTOR_FIELDS = {"x", "u", "v", "f"}


def _field_shape(field, n):
    if field in VECTOR_FIELDS:
        return (n, 3)
    if field == "stress":
        return (n, 3, 3)
    return (n,)
FP64_EXACT = 0
FP64 = 1
MIXED = 2
ORDER_INPUT, ORDER_MORTON = 0, 1

_lib = None


class CpdParams(ctypes.Structure):
    _fields_ = [
        ("pd_model", ctypes.c_int32),
        ("fracture", ctypes.c_int32),
        ("influence_type", ctypes.c_int32),
        ("contact_model", ctypes.c_int32),
        ("horizon", ctypes.c_double),
        ("K", ctypes.c_double),
        ("G", ctypes.c_double),
        ("G0", ctypes.c_double),
        ("contact_radius", ctypes.c_double),
        ("radius_extend", ctypes.c_double),
        ("nu", ctypes.c_double),
        ("E", ctypes.c_double),
        ("restitution", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("rebuild_every", ctypes.c_int32),
        ("per_particle_radius", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("ordering", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("contact_horizon", ctypes.c_double),
        ("contact_K", ctypes.c_double),
    ]


class CpdError(RuntimeError):
    pass


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("max_active", ctypes.c_int32),
        ("steps_per_launch", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
        ("hbm_budget_bytes", ctypes.c_uint64),
        ("setup_threads", ctypes.c_int32),
        ("batch_max_particles", ctypes.c_int32),
        ("evict_after_s", ctypes.c_double),
    ]


class JobStatus(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int32),
        ("steps", ctypes.c_int32),
        ("steps_done", ctypes.c_int32),
        ("priority", ctypes.c_int32),
        ("n", ctypes.c_int64),
        ("bonds", ctypes.c_int64),
        ("device_bytes", ctypes.c_uint64),
        ("submit_time", ctypes.c_double),
        ("admit_time", ctypes.c_double),
        ("ready_time", ctypes.c_double),
        ("start_time", ctypes.c_double),
        ("finish_time", ctypes.c_double),
        ("total_strain_energy", ctypes.c_double),
        ("total_damage", ctypes.c_double),
        ("kernel_launches", ctypes.c_int64),
        ("evictions", ctypes.c_int64),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64),
        ("done", ctypes.c_int64),
        ("failed", ctypes.c_int64),
        ("resident", ctypes.c_int64),
        ("queued", ctypes.c_int64),
        ("resident_bytes", ctypes.c_uint64),
        ("peak_resident_bytes", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_int64),
        ("bond_updates", ctypes.c_double),
    ]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3


# Every symbol the header declares, with its ctypes signature.
_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "cpd_abi_version": (_I32, []),
    "cpd_state_bytes": (_I32, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "cpd_step_energy": (_I32, [_P, _I32, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double)]),
    "cpd_save_state": (_I32, [_P, ctypes.c_void_p, ctypes.c_uint64]),
    "cpd_load_state": (_I32, [_P, ctypes.c_void_p, ctypes.c_uint64]),
    "cpd_last_error": (ctypes.c_char_p, []),
    "cpd_system_create": (_I32, [ctypes.POINTER(CpdParams), ctypes.POINTER(_P)]),
    "cpd_system_destroy": (_I32, [_P]),
    "cpd_set_stream": (_I32, [_P, _P]),
    "cpd_get_stream": (_I32, [_P, ctypes.POINTER(_P)]),
    "cpd_model_constants": (_I32, [_P, _DP]),
    "cpd_upload_particles": (_I32, [_P, _I64, _I64, _P, _P, _P, _P, _P]),
    "cpd_set_state": (_I32, [_P, _P, _P]),
    "cpd_build_neighbors": (_I32, [_P]),
    "cpd_neighbor_stats": (_I32, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I64)]),
    "cpd_download_neighbors": (_I32, [_P, _P, _P, _P]),
    "cpd_prenotch": (_I32, [_P, _I32, _P, _P, _P]),
    "cpd_add_boundary_condition": (_I32, [_P, _I32, _I32, _I64, _P, _P]),
    "cpd_clear_boundary_conditions": (_I32, [_P]),
    "cpd_compute_weighted_volume": (_I32, [_P]),
    "cpd_compute_dilatation": (_I32, [_P]),
    "cpd_compute_force": (_I32, [_P]),
    "cpd_compute_energy": (_I32, [_P, _DP, _DP]),
    "cpd_compute_stress": (_I32, [_P]),
    "cpd_compute_energy_noalloc": (_I32, [_P, _P, _P, _P]),
    "cpd_init": (_I32, [_P]),
    "cpd_step": (_I32, [_P, _I32]),
    "cpd_synchronize": (_I32, [_P]),
    "cpd_step_stage": (_I32, [_P, _I32]),
    "cpd_download": (_I32, [_P, _I32, _P]),
    "cpd_max_displacement": (_D, [_P]),
    "cpd_contact_rebuilds": (_I64, [_P]),
    "cpd_device_field": (_I32, [_P, _I32, ctypes.POINTER(_P), ctypes.POINTER(_I64)]),
    "cpd_bond_bits": (_I32, [_P, ctypes.POINTER(_P), ctypes.POINTER(_I32),
                             ctypes.POINTER(_I64)]),
    "cpd_set_kernel_timing": (_I32, [_P, _I32]),
    "cpd_kernel_time": (_I32, [_P, _DP, ctypes.POINTER(_I64), _DP]),
    "cpd_kernel_launches": (_I64, [_P]),
    "cpd_stencil_stats": (_I32, [_P, ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ctypes.c_int32)]),
    "cpd_device_bytes": (_I32, [_P, ctypes.POINTER(ctypes.c_uint64)]),
    "cpd_batch_create": (_I32, [ctypes.POINTER(_P), _I32, ctypes.POINTER(_I32),
                                ctypes.POINTER(_P)]),
    "cpd_batch_destroy": (_I32, [_P]),
    "cpd_batch_step": (_I32, [_P, _I32]),
    "cpd_batch_remaining": (_I32, [_P, _I32, ctypes.POINTER(_I32)]),
    "cpd_batch_release": (_I32, [_P, _I32]),
    "cpd_batch_synchronize": (_I32, [_P]),
    "cpd_batch_set_candidate": (_I32, [_P, _I32]),
    "cpd_batch_tuning": (_I32, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I32),
                                ctypes.POINTER(_I32), ctypes.POINTER(_I32), _DP]),
    "cpd_batch_launches": (_I64, [_P]),
    "cpd_job_create": (_I32, [ctypes.POINTER(CpdParams), _I32, ctypes.POINTER(_P)]),
    "cpd_job_destroy": (_I32, [_P]),
    "cpd_job_set_particles": (_I32, [_P, _I64, _I64, _P, _P, _P, _P, _P]),
    "cpd_job_set_state": (_I32, [_P, _P, _P]),
    "cpd_job_prenotch": (_I32, [_P, _I32, _P, _P, _P]),
    "cpd_job_add_boundary_condition": (_I32, [_P, _I32, _I32, _I64, _P, _P]),
    "cpd_job_keep_fields": (_I32, [_P, ctypes.c_uint32]),
    "cpd_server_create": (_I32, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]),
    "cpd_server_destroy": (_I32, [_P]),
    "cpd_server_submit": (_I32, [_P, _P, ctypes.POINTER(_I64)]),
    "cpd_server_clock": (_D, [_P]),
    "cpd_server_wait": (_I32, [_P, _I64, _D]),
    "cpd_server_drain": (_I32, [_P, _D]),
    "cpd_server_job_status": (_I32, [_P, _I64, ctypes.POINTER(JobStatus)]),
    "cpd_server_job_error": (_I32, [_P, _I64, ctypes.c_char_p, _I64]),
    "cpd_server_download": (_I32, [_P, _I64, _I32, _P]),
    "cpd_server_release": (_I32, [_P, _I64]),
    "cpd_server_evict": (_I32, [_P, _I64]),
    "cpd_server_stats_get": (_I32, [_P, ctypes.POINTER(ServerStats)]),
}


def load(path=LIB_PATH):
    """Load the CUDA library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CpdError(
            f"{path} not found: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()' or make -C "
            "cabanapd_b200/csrc)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data


class System:
    """One simulation on the GPU (a cpd_system handle)."""

    backend = "cuda"

    def __init__(self, params, device=0, precision=FP64_EXACT, ordering=ORDER_INPUT):
        lib = load()
        p = _params_struct(params, precision, ordering, device)
        self._lib = lib
        h = _P()
        self._check(lib.cpd_system_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.n = 0

    def _check(self, rc):
        if rc != 0:
            raise CpdError(f"cabanapd_b200 error {rc}: {self._lib.cpd_last_error().decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cpd_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def model_constants(self):
        out = np.zeros(10)
        self._check(self._lib.cpd_model_constants(self._h, out.ctypes.data_as(_DP)))
        keys = ["c", "s0", "bond_break_coeff", "theta_coeff", "s_coeff", "Rs",
                "Es", "beta", "coeff_h_n", "coeff_h_d"]
        return dict(zip(keys, out.tolist()))

    def set_particles(self, x, vol, rho=None, nofail=None, radius=None, n_frozen=0):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        n = x.shape[0]
        vol = np.ascontiguousarray(vol, dtype=np.float64)
        rho = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        nofail = None if nofail is None else np.ascontiguousarray(nofail, dtype=np.int32)
        radius = None if radius is None else np.ascontiguousarray(radius, dtype=np.float64)
        self._check(self._lib.cpd_upload_particles(
            self._h, n, int(n_frozen), _ptr(x), _ptr(vol), _ptr(rho), _ptr(nofail),
            _ptr(radius)))
        self.n = n

    def set_state(self, u=None, v=None):
        u = None if u is None else np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        v = None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.cpd_set_state(self._h, _ptr(u), _ptr(v)))

    def build_neighbors(self):
        self._check(self._lib.cpd_build_neighbors(self._h))

    def neighbor_stats(self):
        mx, tot = _I32(), _I64()
        self._check(self._lib.cpd_neighbor_stats(self._h, ctypes.byref(mx), ctypes.byref(tot)))
        return mx.value, tot.value

    def neighbors(self):
        mx, _ = self.neighbor_stats()
        counts = np.zeros(self.n, dtype=np.int32)
        idx = np.zeros((self.n, max(mx, 1)), dtype=np.int32)
        mu = np.zeros((self.n, max(mx, 1)), dtype=np.int32)
        self._check(self._lib.cpd_download_neighbors(self._h, _ptr(counts), _ptr(idx), _ptr(mu)))
        return counts, idx[:, :mx], mu[:, :mx]

    def prenotch(self, v1, v2, p0):
        v1 = np.ascontiguousarray(v1, dtype=np.float64).reshape(-1, 3)
        v2 = np.ascontiguousarray(v2, dtype=np.float64).reshape(-1, 3)
        p0 = np.ascontiguousarray(p0, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.cpd_prenotch(self._h, p0.shape[0], _ptr(v1), _ptr(v2), _ptr(p0)))

    def add_bc(self, kind, indices, values, component=0):
        idx = np.ascontiguousarray(indices, dtype=np.int64)
        vals = np.ascontiguousarray(np.atleast_1d(values), dtype=np.float64)
        self._check(self._lib.cpd_add_boundary_condition(
            self._h, int(kind), int(component), idx.size, _ptr(idx), _ptr(vals)))

    def clear_bcs(self):
        self._check(self._lib.cpd_clear_boundary_conditions(self._h))

    def compute_weighted_volume(self):
        self._check(self._lib.cpd_compute_weighted_volume(self._h))

    def compute_dilatation(self):
        self._check(self._lib.cpd_compute_dilatation(self._h))

    def compute_force(self):
        self._check(self._lib.cpd_compute_force(self._h))

    def compute_energy(self):
        w, d = _D(), _D()
        self._check(self._lib.cpd_compute_energy(self._h, ctypes.byref(w), ctypes.byref(d)))
        return w.value, d.value

    def compute_stress(self):
        """Per-particle stress of the current state (get("stress") -> [n, 3, 3])."""
        self._check(self._lib.cpd_compute_stress(self._h))

    def init(self):
        self._check(self._lib.cpd_init(self._h))

    def step(self, num_steps):
        """Queue num_steps steps (asynchronous)."""
        self._check(self._lib.cpd_step(self._h, int(num_steps)))

    def step_energy(self, num_steps):
        """num_steps steps, then the (strain energy, damage) totals of the
        final state (cpd_step_energy: the Solver's output step)."""
        w, d = _D(), _D()
        self._check(self._lib.cpd_step_energy(self._h, int(num_steps), ctypes.byref(w),
                                              ctypes.byref(d)))
        return w.value, d.value

    def run(self, num_steps):
        self.step(num_steps)
        self.synchronize()

    def synchronize(self):
        self._check(self._lib.cpd_synchronize(self._h))

    def step_stage(self, stage):
        """One stage of a time step (0 initial half, 1 force, 2 force BCs,
        3 final half), queued asynchronously."""
        self._check(self._lib.cpd_step_stage(self._h, int(stage)))

    def get(self, field, out=None):
        shape = _field_shape(field, self.n)
        if out is None:
            out = np.zeros(shape)
        self._check(self._lib.cpd_download(self._h, FIELDS[field], out.ctypes.data))
        return out

    def max_displacement(self):
        return self._lib.cpd_max_displacement(self._h)

    def contact_rebuilds(self):
        return self._lib.cpd_contact_rebuilds(self._h)

    def device_field(self, field):
        ptr, stride = _P(), _I64()
        self._check(self._lib.cpd_device_field(self._h, FIELDS[field], ctypes.byref(ptr),
                                               ctypes.byref(stride)))
        return ptr.value, stride.value

    def bond_bits(self):
        """(device pointer, words, stride) of the broken-bond bits
        (cpd_bond_bits): uint32 [words][stride], internal order."""
        ptr, words, stride = _P(), _I32(), _I64()
        self._check(self._lib.cpd_bond_bits(self._h, ctypes.byref(ptr), ctypes.byref(words),
                                            ctypes.byref(stride)))
        return ptr.value, words.value, stride.value

    def set_stream(self, stream_handle):
        self._check(self._lib.cpd_set_stream(self._h, stream_handle))

    def get_stream(self):
        s = _P()
        self._check(self._lib.cpd_get_stream(self._h, ctypes.byref(s)))
        return s.value

    def set_kernel_timing(self, enable=True):
        self._check(self._lib.cpd_set_kernel_timing(self._h, 1 if enable else 0))

    def kernel_time(self):
        ms, n, b = _D(), _I64(), _D()
        self._check(self._lib.cpd_kernel_time(self._h, ctypes.byref(ms), ctypes.byref(n),
                                              ctypes.byref(b)))
        return ms.value, n.value, b.value

    def kernel_launches(self):
        return self._lib.cpd_kernel_launches(self._h)

    def stencil_stats(self):
        """(warps on the lattice-stencil bond kernels, warps on the general
        kernels beside them, offset-table entries); zeros when the general
        kernels take every row."""
        w, r, t = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        self._check(self._lib.cpd_stencil_stats(self._h, ctypes.byref(w), ctypes.byref(r),
                                                ctypes.byref(t)))
        return w.value, r.value, t.value

    def save_state(self):
        """Snapshot of the evolving state (cpd_save_state) as a uint8 array."""
        nbytes = ctypes.c_uint64()
        self._check(self._lib.cpd_state_bytes(self._h, ctypes.byref(nbytes)))
        buf = np.empty(nbytes.value, dtype=np.uint8)
        self._check(self._lib.cpd_save_state(self._h, buf.ctypes.data, buf.size))
        return buf

    def load_state(self, buf):
        """Restore a snapshot taken from a system set up the same way."""
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        self._check(self._lib.cpd_load_state(self._h, buf.ctypes.data, buf.size))


class Batch:
    """Many set-up systems advanced together (a cpd_batch handle): per time
    step one persistent-block launch covers every instance, and k-step chunks
    replay from a CUDA graph. The systems stay usable for reads (energy,
    fields); state-changing calls on them fail until the batch is closed.
    steps[i]: the total number of steps system i is to take."""

    def __init__(self, systems, steps):
        lib = load()
        self._lib = lib
        self.systems = list(systems)
        n = len(self.systems)
        hs = (_P * n)(*[s.handle for s in self.systems])
        st = (_I32 * n)(*[int(k) for k in steps])
        h = _P()
        self._check(lib.cpd_batch_create(hs, n, st, ctypes.byref(h)))
        self._h = h

    def _check(self, rc):
        if rc != 0:
            raise CpdError(f"cabanapd_b200 error {rc}: {self._lib.cpd_last_error().decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cpd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, chunk_steps):
        """One chunk: every instance takes min(chunk_steps, its steps left)."""
        self._check(self._lib.cpd_batch_step(self._h, int(chunk_steps)))

    def run(self, chunk_steps=32):
        """Chunks until every instance has taken its steps; synchronises."""
        while max(self.remaining(i) for i in range(len(self.systems))) > 0:
            self.step(chunk_steps)
        self.synchronize()

    def release(self, instance):
        """Hand back a finished instance's system (it may step or be
        destroyed again) while the batch runs on."""
        self._check(self._lib.cpd_batch_release(self._h, int(instance)))

    def remaining(self, instance):
        r = _I32()
        self._check(self._lib.cpd_batch_remaining(self._h, int(instance), ctypes.byref(r)))
        return r.value

    def synchronize(self):
        self._check(self._lib.cpd_batch_synchronize(self._h))

    def set_candidate(self, candidate):
        """Fix the launch shape (-1: the autotuner chooses)."""
        self._check(self._lib.cpd_batch_set_candidate(self._h, int(candidate)))

    def tuning(self):
        """(chosen, [(blocks_per_sm, order, bond-updates/s), ...])."""
        n, chosen = _I32(), _I32()
        self._check(self._lib.cpd_batch_tuning(self._h, ctypes.byref(n), None, None, None, None))
        g = (_I32 * n.value)()
        o = (_I32 * n.value)()
        t = (_D * n.value)()
        self._check(self._lib.cpd_batch_tuning(self._h, ctypes.byref(n), ctypes.byref(chosen),
                                               g, o, t))
        return chosen.value, [(g[k], o[k], t[k]) for k in range(n.value)]

    def launches(self):
        return int(self._lib.cpd_batch_launches(self._h))


def _params_struct(params, precision=FP64_EXACT, ordering=ORDER_INPUT, device=0):
    p = CpdParams()
    p.influence_type = -1
    for k, _ in CpdParams._fields_:
        if k in params:
            setattr(p, k, params[k])
    p.precision = params.get("precision", precision)
    p.ordering = params.get("ordering", ordering)
    p.device = params.get("device", device)
    return p


class Server:
    """Job server (cpd_server): continuous batching of independent
    simulations on one GPU with admission against a device-memory budget.

    submit() takes a problem dict as built by cabanapd_b200.problems
    (params, x, vol, rho, nofail, radius, u0, v0, notches, bcs, num_steps)
    and returns a job id; results stay on the host until release()."""

    def __init__(self, device=0, max_active=16, steps_per_launch=32, use_graphs=True,
                 hbm_budget_bytes=150 * 10**9, setup_threads=4, batch_max_particles=0,
                 evict_after_s=0.0):
        lib = load()
        self._lib = lib
        cfg = ServerConfig(device, max_active, steps_per_launch, 1 if use_graphs else 0,
                           int(hbm_budget_bytes), int(setup_threads), int(batch_max_particles),
                           float(evict_after_s))
        h = _P()
        self._check(lib.cpd_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._n = {}

    def _check(self, rc):
        if rc != 0:
            raise CpdError(f"cabanapd_b200 error {rc}: {self._lib.cpd_last_error().decode()}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.cpd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self):
        return self._lib.cpd_server_clock(self._h)

    def submit(self, prob, precision=FP64_EXACT, keep=("u",)):
        lib = self._lib
        p = _params_struct(prob["params"], precision=precision)
        job = _P()
        self._check(lib.cpd_job_create(ctypes.byref(p), int(prob["num_steps"]), ctypes.byref(job)))
        submitted = False
        try:
            x = np.ascontiguousarray(prob["x"], dtype=np.float64).reshape(-1, 3)
            vol = np.ascontiguousarray(prob["vol"], dtype=np.float64)
            arrays = {}
            for key, dt in (("rho", np.float64), ("nofail", np.int32), ("radius", np.float64)):
                arrays[key] = (None if prob.get(key) is None
                               else np.ascontiguousarray(prob[key], dtype=dt))
            self._check(lib.cpd_job_set_particles(
                job, x.shape[0], int(prob.get("n_frozen", 0)), _ptr(x), _ptr(vol),
                _ptr(arrays["rho"]), _ptr(arrays["nofail"]), _ptr(arrays["radius"])))
            u0, v0 = prob.get("u0"), prob.get("v0")
            if u0 is not None or v0 is not None:
                u0 = None if u0 is None else np.ascontiguousarray(u0, dtype=np.float64)
                v0 = None if v0 is None else np.ascontiguousarray(v0, dtype=np.float64)
                self._check(lib.cpd_job_set_state(job, _ptr(u0), _ptr(v0)))
            if prob.get("notches") is not None:
                v1, v2, p0 = (np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 3)
                              for a in prob["notches"])
                self._check(lib.cpd_job_prenotch(job, v1.shape[0], _ptr(v1), _ptr(v2), _ptr(p0)))
            for kind, comp, idx, vals in prob.get("bcs", []):
                idx = np.ascontiguousarray(idx, dtype=np.int64)
                vals = np.ascontiguousarray(np.atleast_1d(vals), dtype=np.float64)
                self._check(lib.cpd_job_add_boundary_condition(
                    job, int(kind), int(comp), idx.shape[0], _ptr(idx), _ptr(vals)))
            mask = 0
            for f in keep:
                mask |= 1 << FIELDS[f]
            self._check(lib.cpd_job_keep_fields(job, mask))
            jid = _I64()
            submitted = True
            self._check(lib.cpd_server_submit(self._h, job, ctypes.byref(jid)))
        finally:
            if not submitted:
                lib.cpd_job_destroy(job)
        self._n[jid.value] = x.shape[0]
        return jid.value

    def wait(self, job_id, timeout=600.0):
        self._check(self._lib.cpd_server_wait(self._h, int(job_id), float(timeout)))
        return self.status(job_id)

    def drain(self, timeout=3600.0):
        self._check(self._lib.cpd_server_drain(self._h, float(timeout)))

    def status(self, job_id):
        st = JobStatus()
        self._check(self._lib.cpd_server_job_status(self._h, int(job_id), ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in JobStatus._fields_}

    def error(self, job_id):
        buf = ctypes.create_string_buffer(1024)
        self._check(self._lib.cpd_server_job_error(self._h, int(job_id), buf, 1024))
        return buf.value.decode()

    def get(self, job_id, field):
        n = self._n[job_id]
        out = np.empty(_field_shape(field, n), dtype=np.float64)
        self._check(self._lib.cpd_server_download(self._h, int(job_id), FIELDS[field],
                                                  out.ctypes.data))
        return out

    def evict(self, job_id):
        """Save a running job's state to the host, free its device memory and
        queue it again; it resumes from the snapshot."""
        self._check(self._lib.cpd_server_evict(self._h, int(job_id)))

    def release(self, job_id):
        self._check(self._lib.cpd_server_release(self._h, int(job_id)))
        self._n.pop(job_id, None)

    def stats(self):
        st = ServerStats()
        self._check(self._lib.cpd_server_stats_get(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}
