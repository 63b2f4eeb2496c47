"""ctypes binding of the CPU oracle (oracle/oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline legs as the checker / CPU baseline. The product
package (cabanapd_b200) never imports this module.

The class mirrors cabanapd_b200.System method-for-method so that a problem
description can be run on either backend with the same driver code.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

FIELDS = {"x": 0, "u": 1, "v": 2, "f": 3, "vol": 4, "rho": 5, "m": 6,
          "theta": 7, "W": 8, "phi": 9, "radius": 10, "stress": 11}
VECTOR_FIELDS = {"x", "u", "v", "f"}


class OrcParams(ctypes.Structure):
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
        ("contact_horizon", ctypes.c_double),
        ("contact_K", ctypes.c_double),
    ]


def build():
    """Compile the oracle library with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    P = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.orc_create.restype = P
    lib.orc_create.argtypes = [ctypes.POINTER(OrcParams)]
    lib.orc_destroy.argtypes = [P]
    lib.orc_last_error.restype = ctypes.c_char_p
    lib.orc_model_constants.argtypes = [P, dp]
    lib.orc_set_particles.argtypes = [P, ctypes.c_int64, ctypes.c_int64, dp, dp,
                                      dp, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_set_state.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
    lib.orc_set_field.argtypes = [P, ctypes.c_int32, dp]
    lib.orc_build_neighbors.argtypes = [P]
    lib.orc_neighbor_stats.argtypes = [P, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.POINTER(ctypes.c_int64)]
    lib.orc_get_neighbors.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]
    lib.orc_prenotch.argtypes = [P, ctypes.c_int32, dp, dp, dp]
    lib.orc_get_bond_bits.argtypes = [P, ctypes.c_void_p]
    lib.orc_add_bc.argtypes = [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64,
                               ctypes.c_void_p, dp]
    for name in ("orc_compute_weighted_volume", "orc_compute_dilatation",
                 "orc_compute_force", "orc_compute_stress", "orc_init"):
        getattr(lib, name).argtypes = [P]
    lib.orc_compute_energy.argtypes = [P, dp, dp]
    lib.orc_run.argtypes = [P, ctypes.c_int32]
    lib.orc_get.argtypes = [P, ctypes.c_int32, dp]
    lib.orc_max_displacement.restype = ctypes.c_double
    lib.orc_max_displacement.argtypes = [P]
    lib.orc_contact_rebuilds.restype = ctypes.c_int64
    lib.orc_contact_rebuilds.argtypes = [P]
    lib.orc_critical_timestep.restype = ctypes.c_double
    lib.orc_critical_timestep.argtypes = [ctypes.c_double] * 3 + [
        ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double]
    lib.orc_num_threads.restype = ctypes.c_int
    lib.orc_set_num_threads.argtypes = [ctypes.c_int32]
    _lib = lib
    return lib


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleSystem:
    """One oracle simulation; same call surface as cabanapd_b200.System."""

    backend = "oracle"

    def __init__(self, params):
        lib = load()
        p = OrcParams(**{k: params[k] for k, _ in OrcParams._fields_ if k in params})
        if "influence_type" not in params:
            p.influence_type = -1
        self._lib = lib
        self._h = lib.orc_create(ctypes.byref(p))
        if not self._h:
            raise RuntimeError(lib.orc_last_error().decode())
        self.n = 0

    def close(self):
        if self._h:
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self._lib.orc_last_error().decode())

    def model_constants(self):
        out = np.zeros(10)
        self._lib.orc_model_constants(self._h, _dptr(out))
        keys = ["c", "s0", "bond_break_coeff", "theta_coeff", "s_coeff", "Rs",
                "Es", "beta", "coeff_h_n", "coeff_h_d"]
        return dict(zip(keys, out.tolist()))

    def set_particles(self, x, vol, rho=None, nofail=None, radius=None, n_frozen=0):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        n = x.shape[0]
        vol = np.ascontiguousarray(vol, dtype=np.float64)
        self._keep = []
        rho_a = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64)
        nf = None if nofail is None else np.ascontiguousarray(nofail, dtype=np.int32)
        rad = None if radius is None else np.ascontiguousarray(radius, dtype=np.float64)
        self._check(self._lib.orc_set_particles(
            self._h, n, n_frozen, _dptr(x), _dptr(vol),
            _dptr(rho_a) if rho_a is not None else None,
            nf.ctypes.data if nf is not None else None,
            rad.ctypes.data if rad is not None else None))
        self.n = n

    def set_state(self, u=None, v=None):
        ua = None if u is None else np.ascontiguousarray(u, dtype=np.float64).reshape(-1, 3)
        va = None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.orc_set_state(
            self._h, ua.ctypes.data if ua is not None else None,
            va.ctypes.data if va is not None else None))

    def set_field(self, field, values):
        """Overwrite a whole vector field ("u", "v" or "f"), [n][3]."""
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.orc_set_field(self._h, FIELDS[field], _dptr(a)))

    def build_neighbors(self):
        self._check(self._lib.orc_build_neighbors(self._h))

    def neighbor_stats(self):
        mx = ctypes.c_int32()
        tot = ctypes.c_int64()
        self._lib.orc_neighbor_stats(self._h, ctypes.byref(mx), ctypes.byref(tot))
        return mx.value, tot.value

    def neighbors(self):
        mx, _ = self.neighbor_stats()
        counts = np.zeros(self.n, dtype=np.int32)
        idx = np.zeros((self.n, max(mx, 1)), dtype=np.int32)
        mu = np.zeros((self.n, max(mx, 1)), dtype=np.int32)
        self._lib.orc_get_neighbors(self._h, counts.ctypes.data, idx.ctypes.data,
                                    mu.ctypes.data)
        return counts, idx[:, :mx], mu[:, :mx]

    def bond_bits(self):
        """Broken-bond state packed as uint32 [words][n] (the product's
        cpd_bond_bits layout without its row padding)."""
        mx, _ = self.neighbor_stats()
        bits = np.zeros(((mx + 31) // 32, self.n), dtype=np.uint32)
        self._check(self._lib.orc_get_bond_bits(self._h, bits.ctypes.data))
        return bits

    def prenotch(self, v1, v2, p0):
        v1 = np.ascontiguousarray(v1, dtype=np.float64).reshape(-1, 3)
        v2 = np.ascontiguousarray(v2, dtype=np.float64).reshape(-1, 3)
        p0 = np.ascontiguousarray(p0, dtype=np.float64).reshape(-1, 3)
        self._check(self._lib.orc_prenotch(self._h, p0.shape[0], _dptr(v1),
                                           _dptr(v2), _dptr(p0)))

    def add_bc(self, kind, indices, values, component=0):
        idx = np.ascontiguousarray(indices, dtype=np.int64)
        vals = np.ascontiguousarray(np.atleast_1d(values), dtype=np.float64)
        self._check(self._lib.orc_add_bc(self._h, kind, component, idx.size,
                                         idx.ctypes.data, _dptr(vals)))

    def compute_weighted_volume(self):
        self._check(self._lib.orc_compute_weighted_volume(self._h))

    def compute_dilatation(self):
        self._check(self._lib.orc_compute_dilatation(self._h))

    def compute_force(self):
        self._check(self._lib.orc_compute_force(self._h))

    def compute_energy(self):
        w = ctypes.c_double()
        d = ctypes.c_double()
        self._check(self._lib.orc_compute_energy(self._h, ctypes.byref(w), ctypes.byref(d)))
        return w.value, d.value

    def init(self):
        self._check(self._lib.orc_init(self._h))

    def run(self, num_steps):
        self._check(self._lib.orc_run(self._h, int(num_steps)))

    def compute_stress(self):
        self._check(self._lib.orc_compute_stress(self._h))

    def get(self, field):
        if field in VECTOR_FIELDS:
            out = np.zeros((self.n, 3))
        elif field == "stress":
            out = np.zeros((self.n, 3, 3))
        else:
            out = np.zeros(self.n)
        self._check(self._lib.orc_get(self._h, FIELDS[field], _dptr(out)))
        return out

    def max_displacement(self):
        return self._lib.orc_max_displacement(self._h)

    def contact_rebuilds(self):
        return self._lib.orc_contact_rebuilds(self._h)


def critical_timestep(dx, dy, dz, m, horizon, K, rho):
    return load().orc_critical_timestep(dx, dy, dz, m, horizon, K, rho)


def set_num_threads(n):
    load().orc_set_num_threads(int(n))


def num_threads():
    return load().orc_num_threads()
