"""Single-point reference sums and analytic checks restated from the
reference's unit test unit_test/tstForce.hpp (lines cited per function).

They assume a full, uniform-volume lattice neighbourhood around a point and
are used by the tests exactly as the reference's checkResults /
checkParticle use them (tstForce.hpp:666-893).
"""
import math

import numpy as np


def _offsets(horizon, m):
    dx = horizon / m
    out = []
    for i in range(-m, m + 1):
        for j in range(-m, m + 1):
            for k in range(-m, m + 1):
                xi_x, xi_y, xi_z = dx * i, dx * j, dx * k
                xi = math.sqrt(xi_x * xi_x + xi_y * xi_y + xi_z * xi_z)
                if xi > 0.0 and xi < horizon + 1e-14:
                    out.append((xi_x, xi_y, xi_z, xi))
    return out, dx


class PMBRef:
    """force_models/CabanaPD_PMB.hpp:57-71 model functions."""

    def __init__(self, c):
        self.c = c

    def force_coeff(self, s, vol):
        return self.c * s * vol

    def energy(self, s, xi, vol):
        return 0.25 * self.c * s * s * xi * vol


class LPSRef:
    """force_models/CabanaPD_LPS.hpp:85-148 model functions."""

    def __init__(self, theta_coeff, s_coeff, influence_type):
        self.tc = theta_coeff
        self.sc = s_coeff
        self.infl_type = influence_type

    def influence(self, xi):
        return 1.0 / xi if self.infl_type == 1 else 1.0

    def force_coeff(self, s, xi, vol, m_i, m_j, th_i, th_j):
        return (self.tc * th_i / m_i + self.tc * th_j / m_j +
                s * (self.sc / m_i + self.sc / m_j)) * self.influence(xi) * xi * vol

    def energy(self, s, xi, vol, m_i, th_i, nb):
        return (1.0 / nb * 0.5 * self.tc / 3.0 * (th_i * th_i) +
                0.5 * (self.sc / m_i) * self.influence(xi) * s * s * xi * xi * vol)


def ref_neighbors(horizon, m):
    """tstForce.hpp:374-392 computeReferenceNeighbors."""
    return float(len(_offsets(horizon, m)[0]))


def ref_weighted_volume(model, horizon, m, vol):
    """tstForce.hpp:330-350."""
    offs, _ = _offsets(horizon, m)
    return sum(model.influence(xi) * xi * xi * vol for _, _, _, xi in offs)


def _quad_stretch(u11, x, xi_x, xi_y, xi_z, xi):
    eta_u = u11 * (2 * x * xi_x + xi_x * xi_x)
    rx = xi_x + eta_u
    r = math.sqrt(rx * rx + xi_y * xi_y + xi_z * xi_z)
    return (r - xi) / xi, rx, r


def ref_dilatation_linear(model, horizon, m, s0, vol, wv):
    """tstForce.hpp:352-372."""
    offs, _ = _offsets(horizon, m)
    return sum(3.0 / wv * model.influence(xi) * s0 * xi * xi * vol
               for _, _, _, xi in offs)


def ref_dilatation_quadratic(model, horizon, m, u11, vol, wv, x):
    """tstForce.hpp:395-421 (quadratic u_x = u11 x^2)."""
    total = 0.0
    for xi_x, xi_y, xi_z, xi in _offsets(horizon, m)[0]:
        s, _, _ = _quad_stretch(u11, x, xi_x, xi_y, xi_z, xi)
        total += 3.0 / wv * model.influence(xi) * s * xi * xi * vol
    return total


def ref_W(model, kind, horizon, m, coeff, x):
    """tstForce.hpp:136-196 (PMB) and :460-512 (LPS)."""
    offs, dx = _offsets(horizon, m)
    vol = dx * dx * dx
    total = 0.0
    if isinstance(model, PMBRef):
        for xi_x, xi_y, xi_z, xi in offs:
            s = coeff if kind == "linear" else _quad_stretch(coeff, x, xi_x, xi_y, xi_z, xi)[0]
            total += model.energy(s, xi, vol)
        return total
    wv = ref_weighted_volume(model, horizon, m, vol)
    nb = ref_neighbors(horizon, m)
    if kind == "linear":
        th = ref_dilatation_linear(model, horizon, m, coeff, vol, wv)
    else:
        th = ref_dilatation_quadratic(model, horizon, m, coeff, vol, wv, x)
    for xi_x, xi_y, xi_z, xi in offs:
        s = coeff if kind == "linear" else _quad_stretch(coeff, x, xi_x, xi_y, xi_z, xi)[0]
        total += model.energy(s, xi, vol, wv, th, nb)
    return total


def ref_fx(model, kind, horizon, m, u11, x):
    """tstForce.hpp:207-236 (PMB) and :514-553 (LPS); linear case is 0."""
    if kind == "linear":
        return 0.0
    offs, dx = _offsets(horizon, m)
    vol = dx * dx * dx
    total = 0.0
    if isinstance(model, PMBRef):
        for xi_x, xi_y, xi_z, xi in offs:
            s, rx, r = _quad_stretch(u11, x, xi_x, xi_y, xi_z, xi)
            total += model.force_coeff(s, vol) * rx / r
        return total
    wv = ref_weighted_volume(model, horizon, m, vol)
    th_i = ref_dilatation_quadratic(model, horizon, m, u11, vol, wv, x)
    for xi_x, xi_y, xi_z, xi in offs:
        s, rx, r = _quad_stretch(u11, x, xi_x, xi_y, xi_z, xi)
        th_j = ref_dilatation_quadratic(model, horizon, m, u11, vol, wv, x + xi_x)
        total += model.force_coeff(s, xi, vol, wv, wv, th_i, th_j) * rx / r
    return total


def ref_stress(model, kind, horizon, m, s0):
    """tstForce.hpp:91-133 (PMB) and :345-392 (LPS) computeReferenceStress:
    the diagonal (xx, yy, zz) at a point with a full neighbourhood under the
    linear field; the quadratic case is not computed (:394-399: zeros)."""
    if kind != "linear":
        return [0.0, 0.0, 0.0]
    offs, dx = _offsets(horizon, m)
    vol = dx * dx * dx
    sigma = [0.0, 0.0, 0.0]
    if isinstance(model, PMBRef):
        f_mag = model.force_coeff(s0, vol)
    else:
        wv = ref_weighted_volume(model, horizon, m, vol)
        th = ref_dilatation_linear(model, horizon, m, s0, vol, wv)
    for xi_x, xi_y, xi_z, xi in offs:
        if not isinstance(model, PMBRef):
            f_mag = model.force_coeff(s0, xi, vol, wv, wv, th, th)
        f_x = f_mag * xi_x / xi
        f_y = f_mag * xi_y / xi
        f_z = f_mag * xi_z / xi
        sigma[0] += 0.5 * f_x * xi_x
        sigma[1] += 0.5 * f_y * xi_y
        sigma[2] += 0.5 * f_z * xi_z
    return sigma


def float_eq(a, b, ulps=4):
    """GTest EXPECT_FLOAT_EQ: equal as floats within 4 ULPs."""
    fa, fb = np.float32(a), np.float32(b)
    if fa == fb:
        return True
    ia = np.array([fa], dtype=np.float32).view(np.int32)[0]
    ib = np.array([fb], dtype=np.float32).view(np.int32)[0]
    # map sign-magnitude to a monotonic integer line
    ia = ia if ia >= 0 else -(ia & 0x7FFFFFFF)
    ib = ib if ib >= 0 else -(ib & 0x7FFFFFFF)
    return abs(int(ia) - int(ib)) <= ulps


def analytic_W(model_kind, kind, K, G, coeff, horizon, x):
    """tstForce.hpp:777-832 checkAnalyticalStrainEnergy -> (value, rel band)
    (band None = FLOAT_EQ)."""
    if kind == "linear":
        val = 9.0 / 2.0 * K * coeff * coeff
        return val, (0.15 if model_kind == "pmb" else None)
    if model_kind == "pmb":
        return 18.0 * K * coeff * coeff * (1.0 / 5.0 * x * x + horizon * horizon / 42.0), 0.05
    return coeff * coeff * ((2.0 * K + 8.0 / 3.0 * G) * x * x +
                            75.0 / 2.0 * G * horizon * horizon / 49.0), 0.20


def analytic_fx(model_kind, K, G, coeff):
    """tstForce.hpp:834-862 checkAnalyticalForce (quadratic)."""
    if model_kind == "pmb":
        return 18.0 / 5.0 * K * coeff
    return 2.0 * (K + 4.0 / 3.0 * G) * coeff
