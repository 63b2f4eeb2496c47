"""The benchmark workloads at their full sizes and lengths.

Two questions the short parity tests leave open are answered here:

1. Does the plain-FP64 path keep the oracle's broken-bond set and fields at
   the full 11.52 M-particle plate (800 x 400 x 36, 1.355 G bonds)?  20 steps
   against the CPU oracle: identical bond bits, fields within 1e-12
   (norm-wise), totals within 1e-10.
2. Over the full run of each workload, does the mixed-precision path break
   the same bonds as the plain-FP64 path?  The two run side by side from the
   same start; every ``CHECK`` steps their bond bits are compared word for
   word on the device (cpd_bond_bits). Each test records the number of
   directed bonds whose state differs, the first step at which any differs
   and the per-field errors at the end, prints them, and appends them to the
   JSON file named by CPD_FULL_LENGTH_JSON when that is set.

Runs: the 1.2 M-particle plate (376 x 188 x 17) and the full plate, 2000
steps each; the 8 M-particle LPS box with 20 random notches, 1000 steps; the
4 M-sphere Hertz packing, 5000 steps (contact lists instead of bond bits).
On the full plate the crack path is sensitive to perturbations of the size
of the mixed path's state error; that run is compared with an FP64 control
whose velocities take noise of that size (test_full_plate_crack_path_sensitivity).
"""
import json
import os
import time

import numpy as np
import pytest

from cabanapd_b200 import problems as P

pytestmark = pytest.mark.gpu

FP64, MIXED = 1, 2
CHECK = 25


def _nrel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def _record(name, summary):
    print(f"\n[full length] {name}: {json.dumps(summary)}")
    path = os.environ.get("CPD_FULL_LENGTH_JSON")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps({"case": name, **summary}) + "\n")


class _DevArray:
    """__cuda_array_interface__ over a device pointer owned by a system."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None}


def _bits(sysm):
    import torch
    ptr, words, stride = sysm.bond_bits()
    return torch.as_tensor(_DevArray(ptr, (words, stride), "<i4"), device="cuda:0")


_POP = None


def _popcount(t):
    """Number of set bits of an int32 device tensor."""
    import torch
    global _POP
    if _POP is None:
        _POP = torch.tensor([bin(k).count("1") for k in range(256)], dtype=torch.int64,
                            device="cuda:0")
    total = 0
    flat = t.reshape(-1)
    for c in range(0, flat.numel(), 1 << 26):
        total += int(_POP[flat[c:c + (1 << 26)].contiguous().view(torch.uint8).long()].sum())
    return total


def _bond_diff(a, b):
    import torch
    d = torch.bitwise_xor(_bits(a), _bits(b))
    if int(torch.count_nonzero(d)) == 0:
        return 0
    return _popcount(d)


def _pair_run(prob, steps, bits=True, precision_b=MIXED, noise=0.0):
    """Runs prob on the FP64 path beside the same problem on precision_b,
    comparing bond bits every CHECK steps. noise > 0: every CHECK steps the
    second system's velocities are multiplied by (1 + noise N(0, 1)), a
    random perturbation of the size of the mixed path's state error."""
    import cabanapd_b200
    fp = cabanapd_b200.System(dict(prob["params"], precision=FP64))
    mx = cabanapd_b200.System(dict(prob["params"], precision=precision_b))
    P.setup(fp, prob)
    P.setup(mx, prob)
    rng = np.random.default_rng(7)
    first, worst, done = None, 0, 0
    diffs = []
    t0 = time.time()
    while done < steps:
        k = min(CHECK, steps - done)
        fp.step(k)
        mx.step(k)
        fp.synchronize()
        mx.synchronize()
        done += k
        if noise > 0.0:
            v = mx.get("v")
            mx.set_state(None, v * (1.0 + noise * rng.standard_normal(v.shape)))
        if bits:
            d = _bond_diff(fp, mx)
            diffs.append(d)
            worst = max(worst, d)
            if d and first is None:
                first = done
    out = {"steps": steps, "particles": int(fp.n), "bonds": int(fp.neighbor_stats()[1]),
           "check_every": CHECK, "wall_s": round(time.time() - t0, 1)}
    wf, df = fp.compute_energy()
    wm, dm = mx.compute_energy()
    if bits:
        intact = _popcount(_bits(fp))
        out.update({"broken_bonds_fp64": out["bonds"] - intact,
                    "differing_bonds_final": diffs[-1], "differing_bonds_max": worst,
                    "first_step_differing": first})
    for fld in ("u", "v", "f"):
        out[f"err_{fld}"] = _nrel(mx.get(fld), fp.get(fld))
    out["err_strain_energy"] = _rel(wm, wf)
    out["damage_fp64"], out["damage_mixed"] = df, dm
    return out, fp, mx


@pytest.mark.parametrize("case", ["plate_1p2m", "lps_box"])
def test_mixed_breaks_the_fp64_bonds_over_the_full_run(case):
    if case == "plate_1p2m":
        prob, steps = P.plate_impact(num_cells=(376, 188, 17)), 2000
    else:
        prob, steps = P.lps_random_notches(), 1000
    out, fp, mx = _pair_run(prob, steps)
    _record(case, out)
    assert out["broken_bonds_fp64"] > 0
    assert out["differing_bonds_max"] == 0
    assert out["err_u"] <= 1e-6


def test_full_plate_crack_path_sensitivity():
    """The full plate over 2000 steps: the mixed path beside the FP64 path,
    and, as the control, the FP64 path beside itself with its velocities
    multiplied by (1 + 1e-8 N(0, 1)) every 25 steps (noise of the size of
    the mixed path's state error, ~1e-8 relative in u). Once the crack runs
    far, a bond whose stretch lies within that error of s0 breaks a step
    earlier or later, and the crack front then differs locally. The mixed
    path must agree with the FP64 path's bonds for the first 1000 steps,
    and its differences must stay below 0.2% of the broken bonds."""
    prob = P.plate_impact(num_cells=(800, 400, 36))
    steps = 2000
    out, fp, mx = _pair_run(prob, steps)
    del fp, mx
    ctl, fp, fq = _pair_run(prob, steps, precision_b=FP64, noise=1e-8)
    del fp, fq
    out["control_fp64_velocity_noise_1e-8"] = {k: ctl[k] for k in (
        "differing_bonds_final", "differing_bonds_max", "first_step_differing", "err_u",
        "err_v", "err_f", "err_strain_energy", "damage_mixed")}
    _record("plate_full", out)
    assert out["broken_bonds_fp64"] > 0
    assert out["first_step_differing"] is None or out["first_step_differing"] >= 1000
    assert out["differing_bonds_max"] <= 2e-3 * out["broken_bonds_fp64"]


def test_mixed_hertz_packing_over_the_full_run():
    prob = P.dem_packing()
    out, fp, mx = _pair_run(prob, 5000, bits=False)
    out["contact_rebuilds"] = [int(fp.contact_rebuilds()), int(mx.contact_rebuilds())]
    out["contacts"] = [int(fp.neighbor_stats()[1]), int(mx.neighbor_stats()[1])]
    _record("dem_packing", out)
    assert out["contact_rebuilds"][0] == out["contact_rebuilds"][1]
    assert out["err_u"] <= 1e-6


def test_fp64_full_plate_matches_the_oracle(oracle):
    """The plain-FP64 path against the oracle on the full plate: identical
    bond bits, fields within 1e-12 norm-wise, totals within 1e-10."""
    import cabanapd_b200
    prob = P.plate_impact(num_cells=(800, 400, 36))
    g = cabanapd_b200.System(dict(prob["params"], precision=FP64))
    o = oracle.OracleSystem(prob["params"])
    P.setup(g, prob)
    P.setup(o, prob)
    out = {"particles": int(g.n), "bonds": int(g.neighbor_stats()[1]), "checks": []}
    assert g.neighbor_stats() == o.neighbor_stats()
    for steps in (10, 10):
        g.run(steps)
        o.run(steps)
        bg = _bits(g)[:, :g.n].cpu().numpy().view(np.uint32)
        bo = o.bond_bits()
        same = bool(np.array_equal(bg, bo))
        errs = {fld: _nrel(g.get(fld), o.get(fld)) for fld in ("u", "v", "f")}
        wg, dg = g.compute_energy()
        wo, do = o.compute_energy()
        out["checks"].append({"bits_identical": same, **{f"err_{k}": v for k, v in errs.items()},
                              "err_strain_energy": _rel(wg, wo), "err_damage": _rel(dg, do)})
        assert same
        assert all(v <= 1e-12 for v in errs.values()), errs
        assert _rel(wg, wo) <= 1e-10 and _rel(dg, do) <= 1e-10
    _record("plate_full_fp64_vs_oracle", out)
