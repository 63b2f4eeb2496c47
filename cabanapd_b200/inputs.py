"""CabanaPD JSON input semantics (reference: src/CabanaPD_Input.hpp).

Input files hold ``{"key": {"value": ..., "unit": ...}}`` entries. The
constructor derives the same keys as the reference ``Inputs`` class
(CabanaPD_Input.hpp:30-128): low/high corners or system size, num_cells or
dx, horizon or m, timestep safety factor, num_steps (C++ ``int`` truncation
of final_time / timestep), output file names, and mass scaling.
"""
import json
import math

PI = 3.14159265358979323846


class Inputs:
    """Parsed CabanaPD input deck with the reference's derived keys."""

    def __init__(self, source, export_file=None):
        if isinstance(source, dict):
            self.inputs = json.loads(json.dumps(source))
            filename = "<dict>"
        else:
            filename = str(source)
            with open(filename) as fh:
                self.inputs = json.load(fh)
        inp = self.inputs
        self._setup_size()
        tf = float(inp["final_time"]["value"])
        dt = float(inp["timestep"]["value"])
        # CabanaPD_Input.hpp:43-61 mass scaling, applied once.
        if "mass_scaling_factor" in inp and "density_input" not in inp:
            ms = float(inp["mass_scaling_factor"]["value"])
            rho0 = float(inp["density"]["value"])
            inp["density_input"] = {"value": rho0, "unit": inp["density"].get("unit", "")}
            inp["density"]["value"] = rho0 * ms
            inp["timestep_input"] = {"value": dt, "unit": inp["timestep"].get("unit", "")}
            dt = dt * math.sqrt(ms)
            inp["timestep"]["value"] = dt
        if "horizon" in inp and "m" in inp:
            raise RuntimeError("Cannot input both horizon and m.")
        dx = float(inp["dx"]["value"][0])
        if "horizon" in inp:
            horizon = float(inp["horizon"]["value"])
            m = int(math.floor(horizon / dx))
            if horizon < dx:
                raise RuntimeError(
                    "Input horizon must be greater than or equal to dx to "
                    "result in any neighbour-particles")
            inp["m"] = {"value": m}
        elif "m" in inp:
            m = int(inp["m"]["value"])
            if m < 1:
                raise RuntimeError("Input m must be greater than or equal to 1.")
            inp["horizon"] = {"value": float(m) * dx + 0.01 * dx}
        if "timestep_safety_factor" not in inp:
            inp["timestep_safety_factor"] = {"value": 0.85}
        if "bulk_modulus" not in inp and "elastic_modulus" not in inp:
            raise RuntimeError("Must input either bulk_modulus or elastic_modulus.")
        # C++ int conversion truncates toward zero.
        inp["num_steps"] = {"value": int(tf / dt)}
        inp.setdefault("output_file", {"value": "cabanaPD.out"})
        inp.setdefault("error_file", {"value": "cabanaPD.err"})
        inp["input_file"] = {"value": filename}
        inp.setdefault("output_reference", {"value": True})
        if export_file is not None:
            with open(export_file, "w") as fh:
                json.dump(inp, fh)

    def _setup_size(self):
        """CabanaPD_Input.hpp:130-215 setupSize."""
        inp = self.inputs
        if "system_size" in inp:
            size = [float(s) for s in inp["system_size"]["value"]]
            if len(size) != 3:
                raise RuntimeError("CabanaPD requires 3d (system_size).")
            unit = inp["system_size"].get("unit", "")
            inp["low_corner"] = {"value": [-0.5 * s for s in size], "unit": unit}
            inp["high_corner"] = {"value": [0.5 * s for s in size], "unit": unit}
        elif "low_corner" in inp and "high_corner" in inp:
            lo = [float(v) for v in inp["low_corner"]["value"]]
            hi = [float(v) for v in inp["high_corner"]["value"]]
            if len(lo) != 3 or len(hi) != 3:
                raise RuntimeError("CabanaPD requires 3d (low_corner/high_corner).")
            inp["system_size"] = {"value": [h - l for l, h in zip(lo, hi)],
                                  "unit": inp["low_corner"].get("unit", "")}
        else:
            raise RuntimeError("Must input either system_size or both low_corner "
                               "and high_corner.")
        size = [float(s) for s in inp["system_size"]["value"]]
        if "dx" in inp:
            dxv = [float(d) for d in inp["dx"]["value"]]
            if len(dxv) != 3:
                raise RuntimeError("CabanaPD requires 3d (dx).")
            inp["num_cells"] = {"value": [int(s / d) for s, d in zip(size, dxv)]}
        elif "num_cells" in inp:
            nc = [int(v) for v in inp["num_cells"]["value"]]
            if len(nc) != 3:
                raise RuntimeError("CabanaPD requires 3d (num_cells).")
            inp["dx"] = {"value": [s / float(n) for s, n in zip(size, nc)],
                         "unit": inp["system_size"].get("unit", "")}
        else:
            raise RuntimeError("Must input either num_cells or dx.")

    def __getitem__(self, key):
        return self.inputs[key]["value"]

    def __contains__(self, key):
        return key in self.inputs

    def contains(self, key):
        return key in self.inputs

    def units(self, key):
        return self.inputs[key].get("unit", "")

    def get_vector(self, key):
        v = self.inputs[key]["value"]
        return [float(a) for a in v] if isinstance(v, list) else [float(v)]

    def compute_critical_timestep(self):
        """CabanaPD_Input.hpp:217-301 (mechanics) + :385-399.

        Returns dt_crit (unscaled) and stores safety * dt_crit as
        ``critical_timestep_mechanics`` the way the reference does.
        """
        dxv = [float(d) for d in self.inputs["dx"]["value"]]
        if "bulk_modulus" in self.inputs:
            K = self.get_vector("bulk_modulus")
        else:
            E = self.get_vector("elastic_modulus")
            denom = 3.0 * (1.0 - 2.0 * 0.25)
            K = [e / denom for e in E]
        rho = self.get_vector("density")
        ratios = [r / k for r, k in zip(rho, K)]
        imin = ratios.index(min(ratios))
        dt_crit = critical_timestep(dxv[0], dxv[1], dxv[2], int(self["m"]),
                                    float(self["horizon"]), K[imin], rho[imin])
        safety = float(self["timestep_safety_factor"])
        self.inputs["critical_timestep_mechanics"] = {"value": safety * dt_crit}
        return dt_crit


def critical_timestep(dx, dy, dz, m, horizon, K, rho):
    """Silling & Askari stable step over the lattice neighbourhood of a bulk
    point (CabanaPD_Input.hpp:217-301), same operation order as the
    reference so the double result is identical."""
    v_p = dx * dy * dz
    c = 18.0 * K / (PI * horizon * horizon * horizon * horizon)
    total = 0.0
    for i in range(-(m + 1), m + 2):
        xi_1 = i * dx
        for j in range(-(m + 1), m + 2):
            xi_2 = j * dy
            for k in range(-(m + 1), m + 2):
                xi_3 = k * dz
                r2 = xi_1 * xi_1 + xi_2 * xi_2 + xi_3 * xi_3
                if r2 < horizon * horizon + 1e-10 and r2 > 0:
                    xi = math.sqrt(r2)
                    total += v_p * c / xi
    return math.sqrt(2.0 * rho / total)
