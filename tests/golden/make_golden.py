"""Generates tests/golden/reference_expectations.json from the reference's
own test sources (read as text; the reference cannot be built here).

Run from the repository root, naming the CabanaPD source tree:
    python tests/golden/make_golden.py <path to the CabanaPD tree>
The tests read only the committed JSON, never the reference tree.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _read(root, rel):
    with open(os.path.join(root, rel)) as fh:
        return fh.read()


def main(root):
    out = {}
    kw = _read(root, "regression_test/tstKalthoffWinkler.hpp")
    m = re.search(r"EXPECT_NEAR\(\s*max_crack_y,\s*([0-9.eE+-]+),\s*([0-9.eE+-]+)\s*\)", kw)
    out["kalthoff_winkler"] = {
        "source": "regression_test/tstKalthoffWinkler.hpp:53",
        "max_crack_y": float(m.group(1)), "tolerance": float(m.group(2)),
        "input": json.loads(_read(root, "regression_test/inputs/kalthoff_winkler.json")),
    }
    hz = _read(root, "regression_test/tstHertz.hpp")
    m = re.search(r"EXPECT_NEAR\(\s*std::sqrt\(\s*ke_f\s*/\s*ke_i\s*\),\s*e,\s*([0-9.eE+-]+)\s*\)", hz)
    out["hertz"] = {
        "source": "regression_test/tstHertz.hpp:135",
        "tolerance": float(m.group(1)),
        "input": json.loads(_read(root, "regression_test/inputs/hertzian_contact.json")),
    }
    ew = _read(root, "regression_test/tstElasticWave.hpp")
    block = re.search(r"std::vector<double> coeff\{(.*?)\};", ew, re.S).group(1)
    coeffs = [float(c) for c in re.findall(r"[-+]?[0-9.]+e[-+][0-9]+", block)]
    rel = re.search(r"EXPECT_LT\(\s*rel_err,\s*([0-9.eE+-]+)\s*\)", ew)
    l2 = re.search(r"EXPECT_LT\(\s*std::sqrt\(\s*total_err\s*\),\s*([0-9.eE+-]+)\s*\)", ew)
    out["elastic_wave"] = {
        "source": "regression_test/tstElasticWave.hpp:54-96",
        "poly_coeff_descending": coeffs,
        "rel_tol": float(rel.group(1)), "l2_tol": float(l2.group(1)),
        "input": json.loads(_read(root, "regression_test/inputs/elastic_wave.json")),
    }
    tf = _read(root, "unit_test/tstForce.hpp")
    # test_neighbor cases: (m, dx numerator, dx denominator).
    cases = re.findall(r"m = (\d+);\s*(?:double )?dx = ([0-9.]+) / ([0-9.]+);", tf)
    out["neighbor_cases"] = {
        "source": "unit_test/tstForce.hpp:996-1015",
        "cases": [[int(a), float(b), float(c)] for a, b, c in cases[:2]],
    }
    with open(os.path.join(HERE, "reference_expectations.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "reference_expectations.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the CabanaPD tree>")
    main(sys.argv[1])
