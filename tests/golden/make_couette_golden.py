"""Writes couette_zouhe_profiles.json from the reference's Couette Zou-He runs.

The reference repository ships the velocity profiles of its D3Q19 regularized
Couette flow between velocity Zou-He plates (doc/Simulations/Analysis/
Regularized/D3Q19/Couette Zou He/data: 200uz300.csv and 201uz1200.csv, run
info in *_info.txt; FP64, the plates at y = 0 and y = NY - 1 moving at
uz = -Umax/2 and +Umax/2).  This script copies them into a small fixture so
the tests do not read the reference at run time.  Run from the repository root:

    python tests/golden/make_couette_golden.py /path/to/reference
"""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_duct_golden import read_csv, read_info  # noqa: E402


def main(ref):
    d = os.path.join(ref, "doc", "Simulations", "Analysis", "Regularized", "D3Q19", "Couette Zou He", "data")
    cases = []
    for cid, steps in (("200", 300), ("201", 1200)):
        info = read_info(os.path.join(d, cid + "_info.txt"))
        case = {"id": cid, "nx": int(info["NX"]), "ny": int(info["NY"]), "nz": int(info["NZ"]),
                "tau": float(info["Tau"]), "u_max": float(info["Umax"]), "steps": int(info["Nsteps"]),
                "uz_profile": read_csv(os.path.join(d, f"{cid}uz{steps}.csv"))}
        assert case["steps"] == steps
        cases.append(case)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "couette_zouhe_profiles.json")
    json.dump({"source": "doc/Simulations/Analysis/Regularized/D3Q19/Couette Zou He/data", "cases": cases},
              open(out, "w"), indent=1)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("VLBM_REFERENCE_ROOT"):
        sys.exit("usage: python " + sys.argv[0] + " /path/to/reference  (or set VLBM_REFERENCE_ROOT)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["VLBM_REFERENCE_ROOT"])
