"""Writes lid_cavity_profiles.json from the reference's lid-driven cavity runs.

The reference repository ships the centre-line velocity profiles of its D3Q19
regularized lid-driven cavity, Re = 1000 (doc/Simulations/Analysis/
Regularized/D3Q19/Lid Driven HWBB/data: 100u{x,y}192000.csv on 256 x 256 and
101u{x,y}768000.csv on 512 x 512, NZ = 1, run info in *_info.txt; FP64):
ux along the vertical line and uy along the horizontal line through the
cavity centre.  This script copies them into a small fixture so the tests do
not read the reference at run time.  Run from the repository root:

    python tests/golden/make_lid_golden.py /path/to/reference
"""
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from make_duct_golden import read_csv, read_info  # noqa: E402


def main(ref):
    d = os.path.join(ref, "doc", "Simulations", "Analysis", "Regularized", "D3Q19", "Lid Driven HWBB", "data")
    cases = []
    for cid, steps in (("100", 192000), ("101", 768000)):
        info = read_info(os.path.join(d, cid + "_info.txt"))
        case = {"id": cid, "nx": int(info["NX"]), "ny": int(info["NY"]), "nz": int(info["NZ"]),
                "tau": float(info["Tau"]), "u_max": float(info["Umax"]), "steps": int(info["Nsteps"]),
                "ux_vertical": read_csv(os.path.join(d, f"{cid}ux{steps}.csv")),
                "uy_horizontal": read_csv(os.path.join(d, f"{cid}uy{steps}.csv"))}
        assert case["steps"] == steps
        cases.append(case)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lid_cavity_profiles.json")
    json.dump({"source": "doc/Simulations/Analysis/Regularized/D3Q19/Lid Driven HWBB/data", "cases": cases},
              open(out, "w"), indent=1)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("VLBM_REFERENCE_ROOT"):
        sys.exit("usage: python " + sys.argv[0] + " /path/to/reference  (or set VLBM_REFERENCE_ROOT)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["VLBM_REFERENCE_ROOT"])
