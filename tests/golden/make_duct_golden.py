"""Writes duct_interp_profiles.json from the reference's circular- and annular-duct runs.

The reference repository ships velocity profiles of its interpolated
bounce-back circular duct (doc/Simulations/Analysis/Regularized/D3Q19/
circularDuctInterp/data: 200*.csv and 201*.csv, run info in *_info.txt) and
annular duct (annularDuctInterp/data: 00{0,1,2}uzN-S*.csv).  This
script copies the numbers it needs into a small fixture so the tests do not
read the reference at run time.  Run from the repository root:

    python tests/golden/make_duct_golden.py /path/to/reference
"""
import json
import os
import sys


def read_csv(path):
    out = []
    for line in open(path):
        line = line.strip()
        if line:
            k, v = line.split(",")
            out.append([int(k), float(v)])
    return out


def read_info(path):
    info = {}
    for line in open(path):
        if ":" in line:
            k, v = line.split(":", 1)
            info[k.strip()] = v.strip()
    return info


def main(ref):
    d = os.path.join(ref, "doc", "Simulations", "Analysis", "Regularized", "D3Q19", "circularDuctInterp", "data")
    cases = []
    for cid, steps in (("200", 1100), ("201", 4400)):
        info = read_info(os.path.join(d, cid + "_info.txt"))
        case = {"id": cid, "nx": int(info["NX"]), "ny": int(info["NY"]), "nz": int(info["NZ"]),
                "tau": float(info["Tau"]), "fz": float(info["FZ"]), "steps": int(info["Nsteps"]),
                "uz_north_south": read_csv(os.path.join(d, f"{cid}uzN-S{steps}.csv")),
                "uz_sw_ne": read_csv(os.path.join(d, f"{cid}uzSW-NE{steps}.csv"))}
        assert case["steps"] == steps
        cases.append(case)
    # annular duct (annularDuctInterpBounceBack.cu): profile along the vertical line
    # through the axis, which crosses both cylinders
    da = os.path.join(ref, "doc", "Simulations", "Analysis", "Regularized", "D3Q19", "annularDuctInterp", "data")
    annular = []
    for cid, steps in (("000", 900), ("001", 3600), ("002", 14400)):
        info = read_info(os.path.join(da, cid + "_info.txt"))
        case = {"id": "annular_" + cid, "nx": int(info["NX"]), "ny": int(info["NY"]), "nz": int(info["NZ"]),
                "tau": float(info["Tau"]), "fz": float(info["FZ"]), "steps": int(info["Nsteps"]),
                "uz_north_south": read_csv(os.path.join(da, f"{cid}uzN-S{steps}.csv"))}
        assert case["steps"] == steps
        annular.append(case)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "duct_interp_profiles.json")
    json.dump({"source": "doc/Simulations/Analysis/Regularized/D3Q19/circularDuctInterp/data",
               "cases": cases,
               "annular_source": "doc/Simulations/Analysis/Regularized/D3Q19/annularDuctInterp/data",
               "annular_cases": annular}, open(out, "w"), indent=1)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("VLBM_REFERENCE_ROOT"):
        sys.exit("usage: python " + sys.argv[0] + " /path/to/reference  (or set VLBM_REFERENCE_ROOT)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["VLBM_REFERENCE_ROOT"])
