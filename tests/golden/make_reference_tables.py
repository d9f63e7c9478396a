"""Generate tests/golden/reference_bc_tables.json from the reference sources.

Reads (as text) the boundary-condition schemes of CERNN/VISCOPLASTIC-LBM:
  src/CUDA/boundaryConditionsSchemes/bounceBack.cu       (half-way bounce-back)
  src/CUDA/boundaryConditionsSchemes/freeSlip.cu         (free slip)
  src/CUDA/boundaryConditionsSchemes/D3Q19_VelBounceBack.cu (moving wall)
and the velocity sets src/CUDA/velocitySets/D3Q19.h, D3Q27.h, and records, per
scheme/direction and velocity set, which population is overwritten from which.
The fixture is committed; this script only runs where the reference is mounted.

Usage: python tests/golden/make_reference_tables.py /path/to/reference
"""
import json
import os
import re
import sys

DIRS = ["N", "S", "W", "E", "F", "B", "NW", "NE", "NF", "NB", "SW", "SE", "SF", "SB",
        "WF", "WB", "EF", "EB", "NWF", "NWB", "NEF", "NEB", "SWF", "SWB", "SEF", "SEB"]


def split_functions(text, prefix):
    out = {}
    for m in re.finditer(r"void\s+" + prefix + r"(\w+)\s*\(", text):
        name = m.group(1)
        start = text.index("{", m.end())
        depth, i = 0, start
        while True:
            if text[i] == "{":
                depth += 1
            elif text[i] == "}":
                depth -= 1
                if depth == 0:
                    break
            i += 1
        out[name] = text[start + 1:i]
    return out


def q_sections(body):
    """Yield (line, only_q27) for each statement line of a function body."""
    only27 = False
    for line in body.splitlines():
        s = line.strip()
        if s.startswith("#ifdef D3Q27"):
            only27 = True
            continue
        if s.startswith("#endif"):
            only27 = False
            continue
        yield s, only27


def parse_bounce_back(path):
    funcs = split_functions(open(path).read(), "gpuBCBounceBack")
    pat = re.compile(r"fPostStream\[idxPop\(x, y, z, (\d+)\)\]\s*=\s*fPostCol\[idxPop\(x, y, z, (\d+)\)\]")
    tab = {}
    for name, body in funcs.items():
        q19, q27 = [], []
        for s, only27 in q_sections(body):
            m = pat.search(s)
            if not m:
                continue
            pair = [int(m.group(1)), int(m.group(2))]
            q27.append(pair)
            if not only27:
                q19.append(pair)
        tab[name] = {"19": q19, "27": q27}
    return tab


def parse_free_slip(path):
    funcs = split_functions(open(path).read(), "gpuBCFreeSlip")
    pat = re.compile(r"fPostStream\[idxPop\(x, y, z, (\d+)\)\]\s*=\s*fPostCol\[idxPop\((\w+), (\w+), (\w+), (\d+)\)\]")
    off = {"x": 0, "y": 0, "z": 0, "xp1": 1, "xm1": -1, "yp1": 1, "ym1": -1, "zp1": 1, "zm1": -1}
    tab = {}
    for name, body in funcs.items():
        q19, q27 = [], []
        for s, only27 in q_sections(body):
            m = pat.search(s)
            if not m:
                continue
            row = [int(m.group(1)), int(m.group(5)), [off[m.group(2)], off[m.group(3)], off[m.group(4)]]]
            q27.append(row)
            if not only27:
                q19.append(row)
        tab[name] = {"19": q19, "27": q27}
    return tab


def parse_vel_bb(path):
    funcs = split_functions(open(path).read(), "gpuBCVelBounceBack")
    pat = re.compile(r"f\[idxPop\(x, y, z, (\d+)\)\]\s*=\s*f\[idxPop\(x, y, z, (\d+)\)\]\s*-\s*6\s*\*\s*rho_w\*W(\d)\*\(([^;]*)\);")
    tab = {}
    for name, body in funcs.items():
        rows = []
        for s, _ in q_sections(body):
            m = pat.search(s)
            if m:
                rows.append([int(m.group(1)), int(m.group(2)), int(m.group(3)), m.group(4).replace(" ", "")])
        tab[name] = rows
    return tab


def parse_velocity_set(path):
    text = open(path).read()
    out = {}
    for comp in ("cx", "cy", "cz"):
        m = re.search(r"const char " + comp + r"\[Q\]\s*=\s*\{([^}]*)\}", text)
        out[comp] = [int(v) for v in m.group(1).split(",")]
    return out


def main(ref):
    cuda = os.path.join(ref, "src", "CUDA")
    sch = os.path.join(cuda, "boundaryConditionsSchemes")
    data = {
        "source": "CERNN/VISCOPLASTIC-LBM src/CUDA (parsed as text)",
        "directions": DIRS,
        "bounce_back": parse_bounce_back(os.path.join(sch, "bounceBack.cu")),
        "free_slip": parse_free_slip(os.path.join(sch, "freeSlip.cu")),
        "vel_bounce_back_d3q19": parse_vel_bb(os.path.join(sch, "D3Q19_VelBounceBack.cu")),
        "velocity_sets": {
            "19": parse_velocity_set(os.path.join(cuda, "velocitySets", "D3Q19.h")),
            "27": parse_velocity_set(os.path.join(cuda, "velocitySets", "D3Q27.h")),
        },
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_bc_tables.json")
    with open(dst, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    print("wrote", dst, "bb dirs:", len(data["bounce_back"]), "free-slip dirs:", len(data["free_slip"]))


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("VLBM_REFERENCE_ROOT"):
        sys.exit("usage: python " + sys.argv[0] + " /path/to/reference  (or set VLBM_REFERENCE_ROOT)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["VLBM_REFERENCE_ROOT"])
