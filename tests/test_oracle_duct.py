"""The oracle's interpolated bounce-back pinned to the reference's own
circular-duct results (tests/golden/duct_interp_profiles.json, made by
tests/golden/make_duct_golden.py from the reference's published runs).

Those runs (D3Q19 regularized, FP64, NZ = 1, body force along the duct axis)
used a cylinder of radius NY/2 - 0.5 about the lattice centre; the profiles are
printed with seven significant digits, so the bound is 1e-6 of the peak
velocity.  Both the vertical line through the axis and the diagonal are
checked, which exercises the horizontal, vertical and diagonal wall-distance
rules and both branches (q above and below 1/2)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = json.load(open(os.path.join(HERE, "golden", "duct_interp_profiles.json")))["cases"]


def run_case(vlbm, oracle, c):
    R = c["ny"] / 2.0 - 0.5
    cfg = vlbm.Config.default(nx=c["nx"], ny=c["ny"], nz=c["nz"], vel_set=19, tau=c["tau"], fz=c["fz"],
                              duct_outer_radius=R)
    m = oracle.reference_builder_map("circular_duct", c["nx"], c["ny"], c["nz"], outer_radius=R)
    o = oracle.Oracle(cfg, m)
    o.step(c["steps"])
    return o.macroscopics()["uz"][0], m.reshape(c["nz"], c["ny"], c["nx"])[0]


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_oracle_circular_duct_matches_reference_runs(vlbm, oracle, case):
    uz, m = run_case(vlbm, oracle, case)
    peak = max(v for _, v in case["uz_north_south"])
    xc = case["nx"] // 2
    ns = np.array([v for _, v in case["uz_north_south"]])
    assert np.abs(uz[:, xc] - ns).max() <= 1e-6 * peak
    used_diag = [k for k in range(case["nx"]) if (int(m[k, k]) >> 21) & 1]
    diag = np.array([v for _, v in case["uz_sw_ne"]])
    assert len(used_diag) == len(diag)
    assert np.abs(np.array([uz[k, k] for k in used_diag]) - diag).max() <= 1e-6 * peak
    # the wall rule is the interpolated one: nodes next to the cylinder carry it
    interp = ((m >> 18) & 7) == 6
    assert interp.sum() > 0


ANNULAR = json.load(open(os.path.join(HERE, "golden", "duct_interp_profiles.json")))["annular_cases"]


def annular_radii(ny):
    """The runs' cylinders: outer radius NY/2 - 0.5 (as the circular-duct runs)
    and the inner radius a quarter of it (var.h:154, INNER_RADIUS = OUTER_RADIUS/4)."""
    r_out = ny / 2.0 - 0.5
    return r_out, r_out / 4.0


@pytest.mark.parametrize("case", ANNULAR, ids=[c["id"] for c in ANNULAR])
def test_oracle_annular_duct_matches_reference_runs(vlbm, oracle, case):
    ro, ri = annular_radii(case["ny"])
    cfg = vlbm.Config.default(nx=case["nx"], ny=case["ny"], nz=case["nz"], vel_set=19, tau=case["tau"],
                              fz=case["fz"], duct_outer_radius=ro, duct_inner_radius=ri)
    m = oracle.reference_builder_map("annular_duct", case["nx"], case["ny"], case["nz"], outer_radius=ro,
                                     inner_radius=ri)
    o = oracle.Oracle(cfg, m)
    o.step(case["steps"])
    uz = o.macroscopics()["uz"][0]
    ns = np.array([v for _, v in case["uz_north_south"]])
    assert np.abs(uz[:, case["nx"] // 2] - ns).max() <= 1e-6 * ns.max()
    assert (ns == 0).sum() >= 3        # the line crosses the inner cylinder
