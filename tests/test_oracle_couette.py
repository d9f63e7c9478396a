"""The oracle's velocity Zou-He pinned to the reference's own Couette runs
(tests/golden/couette_zouhe_profiles.json, made by
tests/golden/make_couette_golden.py from the reference's published data).

Those runs (D3Q19 regularized, FP64, NX = NY = NZ, couetteZouHe.cu) move the
plate at y = 0 at uz = -Umax/2 and the plate at y = NY - 1 at +Umax/2; the
profiles are printed with seven significant digits, so the bound is 1e-6 of
the plate speed."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = json.load(open(os.path.join(HERE, "golden", "couette_zouhe_profiles.json")))["cases"]


def couette_config(mod, c):
    u = c["u_max"] / 2.0
    return mod.Config.default(nx=c["nx"], ny=c["ny"], nz=c["nz"], vel_set=19, tau=c["tau"], uz_bc=[0, u, -u])


@pytest.mark.parametrize("case", CASES, ids=[c["id"] for c in CASES])
def test_oracle_couette_zouhe_matches_reference_runs(oracle, case):
    o = oracle.Oracle(couette_config(oracle, case),
                      oracle.reference_builder_map("plates_y_zouhe", case["nx"], case["ny"], case["nz"]))
    o.step(case["steps"])
    uz = o.macroscopics()["uz"]
    ref = np.array([v for _, v in case["uz_profile"]])
    assert np.abs(uz - ref[None, :, None]).max() <= 1e-6 * case["u_max"]
