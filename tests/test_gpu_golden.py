"""The fused step on the GPU against the reference's published runs
(reference-held golden data, committed as fixtures under tests/golden/)."""
import json
import os

import numpy as np
import pytest

from test_oracle_couette import couette_config

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
COUETTE = json.load(open(os.path.join(HERE, "golden", "couette_zouhe_profiles.json")))["cases"]


@pytest.mark.parametrize("storage,tol", [(0, 1e-5), (1, 1e-3)])
@pytest.mark.parametrize("case", COUETTE, ids=[c["id"] for c in COUETTE])
def test_couette_zouhe_matches_reference_runs(vlbm, case, storage, tol):
    """Velocity Zou-He plates (couetteZouHe.cu): FP32 within 1e-5, FP16
    deviation storage within 1e-3 of the plate speed."""
    cfg = couette_config(vlbm, case)
    cfg.storage = storage
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y_ZOUHE)
    sim.step(case["steps"])
    uz = sim.macroscopics()["uz"].astype(np.float64)
    sim.close()
    ref = np.array([v for _, v in case["uz_profile"]])
    assert np.abs(uz - ref[None, :, None]).max() <= tol * case["u_max"]
