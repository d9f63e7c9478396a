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


LID = json.load(open(os.path.join(HERE, "golden", "lid_cavity_profiles.json")))["cases"]


def test_lid_cavity_against_reference_runs(vlbm):
    """The reference's published Re = 1000 lid-driven cavity (256 x 256 x 1,
    192,000 steps, FP64; lidDrivenBounceBack.cu): ux on the vertical and uy on
    the horizontal centre line.  Those runs predate the reference's current
    half-way wall rule (its plates and duct data of the same period show a
    first-order wall offset); the difference from the current rule, which the
    reference build itself reproduces to FP64 round-off (test_ref_parity),
    halves from 256 to 512 nodes: 0.76 % and 0.39 % of the lid speed for ux,
    1.5 % and 0.74 % for uy.
    Bound: 1 % (ux) and 2 % (uy) of the lid speed on 256 x 256."""
    c = LID[0]
    n = c["nx"]
    cfg = vlbm.Config.default(nx=n, ny=n, nz=1, tau=c["tau"], ux_bc=[0, c["u_max"]])
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_LID_DRIVEN)
    sim.step(c["steps"])
    m = sim.macroscopics()
    sim.close()
    ux, uy = m["ux"][0].astype(np.float64), m["uy"][0].astype(np.float64)
    gx = np.array([v for _, v in c["ux_vertical"]])
    gy = np.array([v for _, v in c["uy_horizontal"]])
    # the centre lines of an even lattice: column / row NX/2 - 1 (the closer fit of the two middle ones)
    assert np.abs(ux[:, n // 2 - 1] - gx).max() <= 1e-2 * c["u_max"]
    assert np.abs(uy[n // 2 - 1, :] - gy).max() <= 2e-2 * c["u_max"]
