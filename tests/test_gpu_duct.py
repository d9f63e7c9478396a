"""Circular and annular ducts: interpolated bounce-back and unused nodes on the
GPU against the FP64 oracle and the reference's own duct runs.

Tolerances as the plane-wall parity cases (FP32 vs FP64, <= 100 steps):
populations max |df| <= 5e-6 and velocity max |du| <= 2e-6 + 2e-4 max|u|, over
the fluid nodes.  Nodes outside the cylinders are not updated; their
macroscopics read as the initial state (rho0, zero velocity), as the
reference's never-written macroscopic arrays do."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
POP_TOL = 5e-6
U_ABS_TOL = 2e-6

# (name, builder, (nx, ny, nz), steps, config)
CASES = [
    ("circular_reg_q19", 9, (20, 20, 6), 80, dict(vel_set=19, tau=0.8, fz=2e-4)),
    ("circular_bgk_q27", 9, (18, 21, 5), 60, dict(vel_set=27, collision=1, tau=0.9, fz=2e-4, fx=5e-5)),
    ("circular_bingham_q19_rotating", 9, (22, 22, 8), 70,
     dict(vel_set=19, rheology=1, eta_p=0.1, yield_stress=1e-6, fz=1e-4, duct_outer_rotation=0.004,
          duct_outer_velocity=0.01)),
    ("annular_reg_q19_inner_rotation", 10, (26, 26, 4), 80,
     dict(vel_set=19, tau=0.7, fz=1e-4, duct_inner_rotation=0.01, duct_inner_velocity=-0.02)),
    ("annular_powerlaw_q27", 10, (24, 24, 4), 50,
     dict(vel_set=27, rheology=2, n_index=0.8, k_consistency=0.05, fz=2e-4, duct_outer_velocity=0.01)),
]


def fluid_mask(node_map, shape):
    return (((node_map >> 21) & 1) == 1).reshape(shape)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_duct_matches_oracle(vlbm, oracle, case):
    name, builder, (nx, ny, nz), steps, kw = case
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, **kw)
    sim = vlbm.Simulation(cfg, builder=builder)     # tables straight from the builder
    sim.step(steps)
    sim.sync()
    m = oracle.reference_builder_map(oracle.BUILDER_NAMES[builder], nx, ny, nz)
    np.testing.assert_array_equal(vlbm.build_node_map(builder, nx, ny, nz), m)
    o = oracle.Oracle(cfg, m)
    o.step(steps)
    fluid = fluid_mask(m, (nz, ny, nx))
    assert 0 < fluid.sum() < fluid.size
    fg = sim.populations().astype(np.float64)[:, fluid]
    fo = o.populations()[:, fluid]
    assert np.max(np.abs(fg - fo)) <= POP_TOL, (name, np.max(np.abs(fg - fo)))
    mg, mo = sim.macroscopics(), o.macroscopics()
    ug = np.stack([mg["ux"], mg["uy"], mg["uz"]]).astype(np.float64)
    uo = np.stack([mo["ux"], mo["uy"], mo["uz"]])
    assert np.abs(uo).max() > 1e-3
    assert np.max(np.abs(ug - uo)) <= U_ABS_TOL + 2e-4 * np.abs(uo).max(), (name, np.max(np.abs(ug - uo)))
    assert np.all(mg["rho"][~fluid] == np.float32(cfg.rho0)) and np.all(ug[:, ~fluid] == 0)
    # the same run from a node map gives the same state bit for bit
    sim2 = vlbm.Simulation(cfg, node_map=m)
    sim2.step(steps)
    np.testing.assert_array_equal(sim2.populations()[:, fluid], sim.populations()[:, fluid])


def test_circular_duct_matches_reference_runs(vlbm):
    """The reference's published D3Q19 circular-duct profiles (radius NY/2 - 0.5),
    run on the GPU in FP32: within 3e-5 of the peak velocity (the FP64 oracle
    reproduces them to 1e-6)."""
    cases = json.load(open(os.path.join(HERE, "golden", "duct_interp_profiles.json")))["cases"]
    for c in cases:
        cfg = vlbm.Config.default(nx=c["nx"], ny=c["ny"], nz=c["nz"], vel_set=19, tau=c["tau"], fz=c["fz"],
                                  duct_outer_radius=c["ny"] / 2.0 - 0.5)
        sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CIRCULAR_DUCT)
        sim.step(c["steps"])
        uz = sim.macroscopics()["uz"][0].astype(np.float64)
        ns = np.array([v for _, v in c["uz_north_south"]])
        peak = ns.max()
        assert np.abs(uz[:, c["nx"] // 2] - ns).max() <= 3e-5 * peak, c["id"]


@pytest.mark.parametrize("storage", [1, 2])
def test_duct_half_storage_close_to_fp64(vlbm, oracle, storage):
    """FP16/BF16 deviation storage on the circular duct (z-paired layout)."""
    nx, ny, nz, steps = 24, 24, 8, 400
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=19, tau=0.8, fz=5e-5, storage=storage)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CIRCULAR_DUCT)
    sim.step(steps)
    m = oracle.reference_builder_map("circular_duct", nx, ny, nz)
    o = oracle.Oracle(cfg, m)
    o.step(steps)
    fluid = fluid_mask(m, (nz, ny, nx))
    ug = sim.macroscopics()["uz"].astype(np.float64)[fluid]
    uo = o.macroscopics()["uz"][fluid]
    rel = np.linalg.norm(ug - uo) / np.linalg.norm(uo)
    assert rel < (2e-3 if storage == 1 else 2e-2), rel


def test_hagen_poiseuille(vlbm):
    """Developed flow in the circular duct against u(r) = F (R^2 - r^2) / (4 nu)."""
    n, tau, g = 34, 0.8, 2e-6
    cfg = vlbm.Config.default(nx=n, ny=n, nz=2, vel_set=19, tau=tau, fz=g)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CIRCULAR_DUCT)
    sim.step(6000)
    uz = sim.macroscopics()["uz"][0].astype(np.float64)
    R = n / 2.0 - 1.5
    nu = (tau - 0.5) / 3
    c = (n - 1) / 2.0
    yy, xx = np.mgrid[0:n, 0:n]
    r = np.hypot(xx - c, yy - c)
    inside = r < R - 1.5
    ana = g * (R * R - r * r) / (4 * nu)
    err = np.linalg.norm((uz - ana)[inside]) / np.linalg.norm(ana[inside])
    assert err < 5e-3, err   # the FP64 oracle gives 1.8e-3 on this lattice


def test_annular_duct_matches_reference_runs(vlbm):
    """The reference's published D3Q19 annular-duct profiles (outer radius
    NY/2 - 0.5, inner a quarter of it), run on the GPU in FP32: within 3e-5 of
    the peak velocity."""
    cases = json.load(open(os.path.join(HERE, "golden", "duct_interp_profiles.json")))["annular_cases"]
    for c in cases:
        ro = c["ny"] / 2.0 - 0.5
        cfg = vlbm.Config.default(nx=c["nx"], ny=c["ny"], nz=c["nz"], vel_set=19, tau=c["tau"], fz=c["fz"],
                                  duct_outer_radius=ro, duct_inner_radius=ro / 4.0)
        sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_ANNULAR_DUCT)
        sim.step(c["steps"])
        uz = sim.macroscopics()["uz"][0].astype(np.float64)
        sim.close()
        ns = np.array([v for _, v in c["uz_north_south"]])
        assert np.abs(uz[:, c["nx"] // 2] - ns).max() <= 3e-5 * ns.max(), c["id"]
