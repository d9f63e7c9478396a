"""Report-step data treatment on the device (treatData.cpp:25-89) against the
FP64 restatement in the oracle, on the same device macroscopics.

Both sides sum the same FP32 fields in FP64 (different order): relative
tolerance 1e-12 on residual, mean density and the per-plane mean uz."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def fields(sim):
    m = sim.macroscopics()
    return m["rho"], m["ux"], m["uy"], m["uz"]


def close(a, b, tol=TOL):
    return abs(a - b) <= tol * max(abs(b), 1e-300)


@pytest.mark.parametrize("spheres", [False, True], ids=["plain", "with_sphere"])
def test_treat_data_matches_restatement(vlbm, oracle, spheres):
    cfg = vlbm.Config.default(nx=32, ny=24, nz=16, rheology=1, eta_p=0.1, yield_stress=1e-6, fx=2e-5)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
    if spheres:
        sim.add_spheres(vlbm.IbmConfig.default(max_iterations=2, gy=-1e-5),
                        [vlbm.Sphere(diameter=6, cx=16.0, cy=12.0, cz=8.0, density=1.5, movable=1)])
    sim.step(40)
    t1 = sim.treat_data()
    f1 = fields(sim)
    r1 = oracle.treat_data(*f1)
    assert t1["residual"] == 1.0 and r1["residual"] == 1.0   # first report: u_prev = 0
    assert close(t1["avg_rho"], r1["avg_rho"])
    np.testing.assert_allclose(t1["avg_uz_plane_xz"], r1["avg_uz_plane_xz"], rtol=TOL, atol=1e-300)
    assert t1["step"] == 40
    sim.step(60)
    t2 = sim.treat_data(resid_max=1e-9)
    f2 = fields(sim)
    r2 = oracle.treat_data(*f2, prev=f1[1:], resid_max=1e-9)
    assert 0 < r2["residual"] < 1
    assert close(t2["residual"], r2["residual"])
    assert close(t2["avg_rho"], r2["avg_rho"])
    np.testing.assert_allclose(t2["avg_uz_plane_xz"], r2["avg_uz_plane_xz"], rtol=1e-10, atol=1e-18)
    assert t2["stop"] == r2["stop"] == False
    t3 = sim.treat_data(resid_max=1.0)       # nothing moved since the last report
    assert t3["residual"] == 0.0 and t3["stop"]


def test_treat_data_reproducible_and_reset_by_init(vlbm):
    cfg = vlbm.Config.default(nx=24, ny=20, nz=12, tau=0.8, fx=1e-4)
    out = []
    for _ in range(2):
        sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_DUCT_YZ)
        sim.step(10)
        sim.treat_data()
        sim.step(15)
        out.append(sim.treat_data())
        sim.init_equilibrium(1.0, 0, 0, 0)
        sim.step(5)
        assert sim.treat_data()["residual"] == 1.0
        sim.close()
    assert out[0]["residual"] == out[1]["residual"] and out[0]["avg_rho"] == out[1]["avg_rho"]
    np.testing.assert_array_equal(out[0]["avg_uz_plane_xz"], out[1]["avg_uz_plane_xz"])


def test_poiseuille_run_stops_on_residual(vlbm):
    """The reference's report loop: treat every 500 steps, stop when the
    residual between reports falls below RESID_MAX."""
    cfg = vlbm.Config.default(nx=8, ny=12, nz=4, tau=0.9, fx=1e-5)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
    stopped_at = None
    for k in range(1, 41):
        sim.step(500)
        t = sim.treat_data(resid_max=1e-5)
        if t["stop"]:
            stopped_at = t["step"]
            break
    assert stopped_at is not None and stopped_at < 20000
    ny, nu = 12, (0.9 - 0.5) / 3
    y = np.arange(ny)
    ana = 1e-5 / (2 * nu) * (y + 0.5) * (ny - 0.5 - y)
    ux = sim.macroscopics()["ux"].mean(axis=(0, 2))
    assert np.linalg.norm(ux - ana) / np.linalg.norm(ana) < 2e-3
