"""FP64 global mass/momentum reduction (vlbm_moments_sum) against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("q,builder,size,steps", [
    (19, 1, (33, 17, 9), 40),      # node count not a multiple of the chunk
    (27, 3, (16, 16, 20), 25),
    (19, 6, (64, 64, 8), 11),      # several reduction blocks, odd parity
])
def test_moments_sum_matches_oracle(vlbm, oracle, q, builder, size, steps):
    nx, ny, nz = size
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=q, tau=0.8, fx=1e-4, fz=-3e-5,
                              ux_bc=[0, 0.05])
    m = vlbm.build_node_map(builder, nx, ny, nz)
    sim = vlbm.Simulation(cfg, node_map=m)
    sim.step(steps)
    got = sim.moments_sum()
    o = oracle.Oracle(cfg, m)
    o.step(steps)
    mo = o.macroscopics()
    ref = np.array([mo["rho"].sum(), (mo["rho"] * mo["ux"]).sum(), (mo["rho"] * mo["uy"]).sum(),
                    (mo["rho"] * mo["uz"]).sum()])
    n = nx * ny * nz
    assert abs(got[0] - ref[0]) <= 5e-6 * n
    assert np.all(np.abs(got[1:] - ref[1:]) <= 2e-6 * n)
    # repeated calls are bit-identical (fixed partition and order)
    assert np.array_equal(sim.moments_sum(), got)
