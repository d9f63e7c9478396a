"""Immersed-boundary step for spheres on the GPU against the FP64 oracle.

Tolerances (FP32 Eulerian fields and interpolation vs FP64, <= 60 steps):
  sphere position   |dx| <= 2e-6 + 1e-3 * |x - x0|  (lattice units; sphere radius >= 3)
  sphere velocity   |dv| <= 2e-3 * max|v| + 1e-9 (and the same for the rotation)
  fluid velocity    relative L2 <= 5e-3, max abs <= 5e-6 (settling flows are
                    ~1e-4, so FP32 rounding of rho*u weighs in)
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_case(vlbm, oracle, q, builder, size, spheres, ibm_kw, cfg_kw):
    nx, ny, nz = size
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=q, **cfg_kw)
    ib = vlbm.IbmConfig.default(**ibm_kw)
    m = vlbm.build_node_map(builder, nx, ny, nz)
    sim = vlbm.Simulation(cfg, node_map=m)
    sp = [vlbm.Sphere(**s) for s in spheres]
    sim.add_spheres(ib, sp)
    o = oracle.OracleIbm(cfg, m, ib, sp)
    return sim, o, sp


CLOSED = dict(max_iterations=3, gx=0.0, gy=0.0, gz=-2e-5, wall_x=1, wall_y=1, wall_z=1,
              particle_young=1e5, wall_young=1e5, pp_friction=0.3, pw_friction=0.3)

CASES = [
    ("settling_pair_closed_box_q19", 19, 3, (20, 20, 28),
     [dict(diameter=8, cx=9.5, cy=9.7, cz=14.2, density=1.5, movable=1),
      dict(diameter=8, cx=10.1, cy=10.3, cz=5.0, density=1.5, movable=1)],
     CLOSED, dict(tau=0.8), 40),
    ("bingham_channel_periodic_xz_q19", 19, 1, (24, 20, 24),
     [dict(diameter=8, cx=1.5, cy=9.0, cz=12.0, vx=0.01, wz=0.002, density=1.5, movable=1)],
     dict(max_iterations=1, gx=0.0, gy=-1e-5, gz=0.0),
     dict(rheology=1, eta_p=0.1, yield_stress=1e-6, fx=2e-5), 30),
    ("contacts_pair_and_wall_q27", 27, 3, (24, 20, 24),
     [dict(diameter=8, cx=8.0, cy=10.0, cz=12.0, vx=0.02, density=1.5, movable=1),
      dict(diameter=8, cx=15.9, cy=10.2, cz=12.1, vx=-0.02, density=1.5, movable=1),
      dict(diameter=8, cx=12.0, cy=10.0, cz=3.95, vz=-0.01, wx=0.01, density=1.5, movable=1)],
     dict(CLOSED, max_iterations=2, particle_young=0.5, wall_young=100.0), dict(tau=0.7), 25),
    ("fixed_sphere_in_flow_q19", 19, 1, (24, 16, 16),
     [dict(diameter=6, cx=12.0, cy=8.0, cz=8.0, density=1.0, movable=0)],
     dict(max_iterations=2), dict(tau=0.8, fx=1e-5), 60),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_ibm_step_matches_oracle(vlbm, oracle, case):
    name, q, builder, size, spheres, ibm_kw, cfg_kw, steps = case
    sim, o, sp = make_case(vlbm, oracle, q, builder, size, spheres, ibm_kw, cfg_kw)
    x0 = np.array([[s.cx, s.cy, s.cz] for s in sp])
    sim.step(steps)
    sim.sync()
    o.step(steps)
    pg = sim.particles(len(sp))
    po = o.particles()
    pos = np.array([list(p.pos) for p in pg])
    vel = np.array([list(p.vel) for p in pg])
    w = np.array([list(p.w) for p in pg])
    assert np.all(np.abs(pos - po["pos"]) <= 2e-6 + 1e-3 * np.abs(po["pos"] - x0)), (name, pos - po["pos"])
    vscale = max(np.abs(po["vel"]).max(), 1e-12)
    assert np.abs(vel - po["vel"]).max() <= 2e-3 * vscale + 1e-9, (name, vel - po["vel"])
    wscale = max(np.abs(po["w"]).max(), 1e-12)
    assert np.abs(w - po["w"]).max() <= 2e-3 * wscale + 1e-9, (name, w - po["w"])
    mg, mo = sim.macroscopics(), o.macroscopics()
    ug = np.stack([mg["ux"], mg["uy"], mg["uz"]]).astype(np.float64)
    uo = np.stack([mo["ux"], mo["uy"], mo["uz"]])
    rel = np.linalg.norm(ug - uo) / np.linalg.norm(uo)
    assert rel <= 5e-3, (name, rel)
    assert np.abs(ug - uo).max() <= 5e-6, (name, np.abs(ug - uo).max())
    nodes_g, _ = sim.lagrangian_nodes()
    assert np.abs(nodes_g - o.nodes()).max() <= 1e-6 + 1e-3 * np.abs(po["pos"] - x0).max()


def test_sphere_mesh_matches_reference_mesher(vlbm, oracle):
    cfg = vlbm.Config.default(nx=24, ny=24, nz=24)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CLOSED_BOX)
    c = (11.3, 12.0, 12.7)
    sim.add_spheres(vlbm.IbmConfig.default(), [vlbm.Sphere(diameter=16, cx=c[0], cy=c[1], cz=c[2], density=1.5,
                                                           movable=1)])
    assert sim.info().n_lagrangian_nodes == 608
    pos, _ = sim.lagrangian_nodes()
    xyz, S = oracle.sphere_mesh(16.0)
    np.testing.assert_allclose(pos, xyz + np.array(c)[:, None], atol=1e-12)
    p = sim.particles(1)[0]
    assert p.n_nodes == 608 and abs(p.volume - 4 / 3 * np.pi * 512) < 1e-9


def test_ibm_forces_exported(vlbm):
    cfg = vlbm.Config.default(nx=16, ny=16, nz=16, tau=0.8)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CLOSED_BOX)
    sim.add_spheres(vlbm.IbmConfig.default(**CLOSED),
                    [vlbm.Sphere(diameter=6, cx=8, cy=8, cz=8, vx=0.01, density=1.5, movable=1)])
    sim.step(3)
    f = sim.forces()
    assert np.count_nonzero(f[0]) > 50           # spread force only around the sphere
    assert np.abs(f[0]).max() > 0
    far = f[:, 0:2, :, :]
    assert np.count_nonzero(far) == 0


def test_ibm_reset_is_reproducible(vlbm):
    cfg = vlbm.Config.default(nx=16, ny=16, nz=16, tau=0.8)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_CLOSED_BOX)
    sim.add_spheres(vlbm.IbmConfig.default(**CLOSED),
                    [vlbm.Sphere(diameter=6, cx=8, cy=8, cz=9, density=1.5, movable=1)])
    out = []
    for _ in range(2):
        sim.init_equilibrium(1.0, 0, 0, 0)
        sim.step(10)
        out.append(np.array(list(sim.particles(1)[0].pos)))
    assert np.allclose(out[0], out[1], atol=1e-9, rtol=0)  # float atomics in the spread


def test_ibm_step_bit_reproducible(vlbm):
    """Two runs of the same sphere case give identical fields and particles:
    spread forces are summed in fixed point and sphere forces in a fixed order."""
    name, q, builder, size, spheres, ibm_kw, cfg_kw, steps = CASES[2]
    out = []
    for _ in range(2):
        nx, ny, nz = size
        cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=q, **cfg_kw)
        sim = vlbm.Simulation(cfg, builder=builder)
        sim.add_spheres(vlbm.IbmConfig.default(**ibm_kw), [vlbm.Sphere(**s) for s in spheres])
        sim.step(steps)
        sim.sync()
        m = sim.macroscopics()
        parts = sim.particles(len(spheres))
        out.append((np.stack([m["rho"], m["ux"], m["uy"], m["uz"]]),
                    np.array([list(p.pos) + list(p.vel) + list(p.w) for p in parts])))
        sim.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
