"""Checkpoint and resume (simCheckpoint.cu:216-318) through the C ABI.

A run of K steps, saved, loaded into a fresh simulation and continued for K
more steps must equal an uninterrupted run of 2K steps bit for bit: the
populations as stored (AA parity, half-precision bits), boundary side stores,
Power-Law omega, stochastic-rounding step counters and the IBM state (contact
history included) all travel in the image.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONTACTS = dict(max_iterations=2, gx=0.0, gy=0.0, gz=-2e-5, wall_x=1, wall_y=1, wall_z=1,
                particle_young=0.5, wall_young=100.0, pp_friction=0.3, pw_friction=0.3)
SPHERES = [dict(diameter=8, cx=8.0, cy=10.0, cz=12.0, vx=0.02, density=1.5, movable=1),
           dict(diameter=8, cx=15.9, cy=10.2, cz=12.1, vx=-0.02, density=1.5, movable=1),
           dict(diameter=8, cx=12.0, cy=10.0, cz=3.95, vz=-0.01, wx=0.01, density=1.5, movable=1)]

# (name, config, builder, spheres, K)
CASES = [
    ("f32_bingham_plates_odd", dict(nx=16, ny=12, nz=8, vel_set=19, rheology=1, eta_p=0.1,
                                    yield_stress=1e-6, fx=2e-4), 1, None, 7),
    ("f32_bgk_closed_box_even", dict(nx=9, ny=8, nz=7, vel_set=27, collision=1, tau=0.8, fx=1e-4,
                                     fy=-2e-4), 3, None, 6),
    ("f16_zpair_powerlaw_cavity", dict(nx=12, ny=12, nz=12, vel_set=27, rheology=2, n_index=0.5,
                                       k_consistency=0.02, ux_bc=[0, 0.05], storage=1), 6, None, 9),
    ("bf16_duct_q19", dict(nx=20, ny=10, nz=10, vel_set=19, tau=0.9, fx=1e-4, storage=2), 5, None, 5),
    ("ibm_contacts_q27", dict(nx=24, ny=20, nz=24, vel_set=27, tau=0.7), 3, SPHERES, 11),
    # NX a multiple of 32: z-paired populations in blocks of 32 pair-nodes
    ("f16_blocked_pairs_channel", dict(nx=32, ny=12, nz=8, vel_set=19, rheology=1, eta_p=0.1,
                                       yield_stress=1e-6, fx=2e-4, storage=1), 1, None, 7),
    ("ibm_blocked_pairs_q27", dict(nx=32, ny=20, nz=24, vel_set=27, tau=0.7), 3, SPHERES, 9),
]


def make(vlbm, cfg_kw, builder, spheres):
    cfg = vlbm.Config.default(**cfg_kw)
    sim = vlbm.Simulation(cfg, builder=builder)
    if spheres:
        sim.add_spheres(vlbm.IbmConfig.default(**CONTACTS), [vlbm.Sphere(**s) for s in spheres])
    return sim


def state(sim, spheres):
    m = sim.macroscopics()
    out = {"pops": sim.populations(), "rho": m["rho"], "ux": m["ux"], "uy": m["uy"], "uz": m["uz"],
           "step": sim.info().step}
    if "omega" in m:
        out["omega"] = m["omega"]
    if spheres:
        parts = sim.particles(len(spheres))
        out["parts"] = np.array([list(p.pos) + list(p.vel) + list(p.w) + list(p.f) + list(p.M)
                                 for p in parts])
        pos, frc = sim.lagrangian_nodes()
        out["nodes"] = np.concatenate([pos.ravel(), frc.ravel()])
    return out


def assert_same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_resume_continues_bit_for_bit(vlbm, case):
    name, cfg_kw, builder, spheres, K = case
    ref = make(vlbm, cfg_kw, builder, spheres)
    ref.step(2 * K)
    ref.sync()
    want = state(ref, spheres)
    ref.close()

    a = make(vlbm, cfg_kw, builder, spheres)
    a.step(K)
    a.sync()
    image = a.checkpoint()
    a.close()
    b = make(vlbm, cfg_kw, builder, spheres)
    b.restore(image)
    assert b.info().step == K
    b.step(K)
    b.sync()
    got = state(b, spheres)
    b.close()
    assert_same(got, want)


def test_file_roundtrip_and_missing_file(vlbm, tmp_path):
    name, cfg_kw, builder, spheres, K = CASES[0]
    a = make(vlbm, cfg_kw, builder, spheres)
    a.step(K)
    a.save_checkpoint(str(tmp_path), "run1")
    assert (tmp_path / "run1" / "checkpoint" / "0_state.bin").is_file()
    b = make(vlbm, cfg_kw, builder, spheres)
    b.load_checkpoint(str(tmp_path), "run1")
    a.step(3)
    b.step(3)
    np.testing.assert_array_equal(a.populations(), b.populations())
    with pytest.raises(vlbm.VlbmError) as e:
        b.load_checkpoint(str(tmp_path), "no_such_run")
    assert e.value.status == vlbm.ERR_NOT_FOUND


def test_rejected_images_leave_the_simulation_unchanged(vlbm):
    name, cfg_kw, builder, spheres, K = CASES[0]
    a = make(vlbm, cfg_kw, builder, spheres)
    a.step(K)
    image = a.checkpoint()
    b = make(vlbm, cfg_kw, builder, spheres)
    b.step(2)
    before = b.populations()

    def rejected(img, status=vlbm.ERR_INVALID, sim=b):
        with pytest.raises(vlbm.VlbmError) as e:
            sim.restore(img)
        assert e.value.status == status

    bad = image.copy()
    bad[len(bad) // 2] ^= 0x10                 # one flipped bit in the populations
    rejected(bad)
    rejected(image[:-1])                         # truncated
    rejected(image[:100])
    wrong_version = image.copy()
    wrong_version[8] = 99
    rejected(wrong_version, vlbm.ERR_UNSUPPORTED)
    np.testing.assert_array_equal(b.populations(), before)
    assert b.info().step == 2

    other_size = make(vlbm, dict(cfg_kw, nx=cfg_kw["nx"] + 2), builder, spheres)
    rejected(image, sim=other_size)
    other_geometry = make(vlbm, cfg_kw, vlbm.BUILDER_DUCT_YZ, spheres)
    rejected(image, sim=other_geometry)
    other_storage = make(vlbm, dict(cfg_kw, storage=1), builder, spheres)
    rejected(image, sim=other_storage)

    # a buffer smaller than the image is refused with nothing written
    need = ctypes.c_size_t()
    small = np.zeros(16, dtype=np.uint8)
    st = vlbm.lib().vlbm_checkpoint_save(a._h, small.ctypes.data_as(ctypes.c_void_p), small.size,
                                         ctypes.byref(need))
    assert st == vlbm.ERR_INVALID and need.value == image.size
    assert not small.any()
