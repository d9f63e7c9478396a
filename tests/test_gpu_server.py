"""Continuous-batching server: results alone and in the mix, HBM-budget admission.

Alone vs in the mix (both through the server): bit for bit.  Which kernel steps
a lattice depends only on the lattice (its size and whether it has spheres),
and the IBM step sums its spread forces in fixed point and its sphere forces in
a fixed order, so a result does not depend on the other lattices.

Server vs a plain vlbm_sim: lattices with their own launches (spheres, or a
full wave of the batched kernel) keep the library's layout (LAYOUT_AUTO) and
run the same kernels, so they match a plain simulation in that layout bit for
bit; small lattices run the batched kernel in the natural layout, which
inlines the same per-node code but may contract a multiply-add differently
(one FP32 rounding), so they must match a natural-layout simulation to
relative L2 1e-4 after the few hundred steps run here.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REQS = [
    # (tag, config, builder, steps, spheres)
    (1, dict(nx=40, ny=20, nz=20, vel_set=19, rheology=1, eta_p=0.1, yield_stress=1e-5, fx=2e-5, storage=1), 5, 301, []),
    (2, dict(nx=24, ny=24, nz=24, vel_set=27, tau=0.7, fx=1e-5, fz=-2e-5), 3, 250, []),
    (3, dict(nx=32, ny=16, nz=16, vel_set=19, collision=1, tau=0.9, fx=1e-5), 1, 420, []),
    (4, dict(nx=20, ny=20, nz=20, vel_set=19, tau=0.8), 3, 120,
     [dict(diameter=6, cx=10.0, cy=10.2, cz=11.0, density=1.5, movable=1)]),
    (5, dict(nx=33, ny=18, nz=17, vel_set=27, rheology=1, eta_p=0.2, yield_stress=1e-6, fx=3e-5, storage=1), 5, 77,
     []),
    # smaller spheres admitted after request 4: the staged-box shared memory of
    # the interpolation kernel must still cover request 4's larger boxes
    (6, dict(nx=16, ny=16, nz=16, vel_set=27, tau=0.9, storage=1), 3, 90,
     [dict(diameter=5, cx=5.5, cy=8.0, cz=8.5, density=1.5, movable=1),
      dict(diameter=4, cx=11.0, cy=9.0, cz=7.0, density=2.0, movable=1)]),
    (7, dict(nx=30, ny=10, nz=14, vel_set=19, rheology=2, n_index=0.7, k_consistency=0.05, fx=2e-5, storage=2), 1,
     33, []),
    # cylinder ducts: interpolated bounce-back and unused nodes in the batched kernel
    (8, dict(nx=22, ny=22, nz=12, vel_set=19, rheology=1, eta_p=0.1, yield_stress=1e-6, fz=2e-5, storage=1), 9,
     140, []),
    (9, dict(nx=20, ny=24, nz=6, vel_set=27, tau=0.8, fz=1e-5, duct_inner_rotation=0.01), 10, 95, []),
]
IBM_KW = dict(max_iterations=2, gx=0.0, gy=0.0, gz=-1e-5, wall_x=1, wall_y=1, wall_z=1)


def cfg_of(vlbm, kw):
    c = vlbm.Config.default(**kw)
    c.layout = vlbm.LAYOUT_NATURAL
    return c


def alone(vlbm, kw, builder, steps, spheres):
    cfg = cfg_of(vlbm, kw)
    if spheres:   # the server keeps the library's layout for lattices with spheres
        cfg.layout = vlbm.LAYOUT_AUTO
    sim = vlbm.Simulation(cfg, builder=builder)
    if spheres:
        sim.add_spheres(vlbm.IbmConfig.default(**IBM_KW), [vlbm.Sphere(**s) for s in spheres])
    sim.step(steps)
    sim.sync()
    ux = sim.macroscopics()["ux"].ravel().copy()
    sim.close()
    return ux


def alone_in_server(vlbm, kw, builder, steps, spheres):
    srv = vlbm.Server(device=0, hbm_budget_bytes=1 << 30, max_resident=1)
    srv.submit(cfg_of(vlbm, kw), builder, steps, 0, [vlbm.Sphere(**s) for s in spheres],
               vlbm.IbmConfig.default(**IBM_KW))
    done = drain(srv)
    assert len(done) == 1 and done[0].status == vlbm.OK
    ux = srv.fetch(0, kw["nx"] * kw["ny"] * kw["nz"])
    srv.close()
    return ux


def drain(srv, chunk=64, limit=100000):
    out = []
    for _ in range(limit):
        out += srv.pump(chunk)
        st = srv.stats()
        if st["resident"] == 0 and st["queued"] == 0:
            return out + srv.pump(1)
    raise AssertionError("server did not drain")


def test_results_same_alone_and_in_the_mix(vlbm):
    srv = vlbm.Server(device=0, hbm_budget_bytes=4 << 30, max_resident=8)
    for tag, kw, builder, steps, spheres in REQS:
        srv.submit(cfg_of(vlbm, kw), builder, steps, tag, [vlbm.Sphere(**s) for s in spheres],
                   vlbm.IbmConfig.default(**IBM_KW))
    done = {c.tag: c for c in drain(srv)}
    assert sorted(done) == [r[0] for r in REQS]
    for tag, kw, builder, steps, spheres in REQS:
        c = done[tag]
        assert c.status == vlbm.OK and c.steps == steps
        assert c.submit_time_s <= c.start_time_s <= c.finish_time_s
        n = kw["nx"] * kw["ny"] * kw["nz"]
        mix = srv.fetch(tag, n)
        np.testing.assert_array_equal(mix, alone_in_server(vlbm, kw, builder, steps, spheres),
                                      err_msg=f"request {tag}")
        assert abs(c.mean_ux - mix.astype(np.float64).mean()) <= 1e-12 * np.abs(mix).max()
        ref = alone(vlbm, kw, builder, steps, spheres)
        if spheres:
            np.testing.assert_array_equal(mix, ref, err_msg=f"request {tag}")
        else:
            assert np.linalg.norm(mix - ref) <= 1e-4 * np.linalg.norm(ref), tag
    srv.close()


def test_late_arrivals_join_running_batch(vlbm):
    """Requests submitted while others are on the GPU give the same results."""
    srv = vlbm.Server(device=0, hbm_budget_bytes=4 << 30, max_resident=4)
    a = dict(nx=24, ny=12, nz=12, vel_set=19, rheology=1, eta_p=0.15, yield_stress=1e-5, fx=3e-5, storage=1)
    b = dict(nx=18, ny=14, nz=10, vel_set=27, tau=0.75, fx=2e-5)
    srv.submit(cfg_of(vlbm, a), 5, 200, 10)
    got = srv.pump(37)
    srv.submit(cfg_of(vlbm, b), 5, 101, 11)
    got += srv.pump(13)
    srv.submit(cfg_of(vlbm, a), 5, 55, 12)
    got += drain(srv, chunk=17)
    assert sorted(c.tag for c in got) == [10, 11, 12]
    for tag, kw, steps in [(10, a, 200), (11, b, 101), (12, a, 55)]:
        np.testing.assert_array_equal(srv.fetch(tag, kw["nx"] * kw["ny"] * kw["nz"]),
                                      alone_in_server(vlbm, kw, 5, steps, []), err_msg=f"request {tag}")
    srv.close()


def request_bytes(q, nx, ny, nz, store_bytes=4):
    """The server's admission estimate for a sphere-free Newtonian/Bingham lattice."""
    n = nx * ny * nz
    walls = 2 * (nx * ny + ny * nz + nx * nz)
    return q * n * store_bytes + 25 * n + (1 << 20) + walls * (2 * q * 4 + 24)


def test_budget_admission_limits_residency(vlbm):
    one = request_bytes(19, 32, 32, 32)
    srv = vlbm.Server(device=0, hbm_budget_bytes=int(one * 1.5), max_resident=8)
    kw = dict(nx=32, ny=32, nz=32, tau=0.8, fx=1e-5)
    for tag in range(4):
        srv.submit(cfg_of(vlbm, kw), vlbm.BUILDER_PLATES_Y, 50 + 10 * tag, tag)
    peak, done = 0, []
    for _ in range(1000):
        done += srv.pump(7)
        st = srv.stats()
        peak = max(peak, st["resident"])
        assert st["bytes"] <= one * 1.5
        if st["resident"] == 0 and st["queued"] == 0:
            break
    assert peak == 1
    assert sorted(c.tag for c in done) == [0, 1, 2, 3]
    assert srv.stats()["bytes"] == 0
    srv.close()


def test_oversized_and_invalid_requests_rejected(vlbm):
    srv = vlbm.Server(device=0, hbm_budget_bytes=64 << 20, max_resident=2)
    with pytest.raises(vlbm.VlbmError):
        srv.submit(cfg_of(vlbm, dict(nx=128, ny=128, nz=128)), vlbm.BUILDER_PLATES_Y, 10, 1)
    with pytest.raises(vlbm.VlbmError):
        srv.submit(cfg_of(vlbm, dict(nx=8, ny=8, nz=8, tau=0.3)), vlbm.BUILDER_PLATES_Y, 10, 2)
    with pytest.raises(vlbm.VlbmError):
        srv.submit(cfg_of(vlbm, dict(nx=8, ny=8, nz=8)), vlbm.BUILDER_PLATES_Y, 0, 3)
    srv.close()


def test_many_lattices_share_persistent_blocks(vlbm):
    """More tiles than resident blocks: each block of the batched launch walks
    tiles of several lattices, admitted at different steps (both AA parities
    in one table); every result equals the same request alone."""
    # one kernel family, 36 x 54-74 tiles of 256 nodes: more tiles than the
    # grid's 148 x (blocks per SM) persistent blocks
    kws = [dict(nx=24 + 2 * (k % 5), ny=24, nz=24, vel_set=19, rheology=1, eta_p=0.1,
                yield_stress=1e-5, fx=2e-5, storage=1) for k in range(36)]
    srv = vlbm.Server(device=0, hbm_budget_bytes=8 << 30, max_resident=64)
    for k, kw in enumerate(kws[:24]):
        srv.submit(cfg_of(vlbm, kw), 5, 40 + k, k)
    got = srv.pump(5)
    for k, kw in enumerate(kws[24:], start=24):
        srv.submit(cfg_of(vlbm, kw), 5, 40 + k, k)
    got += drain(srv, chunk=9)
    assert sorted(c.tag for c in got) == list(range(36))
    for k in (0, 7, 23, 24, 30, 35):
        kw = kws[k]
        np.testing.assert_array_equal(srv.fetch(k, kw["nx"] * kw["ny"] * kw["nz"]),
                                      alone_in_server(vlbm, kw, 5, 40 + k, []), err_msg=f"request {k}")
    srv.close()


def test_device_footprint_stays_within_budget(vlbm):
    """Live and cached device bytes of the server's memory cache stay at or
    below the HBM budget through admit / retire cycles of lattices of
    different sizes (the cache frees what it holds beyond the budget)."""
    budget = int(request_bytes(19, 40, 32, 32) * 1.3)
    srv = vlbm.Server(device=0, hbm_budget_bytes=budget, max_resident=8)
    sizes = [(40, 32, 32), (24, 24, 24), (36, 30, 28), (16, 40, 40), (40, 32, 32), (20, 20, 20)]
    for tag, (nx, ny, nz) in enumerate(sizes):
        srv.submit(cfg_of(vlbm, dict(nx=nx, ny=ny, nz=nz, tau=0.8, fx=1e-5)), vlbm.BUILDER_PLATES_Y, 30 + 5 * tag, tag)
    done, peak = [], 0.0
    for _ in range(2000):
        done += srv.pump(5)
        p = srv.profile()
        held = p["device_live_bytes"] + p["device_cached_bytes"]
        peak = max(peak, held)
        assert held <= budget, (held, budget)
        st = srv.stats()
        if st["resident"] == 0 and st["queued"] == 0:
            break
    assert sorted(c.tag for c in done) == list(range(len(sizes)))
    assert all(c.status == vlbm.OK for c in done)
    assert peak > 0
    srv.close()


def test_large_lattice_keeps_the_library_layout(vlbm):
    """A lattice that fills a wave of the batched kernel by itself steps with
    launches of its own in the library's layout (z-paired for FP16): bit for
    bit a plain simulation in LAYOUT_AUTO."""
    kw = dict(nx=96, ny=48, nz=48, vel_set=19, rheology=1, eta_p=0.1, yield_stress=1e-5, fx=2e-5, storage=1)
    got = alone_in_server(vlbm, kw, 5, 61, [])
    sim = vlbm.Simulation(vlbm.Config.default(**kw), builder=5)
    assert sim.info().layout != 0
    sim.step(61)
    sim.sync()
    ref = sim.macroscopics()["ux"].ravel().copy()
    sim.close()
    np.testing.assert_array_equal(got, ref)
