"""z-slab decomposition on the GPU: a lattice split into slabs (zslab.py,
vlbm_halo_pack / vlbm_halo_unpack, vlbm_build_node_map_planes) against the
same lattice in one piece.

The reference splits a lattice into N_GPUS z-slabs with a ghost plane each
and moves the populations crossing a slab face every step
(src/CUDA/lbm.cu:601-657).  This run has one GPU, so every slab lives in one
process on that GPU and the exchange is a device copy between message
buffers, ordered on one stream (LocalSlabs); the multi-process transport is
covered on the host by test_zslab_gloo.py.  With FP32 storage every node of
a slab computes the same values in the same order as in the whole lattice,
so populations and macroscopics must agree bit for bit.
"""
import numpy as np
import pytest
import torch

import zslab

pytestmark = pytest.mark.gpu

# name, Q, collision, rheology, builder, (nx, ny, nz), slabs, layout, extra config
CASES = [
    ("plates_bingham_q19_2", 19, "REG", "BINGHAM", "PLATES_Y", (16, 12, 16), 2, "NATURAL",
     dict(eta_p=0.1, yield_stress=2e-6, fx=4e-5)),
    ("plates_bingham_q19_zpair_blocked_2", 19, "REG", "BINGHAM", "PLATES_Y", (32, 10, 12), 2, "ZPAIR",
     dict(eta_p=0.1, yield_stress=2e-6, fx=4e-5)),
    ("closed_box_powerlaw_q27_3", 27, "REG", "POWERLAW", "CLOSED_BOX", (12, 10, 14), 3, "NATURAL",
     dict(n_index=0.7, k_consistency=0.05, gamma0=1e-9, fz=-2e-5)),
    ("lid_cavity_bgk_q19_2", 19, "BGK", "NEWTONIAN", "LID_CAVITY_CLOSED", (12, 12, 12), 2, "NATURAL",
     dict(tau=0.7, ux_bc=[0.0, 0.05])),
    ("duct_yz_q27_zpair_2", 27, "REG", "NEWTONIAN", "DUCT_YZ", (16, 12, 16), 2, "ZPAIR",
     dict(tau=0.8, fx=2e-5)),
    ("zouhe_couette_q19_2", 19, "REG", "NEWTONIAN", "PLATES_Y_ZOUHE", (8, 12, 12), 2, "NATURAL",
     dict(tau=0.8, uz_bc=[0.0, 0.02, -0.02])),
    ("circular_duct_rotating_q19_3", 19, "REG", "NEWTONIAN", "CIRCULAR_DUCT", (20, 20, 12), 3, "NATURAL",
     dict(tau=0.8, fz=1e-5, duct_outer_rotation=2e-3)),
    ("plates_one_slab_q19_1", 19, "REG", "NEWTONIAN", "PLATES_Y", (8, 10, 8), 1, "NATURAL",
     dict(tau=0.9, fx=1e-5)),
]


def make_cfg(vlbm, q, op, rheo, dims, layout, extra, storage=None):
    nx, ny, nz = dims
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=q,
                              collision=vlbm.OP_REGULARIZED if op == "REG" else vlbm.OP_BGK,
                              rheology=getattr(vlbm, rheo), layout=getattr(vlbm, "LAYOUT_" + layout), device=0,
                              **extra)
    if storage is not None:
        cfg.storage = storage
    return cfg


def perturb(sim, seed):
    """A z-dependent initial state, so that a wrong halo shows at once."""
    rng = np.random.default_rng(seed)
    f = sim.populations()
    return f * (1.0 + 1e-3 * rng.standard_normal(f.shape)).astype(np.float32)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_slabs_equal_the_whole_lattice(vlbm, case):
    name, q, op, rheo, builder, dims, n_slabs, layout, extra = case
    cfg = make_cfg(vlbm, q, op, rheo, dims, layout, extra)
    b = getattr(vlbm, "BUILDER_" + builder)
    whole = vlbm.Simulation(cfg, node_map=vlbm.build_node_map(b, *dims))
    slabs = zslab.LocalSlabs(cfg, b, n_slabs)
    try:
        f0 = perturb(whole, 3)
        whole.set_populations(f0)
        for z0, n, sim in slabs.slabs:
            planes = [(z0 - 1 + k) % dims[2] for k in range(n + 2)]
            sim.set_populations(np.ascontiguousarray(f0[:, planes]))
        done = 0
        for steps in (1, 2, 37):   # ends after an odd and after an even step
            whole.step(steps)
            slabs.step(steps)
            done += steps
            whole.sync()
            torch.cuda.synchronize()
            for _, _, sim in slabs.slabs:
                sim.sync()
            fs, fw = slabs.populations(), whole.populations()
            bad = np.argwhere(fs != fw)
            assert bad.size == 0, f"{name}: after {done} steps, {len(bad)} values differ, first (i, z, y, x) " \
                                  f"{bad[:4].tolist()}, max |d| {np.abs(fs - fw).max():.3e}"
        mw, ms = whole.macroscopics(), slabs.macroscopics()
        for k in ("rho", "ux", "uy", "uz", "omega"):
            assert np.array_equal(ms[k], mw[k]), k
        slabs.refresh()
        total = sum(sim.moments_sum() for _, _, sim in slabs.slabs)
        assert np.allclose(total, whole.moments_sum(), rtol=1e-12, atol=1e-12)
    finally:
        slabs.close()
        whole.close()


@pytest.mark.parametrize("storage", ["STORE_F16", "STORE_BF16"])
def test_half_precision_slabs_stay_within_rounding_of_the_whole_lattice(vlbm, storage):
    """Stochastic rounding draws its bits from the node index, which differs in a
    slab, so half-precision slabs are compared by their distance from the FP32
    run: no larger than the whole half-precision lattice's own (plus 10 %)."""
    dims, extra = (32, 16, 16), dict(eta_p=0.1, yield_stress=2e-6, fx=4e-5)
    b = vlbm.BUILDER_PLATES_Y
    ref = vlbm.Simulation(make_cfg(vlbm, 19, "REG", "BINGHAM", dims, "NATURAL", extra), builder=b)
    cfg = make_cfg(vlbm, 19, "REG", "BINGHAM", dims, "AUTO", extra, storage=getattr(vlbm, storage))
    whole = vlbm.Simulation(cfg, node_map=vlbm.build_node_map(b, *dims))
    slabs = zslab.LocalSlabs(cfg, b, 2)
    try:
        steps = 400
        ref.step(steps)
        whole.step(steps)
        slabs.step(steps)
        torch.cuda.synchronize()
        ur = ref.macroscopics()["ux"]
        ew = np.linalg.norm(whole.macroscopics()["ux"] - ur) / np.linalg.norm(ur)
        es = np.linalg.norm(slabs.macroscopics()["ux"] - ur) / np.linalg.norm(ur)
        assert es <= 1.1 * ew + 1e-5, (es, ew)
    finally:
        slabs.close()
        whole.close()
        ref.close()


def test_slab_refusals(vlbm):
    """Free-slip walls normal to y read their z neighbours' post-collision
    values, a builder id cannot place a slab, and spheres need whole lattices."""
    cfg = vlbm.Config.default(nx=8, ny=10, nz=8, device=0, tau=0.8)
    with pytest.raises(vlbm.VlbmError) as e:
        zslab.LocalSlabs(cfg, vlbm.BUILDER_PLATES_Y_FREE_SLIP, 2)
    assert e.value.status == vlbm.ERR_UNSUPPORTED
    sc = zslab.slab_config(cfg, 0, 4, 8)
    with pytest.raises(vlbm.VlbmError) as e:
        vlbm.Simulation(sc, builder=vlbm.BUILDER_PLATES_Y)
    assert e.value.status == vlbm.ERR_INVALID
    sim = vlbm.Simulation(sc, node_map=zslab.slab_node_map(vlbm.BUILDER_CLOSED_BOX, cfg, 0, 4, 8))
    try:
        with pytest.raises(vlbm.VlbmError) as e:
            sim.add_spheres(vlbm.IbmConfig.default(), [vlbm.Sphere(diameter=4, cx=4, cy=5, cz=3, density=1.5)])
        assert e.value.status == vlbm.ERR_UNSUPPORTED
        buf = torch.empty(sim.halo_bytes(), dtype=torch.uint8, device="cuda")
        for z, dz in ((-1, 1), (6, 1), (1, 0)):
            with pytest.raises(vlbm.VlbmError) as e:
                sim.halo_pack(z, dz, buf)
            assert e.value.status == vlbm.ERR_INVALID
        assert sim.halo_bytes() == 5 * 8 * 10 * 4
    finally:
        sim.close()
    bad = zslab.slab_config(cfg, 0, 4, 8)
    bad.slab_z_offset = 8
    with pytest.raises(vlbm.VlbmError):
        vlbm.Simulation(bad, builder=None)


def test_single_rank_zslab_equals_the_whole_lattice(vlbm):
    """ZSlab outside a process group: one rank whose slab is the whole lattice,
    periodic onto itself through its own message buffers (what
    `bench.py --shard` runs on one GPU); macroscopics after an even and after
    an odd step and the FP64 sums equal the unsharded run's."""
    kw = dict(eta_p=0.1, yield_stress=2e-6, fx=4e-5)
    dims = (32, 12, 10)
    cfg = make_cfg(vlbm, 19, "REG", "BINGHAM", dims, "NATURAL", kw)
    whole = vlbm.Simulation(cfg, node_map=vlbm.build_node_map(vlbm.BUILDER_PLATES_Y, *dims))
    slab = zslab.ZSlab(cfg, vlbm.BUILDER_PLATES_Y)
    try:
        assert (slab.z0, slab.n, slab.transport.world) == (0, dims[2], 1)
        for steps in (7, 1):   # 7 and 8 steps taken: after an even and after an odd step
            whole.step(steps)
            slab.step(steps)
            whole.sync()
            torch.cuda.synchronize()
            mw, ms = whole.macroscopics(), slab.macroscopics()
            for k in ("rho", "ux", "uy", "uz"):
                assert np.array_equal(ms[k], mw[k]), (steps, k)
        assert np.allclose(slab.moments_sum(), whole.moments_sum(), rtol=1e-12, atol=1e-12)
    finally:
        slab.close()
        whole.close()
