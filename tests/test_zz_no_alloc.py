"""The allocation-free reduction entry point against the allocating one.

vlbm_moments_sum_noalloc serves callers that cannot allocate device memory when
they want global mass and momentum (for example a serving process whose HBM is
fully committed to admitted simulations).  It must return what vlbm_moments_sum
returns, on repeated calls, while using only its built-in scratch array.  This
file is collected last so a stop-at-first-failure run has already run every
other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sums(vlbm, fn, sim):
    out = np.zeros(4, dtype=np.float64)
    st = fn(sim.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st == vlbm.OK, vlbm.lib().vlbm_last_error()
    return out


@pytest.mark.parametrize("q,builder,size,steps", [(19, 3, (40, 24, 18), 13), (27, 6, (16, 16, 16), 8)])
def test_noalloc_matches_allocating_entry_point_on_two_calls(vlbm, q, builder, size, steps):
    lib = vlbm.lib()
    nx, ny, nz = size
    cfg = vlbm.Config.default(nx=nx, ny=ny, nz=nz, vel_set=q, tau=0.8, fx=1e-4, fz=-3e-5)
    sim = vlbm.Simulation(cfg, builder=builder)
    sim.step(steps)
    for _ in range(2):
        ref = _sums(vlbm, lib.vlbm_moments_sum, sim)
        got = _sums(vlbm, lib.vlbm_moments_sum_noalloc, sim)
        np.testing.assert_array_equal(got, ref)
        assert abs(got[0] - nx * ny * nz) < 1e-3 * nx * ny * nz
        sim.step(1)


def test_noalloc_rejects_lattices_beyond_its_scratch(vlbm):
    lib = vlbm.lib()
    cfg = vlbm.Config.default(nx=4097, ny=128, nz=128, storage=vlbm.STORE_F16)  # 67,125,248 nodes
    sim = vlbm.Simulation(cfg)
    out = np.zeros(4, dtype=np.float64)
    st = lib.vlbm_moments_sum_noalloc(sim.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert st == vlbm.ERR_INVALID
    assert b"67108864" in lib.vlbm_last_error()
    sim.close()


def test_noalloc_first_on_a_fresh_simulation_allocates_nothing(vlbm):
    """Called first on a fresh simulation (no earlier vlbm_moments_sum), the
    allocation-free path leaves the simulation's device bytes and the device's
    free memory (cudaMemGetInfo) unchanged, and then agrees with the allocating
    entry point."""
    import torch
    lib = vlbm.lib()
    # CUDA loads a module's code and device globals (the scratch array among
    # them) at its first use in the process; a call on another simulation does
    # that first, so the measurement below sees only what the call itself does
    warm = vlbm.Simulation(vlbm.Config.default(nx=8, ny=8, nz=8))
    _sums(vlbm, lib.vlbm_moments_sum_noalloc, warm)
    warm.close()
    cfg = vlbm.Config.default(nx=48, ny=20, nz=16, vel_set=19, tau=0.7, fx=2e-5)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
    sim.step(9)
    sim.sync()
    torch.cuda.synchronize()
    before_sim = sim.info().device_bytes
    before_free = torch.cuda.mem_get_info(0)[0]
    got = [_sums(vlbm, lib.vlbm_moments_sum_noalloc, sim) for _ in range(2)]
    torch.cuda.synchronize()
    assert sim.info().device_bytes == before_sim
    assert torch.cuda.mem_get_info(0)[0] == before_free
    np.testing.assert_array_equal(got[0], got[1])
    np.testing.assert_array_equal(got[0], _sums(vlbm, lib.vlbm_moments_sum, sim))
    sim.close()


def test_noalloc_accepts_the_largest_lattice_its_scratch_covers(vlbm):
    """67,108,864 nodes (16384 partial sums, the whole scratch array) is
    accepted and agrees with the allocating entry point."""
    lib = vlbm.lib()
    cfg = vlbm.Config.default(nx=4096, ny=128, nz=128, storage=vlbm.STORE_F16, fx=1e-5)
    sim = vlbm.Simulation(cfg, builder=vlbm.BUILDER_PLATES_Y)
    sim.step(2)
    got = _sums(vlbm, lib.vlbm_moments_sum_noalloc, sim)
    np.testing.assert_array_equal(got, _sums(vlbm, lib.vlbm_moments_sum, sim))
    assert abs(got[0] - 4096 * 128 * 128) < 1e-6 * 4096 * 128 * 128
    sim.close()
