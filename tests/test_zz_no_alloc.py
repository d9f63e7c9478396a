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
