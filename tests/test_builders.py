"""libvlbm's host builders produce the reference builders' node-map words bit for bit."""
import numpy as np
import pytest

SIZES = [(6, 5, 4), (4, 7, 5), (1, 4, 3), (9, 3, 2)]


@pytest.mark.parametrize("builder", range(9))
@pytest.mark.parametrize("size", SIZES)
def test_builder_bit_exact(vlbm, oracle, builder, size):
    nx, ny, nz = size
    got = vlbm.build_node_map(builder, nx, ny, nz)
    ref = oracle.reference_builder_map(oracle.BUILDER_NAMES[builder], nx, ny, nz)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("builder", [9, 10])
@pytest.mark.parametrize("size", [(17, 17, 2), (24, 20, 3), (33, 32, 1), (16, 40, 2)])
def test_duct_builder_bit_exact(vlbm, oracle, builder, size):
    """Circular and annular ducts (interpolated bounce-back), float geometry as the reference."""
    nx, ny, nz = size
    got = vlbm.build_node_map(builder, nx, ny, nz)
    ref = oracle.reference_builder_map(oracle.BUILDER_NAMES[builder], nx, ny, nz)
    np.testing.assert_array_equal(got, ref)
    used = (got >> vlbm.MAP_IS_USED_OFFSET) & 1
    interp = ((got >> vlbm.MAP_SCHEME_OFFSET) & 7) == vlbm.BC_INTERP_BOUNCE_BACK
    assert 0 < used.sum() < got.size and interp.sum() > 0
    # every unknown direction of a wall node points to a node outside the fluid
    g = got.reshape(nz, ny, nx)
    dirs = [(1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)]
    for y in range(ny):
        for x in range(nx):
            w = int(g[0, y, x])
            if ((w >> vlbm.MAP_SCHEME_OFFSET) & 7) != vlbm.BC_INTERP_BOUNCE_BACK:
                continue
            for d, (dx, dy) in enumerate(dirs):
                xs, ys = x - dx, y - dy
                outside = not (0 <= xs < nx and 0 <= ys < ny) or not ((int(g[0, ys, xs]) >> 21) & 1)
                assert bool((w >> (23 + d)) & 1) == outside, (x, y, d)


def test_builder_rejects_bad_args(vlbm):
    with pytest.raises(vlbm.VlbmError):
        vlbm.build_node_map(99, 4, 4, 4)
