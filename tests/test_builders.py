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


def test_builder_rejects_bad_args(vlbm):
    with pytest.raises(vlbm.VlbmError):
        vlbm.build_node_map(99, 4, 4, 4)
