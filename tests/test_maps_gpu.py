"""GPU grid maps against the reference's cache::populate_no_bias (FP32)."""
import numpy as np
import pytest

from oracle import ref
from unidock_tools import engine, synth

from .conftest import BOX_CENTER, BOX_SIZE

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not ref.available(), reason="reference build missing")]

TYPES = [0, 1, 2, 3, 4, 5, 8, 9, 10, 12, 13]


@pytest.fixture(scope="module")
def maps_pair(receptor):
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375, types=TYPES)
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, BOX_SIZE, 0.375, types=TYPES)
    return M, R


def test_map_frame_matches_reference(maps_pair):
    M, R = maps_pair
    dims, init, fac, n = M.info()
    np.testing.assert_array_equal(dims, R.dims)
    np.testing.assert_array_equal(init, R.init)
    np.testing.assert_array_equal(fac, R.factor)
    assert n == len(TYPES)
    assert tuple(dims) == (61, 61, 61)


@pytest.mark.parametrize("xs", TYPES)
def test_map_values_match_reference(maps_pair, xs):
    M, R = maps_pair
    a, b = M.read(xs), R.get(xs)
    # tolerance: 1e-5 relative to the map's own scale (values near 0 cancel)
    scale = np.abs(b).max()
    err = np.abs(a - b)
    assert err.max() <= 1e-5 * scale, (err.max(), scale)
    # the kernel sums in the reference's order without contraction: expect bit-exact
    assert np.mean(a == b) > 0.999


def test_vinardo_maps(receptor):
    M = engine.Maps(receptor.xyz, receptor.xs, BOX_CENTER, np.full(3, 12.0, np.float32), 0.5,
                    sf=engine.SF_VINARDO, types=[0, 8])
    R = ref.RefMaps(receptor.xyz, receptor.xs, BOX_CENTER, np.full(3, 12.0, np.float32), 0.5, sf=2, types=[0, 8])
    for t in (0, 8):
        a, b = M.read(t), R.get(t)
        assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
