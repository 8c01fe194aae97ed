"""The remapping oracle pinned on the CPU (no GPU, no healpy).

Pins, in the absence of healpy (the reference's own comparison in
tests/test_data_remapping.py): known answers of the HEALPix definition at
nside 1 and 2, the NEST hierarchy measured against the ring geometry that the
SHT oracle shares with the reference, the independent definition of the
counter-clockwise south-origin flat layout, and consistency of the reference's
direct flat->flat formula with the composition of its flat->nest and
nest->flat formulas.  Also the argument checks of cuhpx/hpx_remap.py:24-102.
"""

import itertools

import numpy as np
import pytest

from oracle import hpx_oracle as O
from oracle import remap_oracle as R

ORIENTS = [(o, cw) for o in range(4) for cw in (False, True)]


def ring_pixel_vectors(nside):
    """Unit vectors of every RING pixel centre from the SHT oracle's ring geometry."""
    z = O.ring_z(nside)
    out = []
    for t in range(O.nrings(nside)):
        n = O.nphi_ring(t, nside)
        phi = O.ring_phi0(t, nside) + 2 * np.pi * np.arange(n) / n
        s = np.sqrt(1 - z[t] ** 2)
        out.append(np.stack([s * np.cos(phi), s * np.sin(phi), np.full(n, z[t])], 1))
    return np.concatenate(out)


def test_known_answers():
    assert np.array_equal(R.destination("ring2nest", 1), np.arange(12))
    assert np.array_equal(R.destination("nest2ring", 1), np.arange(12))
    # nside 2: the four pixels of base face 0 in NEST order sit on rings 2, 1, 1, 0
    assert R.destination("nest2ring", 2)[:4].tolist() == [13, 5, 4, 0]
    # polar rings: the north corners (ix = iy = 1) of faces 0-3, the south corners of faces 8-11
    assert R.destination("ring2nest", 2)[[0, 1, 2, 3]].tolist() == [3, 7, 11, 15]
    assert R.destination("ring2nest", 2)[[44, 45, 46, 47]].tolist() == [32, 36, 40, 44]


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 16, 64])
def test_permutations_and_inverses(nside):
    n = 12 * nside * nside
    r2n = R.destination("ring2nest", nside)
    n2r = R.destination("nest2ring", nside)
    assert np.array_equal(np.sort(r2n), np.arange(n))
    assert np.array_equal(n2r[r2n], np.arange(n))
    ix, iy, f = R.ring2xyf(np.arange(n), nside)
    assert np.array_equal(R.xyf2ring(ix, iy, f, nside), np.arange(n))
    for o, cw in ORIENTS:
        a = R.destination("nest2flat", nside, o, cw)
        b = R.destination("flat2nest", nside, o, cw)
        assert np.array_equal(b[a], np.arange(n))
        c = R.destination("ring2flat", nside, o, cw)
        d = R.destination("flat2ring", nside, o, cw)
        assert np.array_equal(d[c], np.arange(n))


@pytest.mark.parametrize("nside", [2, 4, 8])
def test_nest_hierarchy_against_ring_geometry(nside):
    """Every NEST pixel at 2*nside is nearest to the centre of its own parent at nside."""
    child = ring_pixel_vectors(2 * nside)[R.destination("nest2ring", 2 * nside)]  # by NEST index
    parent = ring_pixel_vectors(nside)[R.destination("nest2ring", nside)]
    nearest = np.argmax(child @ parent.T, axis=1)
    assert np.array_equal(nearest, np.arange(12 * 4 * nside * nside) >> 2)


def test_flat_south_counter_clockwise_definition():
    nside = 8
    x = np.arange(12 * nside * nside)
    flat = R.nest2flat(x, "S", False, nside).reshape(12, nside, nside)
    nest = x.reshape(12, nside * nside)
    for iy, ix in itertools.product(range(nside), range(nside)):
        q = int(R._spread(ix)) + 2 * int(R._spread(iy))
        assert np.array_equal(flat[:, iy, ix], nest[:, q])


def test_flat2flat_is_the_composition():
    nside = 4
    for (so, scw), (do, dcw) in itertools.product(ORIENTS, ORIENTS):
        direct = R.destination("flat2flat", nside, so, scw, do, dcw)
        via = R.destination("nest2flat", nside, do, dcw)[R.destination("flat2nest", nside, so, scw)]
        assert np.array_equal(direct, via)


def test_batch_and_dtype_pass_through():
    nside = 4
    rng = np.random.default_rng(0)
    x = rng.standard_normal((2, 3, 12 * nside * nside)).astype(np.float32)
    y = R.nest2ring(x, nside)
    assert y.shape == x.shape and y.dtype == x.dtype
    assert np.array_equal(R.ring2nest(y, nside), x)


def test_argument_errors():
    with pytest.raises(ValueError, match="power of two"):
        R.ring2nest(np.zeros(12 * 9), 3)
    with pytest.raises(RuntimeError, match="number of elements"):
        R.nest2ring(np.zeros(12 * 4 + 1), 2)
    with pytest.raises(RuntimeError, match="S, E, N, W"):
        R.nest2flat(np.zeros(48), "X", False, 2)
    with pytest.raises(RuntimeError, match="src origin"):
        R.flat2flat(np.zeros(48), "Q", False, "S", False, 2)
