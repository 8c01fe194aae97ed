"""The healpy packing oracle against golden vectors of the reference's own index helpers.

``tests/golden/make_healpy_golden.py`` ran ``hp_getidx`` and ``flm_hp_to_2d``
of cuHPX's tests/reproduce_difference_between_healpy_cuhpx.py:58-81 on packed
vectors whose entries are distinct; the oracle must reproduce them exactly.
"""

import os

import numpy as np
import pytest

from oracle import healpy_oracle as H

G = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("L", [8, 13])
def test_index_and_flm2d_match_reference(L):
    d = np.load(os.path.join(G, f"healpy_index_L{L}.npz"))
    idx = np.array([[H.hp_index(L, l, m) for m in range(L)] for l in range(L)])
    assert np.array_equal(idx, d["hp_getidx"])
    assert np.array_equal(H.healpy_to_flm2d(d["packed"], L), d["flm2d"])
    # the dense layout is the non-negative-m half of flm2d
    dense = H.healpy_to_alm(d["packed"], L, L)
    assert np.array_equal(dense, np.where(np.arange(L)[None, :] <= np.arange(L)[:, None], d["flm2d"][:, L - 1:], 0))


@pytest.mark.parametrize("L,M", [(8, 8), (13, 5), (5, 9), (1, 1)])
def test_pack_unpack_round_trip(L, M):
    rng = np.random.default_rng(L * 10 + M)
    a = rng.standard_normal((2, L, M)) + 1j * rng.standard_normal((2, L, M))
    a = np.where(np.arange(M)[None, None, :] <= np.arange(L)[None, :, None], a, 0)
    for cs in (False, True):
        p = H.alm_to_healpy(a, cs)
        assert p.shape == (2, H.packed_size(L, M))
        assert np.array_equal(H.healpy_to_alm(p, L, M, cs), a)
    assert H.packed_size(L, L) == L * (L + 1) // 2
