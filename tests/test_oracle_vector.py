"""The vector (spin-1) oracle against golden vectors of the reference's own VectorSHT / VectoriSHT."""

import os

import numpy as np
import pytest

from oracle import vector_oracle as V

G = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


@pytest.mark.parametrize("name", ["n8", "n8_nocs", "n4_mlt", "n4_mgt"])
def test_vector_oracle_pinned(name):
    d = np.load(os.path.join(G, "vector_small.npz"))
    nside, L, M, cs = (int(v) for v in d[name + "_cfg"])
    # the reference evaluates its ring phases in complex64 (cuhpx/hpx_sht.py:50, 64): ~1e-7
    assert rel(V.vsht(d[name + "_f"], nside, L, M, csphase=bool(cs)), d[name + "_alm"]) < 1e-6
    assert rel(V.visht(d[name + "_a"], nside, csphase=bool(cs)), d[name + "_map"]) < 1e-6


def test_csphase_flips_odd_orders():
    x = np.cos(np.linspace(0.1, 3.0, 7))
    a = V.dlegendre(6, 8, x, csphase=True)
    b = V.dlegendre(6, 8, x, csphase=False)
    assert np.array_equal(a[:, 0::2], b[:, 0::2])
    assert np.array_equal(a[:, 1::2], -b[:, 1::2])
