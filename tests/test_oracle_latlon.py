"""The latitude-longitude oracle (test infrastructure): quadrature exactness and the
Gauss-Legendre round trip, on CPU."""

import numpy as np
import pytest

from oracle import latlon_oracle as LO

GRIDS = ["equiangular", "legendre-gauss", "lobatto"]


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("n", [2, 5, 16, 33])
def test_weights_integrate_polynomials(grid, n):
    z, w = LO.latlon_quadrature(grid, n)
    assert np.all(np.diff(z) < 0)  # north to south
    np.testing.assert_allclose(z, -z[::-1], atol=1e-14)
    exact_deg = {"legendre-gauss": 2 * n - 1, "lobatto": 2 * n - 3, "equiangular": n - 1}[grid]
    for k in range(exact_deg + 1):
        ref = 0.0 if k % 2 else 2.0 / (k + 1)
        assert abs(np.dot(w, z**k) - ref) < 1e-12, (grid, n, k)


@pytest.mark.parametrize("nlat,nlon", [(12, 24), (17, 32)])
def test_gauss_round_trip(nlat, nlon):
    rng = np.random.default_rng(nlat)
    L, M = nlat, nlon // 2 + 1
    a = rng.standard_normal((2, L, M)) + 1j * rng.standard_normal((2, L, M))
    a = np.where(np.arange(M)[None, :] <= np.arange(L)[:, None], a, 0)
    a[..., 0] = a[..., 0].real
    a[..., M - 1] = a[..., M - 1].real  # the ring Nyquist term is real in a real field
    f = LO.latlon_isht(a, nlat, nlon, "legendre-gauss")
    b = LO.latlon_sht(f, L, M, "legendre-gauss")
    assert np.abs(b - a).max() < 1e-11
