"""CPU oracle for spherical-harmonic transforms on latitude-longitude grids -- TEST INFRASTRUCTURE ONLY.

cuHPX's Regridding (cuhpx/hpx_regrid.py:69, 84) delegates these grids to
torch_harmonics.RealSHT / InverseRealSHT.  torch_harmonics is neither vendored
in cuHPX nor installed here, so parity with it is UNPINNED: this module
restates its published algorithm (quadrature-weighted Legendre contraction of
per-ring real FFTs scaled by 2 pi / nlon; synthesis by Legendre sums and an
unnormalised inverse real FFT) in float64 numpy, with the orthonormal Pbar of
hpx_oracle.legendre_column and no Condon-Shortley phase.  It is checked by
properties instead (tests/test_oracle_latlon.py): the weights integrate
polynomials exactly to the rule's degree, and Gauss-Legendre analysis inverts
synthesis to rounding for band-limited coefficients.

Only tests/ may import it; the GPU transforms never call it.
"""

import numpy as np

from .hpx_oracle import legendre_column


def latlon_quadrature(grid, nlat):
    """(z, w): cos(theta) of the rings, north to south, and weights summing to 2."""
    n = int(nlat)
    if grid == "legendre-gauss":
        # numpy's nodes, polished by Newton steps on P_n with P_j' = j P_{j-1} + x P_{j-1}'
        x, _ = np.polynomial.legendre.leggauss(n)
        for _ in range(3):
            p0, p1, d1 = np.ones_like(x), x.copy(), np.ones_like(x)
            for j in range(2, n + 1):
                p0, p1, d1 = p1, ((2 * j - 1) * x * p1 - (j - 1) * p0) / j, j * p1 + x * d1
            if n == 1:
                p1, d1 = x.copy(), np.ones_like(x)
            x = x - p1 / d1
        p0, p1, d1 = np.ones_like(x), x.copy(), np.ones_like(x)
        for j in range(2, n + 1):
            p0, p1, d1 = p1, ((2 * j - 1) * x * p1 - (j - 1) * p0) / j, j * p1 + x * d1
        w = 2.0 / ((1.0 - x * x) * d1 * d1)
        return x[::-1].copy(), w[::-1].copy()
    if grid == "lobatto":
        N = n - 1
        inner = np.sort(np.polynomial.legendre.Legendre.basis(N).deriv().roots().real)
        x = np.concatenate([[-1.0], inner, [1.0]])
        pn = np.polynomial.legendre.Legendre.basis(N)(x)
        w = 2.0 / (N * (N + 1) * pn * pn)
        return x[::-1].copy(), w[::-1].copy()
    if grid == "equiangular":
        # Clenshaw-Curtis on theta_j = pi j / N (poles included)
        N = n - 1
        th = np.pi * np.arange(n) / N
        w = np.zeros(n)
        for j in range(n):
            s = 0.0
            for k in range(1, N // 2 + 1):
                b = 1.0 if 2 * k == N else 2.0
                s += b / (4.0 * k * k - 1.0) * np.cos(2.0 * k * th[j])
            c = 1.0 if j in (0, N) else 2.0
            w[j] = c / N * (1.0 - s)
        return np.cos(th), w
    raise ValueError(grid)


def latlon_sht(f, lmax, mmax, grid):
    """f [..., nlat, nlon] real -> a [..., lmax, mmax] complex."""
    f = np.asarray(f, dtype=np.float64)
    nlat, nlon = f.shape[-2:]
    z, w = latlon_quadrature(grid, nlat)
    F = np.fft.rfft(f, axis=-1) * (2.0 * np.pi / nlon)  # [..., nlat, nlon/2+1]
    mk = min(mmax, F.shape[-1])
    a = np.zeros(f.shape[:-2] + (lmax, mmax), dtype=np.complex128)
    for m in range(mk):
        P = legendre_column(m, lmax, z)  # [lmax, nlat]
        a[..., :, m] = np.einsum("lj,...j->...l", P * w[None, :], F[..., :, m])
    return a


def latlon_isht(a, nlat, nlon, grid):
    """a [..., lmax, mmax] complex -> f [..., nlat, nlon] real."""
    a = np.asarray(a, dtype=np.complex128)
    lmax, mmax = a.shape[-2:]
    z, _ = latlon_quadrature(grid, nlat)
    X = np.zeros(a.shape[:-2] + (nlat, nlon // 2 + 1), dtype=np.complex128)
    for m in range(min(mmax, nlon // 2 + 1)):
        P = legendre_column(m, lmax, z)
        X[..., :, m] = np.einsum("lj,...l->...j", P, a[..., :, m])
    return np.fft.irfft(X, n=nlon, axis=-1) * nlon
