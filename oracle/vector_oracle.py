"""CPU oracle of the spin-1 (vector) HEALPix transforms -- TEST INFRASTRUCTURE ONLY.

Restates in float64 numpy cuHPX's ``VectorSHT`` / ``VectoriSHT``
(cuhpx/hpx_sht.py:286-444) and their table ``_precompute_dlegpoly``
(cuhpx/sht_tools.py:267-304); ``tests/test_oracle_vector.py`` pins it to
golden vectors that ``tests/golden/make_vector_golden.py`` produced by
running the reference's own classes.

A vector map is ``[..., 2, npix]`` (two real components); coefficients are
``[..., 2, L, M]`` complex (spheroidal, toroidal).  With D0, D1 the two rows
of the table (D0: theta-derivative combination of Pbar_l^{m-1} and
Pbar_l^{m+1}; D1: m Pbar_l^m / sin(theta) from Pbar_{l+1}^{m-1} and
Pbar_{l+1}^{m+1}; rows of odd m negated when ``csphase``), weights w_t and
nf_l = 1 / (l (l+1)) (nf_0 = 1), the reference's four einsums per
component amount to, for ring spectra x0, x1 and sums over rings t,

  S_lm = nf_l sum_t w_t (D0 x0 - i D1 x1)      T_lm = nf_l sum_t w_t (-D0 x1 - i D1 x0)

and the synthesis of (S, T) to ring spectra

  s_tm = sum_l (D0 S + i D1 T)                 t_tm = sum_l (-D0 T + i D1 S)
"""

import numpy as np

from . import hpx_oracle as O


def dlegendre(mmax, lmax, x, csphase=True):
    """dpct[2, M, L, K] of cuhpx/sht_tools.py:267-304 (same terms, same order)."""
    pct = O.legendre_table(mmax + 1, lmax + 1, x)
    dpct = np.zeros((2, mmax, lmax, len(x)), dtype=np.float64)
    for l in range(0, lmax):
        dpct[0, 0, l] = -np.sqrt(l * (l + 1)) * pct[1, l]
        for m in range(1, min(l, mmax)):
            dpct[0, m, l] = 0.5 * (
                np.sqrt((l + m) * (l - m + 1)) * pct[m - 1, l] - np.sqrt((l - m) * (l + m + 1)) * pct[m + 1, l]
            )
        if mmax > l:
            # m == l (the reference indexes pct[l - 1] with l = 0 too: a zero times the last row)
            dpct[0, l, l] = np.sqrt(l / 2) * pct[l - 1, l]
        for m in range(1, min(l + 1, mmax)):
            dpct[1, m, l] = (
                0.5
                * np.sqrt((2 * l + 1) / (2 * l + 3))
                * (np.sqrt((l - m + 1) * (l - m + 2)) * pct[m - 1, l + 1] + np.sqrt((l + m + 1) * (l + m + 2)) * pct[m + 1, l + 1])
            )
    if csphase:
        for m in range(1, mmax, 2):
            dpct[:, m] *= -1
    return dpct


def _ein(x, w):
    """'...km,mlk->...lm' (cuhpx/hpx_sht.py:357-378)"""
    return np.einsum("...km,mlk->...lm", x, w)


def _ein_inv(a, w):
    """'...lm,mlk->...km' (cuhpx/hpx_sht.py:409-427)"""
    return np.einsum("...lm,mlk->...km", a, w)


def vsht(f, nside, lmax, mmax, quad_weights="ring", csphase=True):
    """VectorSHT.forward: [..., 2, npix] real -> [..., 2, L, M] complex (cuhpx/hpx_sht.py:286-378)."""
    f = np.asarray(f, dtype=np.float64)
    L, M = lmax, mmax
    x = np.cos(O.ring_theta(nside))
    w = O.ring_weights(nside, quad_weights)
    dpct = dlegendre(M, L, x, csphase)
    l = np.arange(L, dtype=np.float64)
    with np.errstate(divide="ignore"):
        nf = 1.0 / l / (l + 1)
    nf[0] = 1.0
    W = np.einsum("dmlk,k,l->dmlk", dpct, w, nf)
    W[1] = -W[1]
    F = O.ring_rfft(f, M, nside)  # [..., 2, R, M]
    x0r, x0i = F[..., 0, :, :].real, F[..., 0, :, :].imag
    x1r, x1i = F[..., 1, :, :].real, F[..., 1, :, :].imag
    out = np.zeros(f.shape[:-2] + (2, L, M), dtype=np.complex128)
    out[..., 0, :, :] = (_ein(x0r, W[0]) - _ein(x1i, W[1])) + 1j * (_ein(x0i, W[0]) + _ein(x1r, W[1]))
    out[..., 1, :, :] = (-_ein(x0i, W[1]) - _ein(x1r, W[0])) + 1j * (_ein(x0r, W[1]) - _ein(x1i, W[0]))
    return out


def visht(a, nside, csphase=True):
    """VectoriSHT.forward: [..., 2, L, M] complex -> [..., 2, npix] real (cuhpx/hpx_sht.py:381-444)."""
    a = np.asarray(a, dtype=np.complex128)
    L, M = a.shape[-2], a.shape[-1]
    x = np.cos(O.ring_theta(nside))
    D = dlegendre(M, L, x, csphase)
    a0r, a0i = a[..., 0, :, :].real, a[..., 0, :, :].imag
    a1r, a1i = a[..., 1, :, :].real, a[..., 1, :, :].imag
    s = (_ein_inv(a0r, D[0]) - _ein_inv(a1i, D[1])) + 1j * (_ein_inv(a0i, D[0]) + _ein_inv(a1r, D[1]))
    t = (-_ein_inv(a0i, D[1]) - _ein_inv(a1r, D[0])) + 1j * (_ein_inv(a0r, D[1]) - _ein_inv(a1i, D[0]))
    ftm = np.stack((s, t), axis=-3)  # [..., 2, R, M]
    return O.ring_irfft(ftm, M, nside)
