"""CPU oracle of the healpy a_lm packing -- TEST INFRASTRUCTURE ONLY.

cuHPX's coefficients are dense ``[..., L, M]`` (zeros for m > l); healpy packs
the m <= l triangle into one vector, order by order (all degrees of m = 0,
then of m = 1, ...).  The reference states the index map in
``tests/reproduce_difference_between_healpy_cuhpx.py:58-81``:

  hp_getidx(L, l, m) = m (2L - 1 - m) / 2 + l        (L = healpy lmax + 1)
  flm_hp_to_2d: [L, 2L-1] with column L-1+m = packed[hp_getidx(L, l, m)] and
                column L-1-m = (-1)^m conj(column L-1+m)

restated here (``tests/golden/make_healpy_golden.py`` ran the reference's own
functions to pin it).  The reference compares magnitudes with healpy only; the
(-1)^m Condon-Shortley factor between cuHPX's phase convention and healpy's
is the ``csphase`` option here, and its sign is unpinned (healpy is not
installed).
"""

import numpy as np


def hp_index(L, l, m):
    """tests/reproduce_difference_between_healpy_cuhpx.py:62-64 (hp_getidx)."""
    return m * (2 * L - 1 - m) // 2 + l


def packed_size(L, M):
    """Entries of the packed vector for degrees l < L and orders m < min(M, L)."""
    M = min(M, L)
    return M * L - M * (M - 1) // 2


def alm_to_healpy(alm, csphase=False):
    """Dense [..., L, M] -> packed [..., packed_size(L, M)] (entries m <= l)."""
    alm = np.asarray(alm)
    L, M = alm.shape[-2], alm.shape[-1]
    out = np.zeros(alm.shape[:-2] + (packed_size(L, M),), dtype=alm.dtype)
    for m in range(min(M, L)):
        s = -1.0 if (csphase and m & 1) else 1.0
        for l in range(m, L):
            out[..., hp_index(L, l, m)] = s * alm[..., l, m]
    return out


def healpy_to_alm(packed, L, M, csphase=False):
    """Packed [..., packed_size(L, M)] -> dense [..., L, M] with zeros for m > l."""
    packed = np.asarray(packed)
    out = np.zeros(packed.shape[:-1] + (L, M), dtype=packed.dtype)
    for m in range(min(M, L)):
        s = -1.0 if (csphase and m & 1) else 1.0
        for l in range(m, L):
            out[..., l, m] = s * packed[..., hp_index(L, l, m)]
    return out


def healpy_to_flm2d(packed, L):
    """tests/reproduce_difference_between_healpy_cuhpx.py:67-81 (flm_hp_to_2d): [L, 2L-1]."""
    packed = np.asarray(packed)
    out = np.zeros((L, 2 * L - 1), dtype=np.complex128)
    for l in range(L):
        out[l, L - 1] = packed[hp_index(L, l, 0)]
        for m in range(1, l + 1):
            out[l, L - 1 + m] = packed[hp_index(L, l, m)]
            out[l, L - 1 - m] = (-1) ** m * np.conj(out[l, L - 1 + m])
    return out
