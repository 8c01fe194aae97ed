"""Host-side HEALPix ring geometry and quadrature weights.

Same functions and conventions as cuHPX's ``cuhpx/sht_tools.py`` (ring
numbering north to south, ``'ring'`` weights from the HEALPix FITS tables),
written for this package: the weights come from ``data/ring_weights.npz``
(converted once from the FITS tables by ``data/make_ring_weights.py``), so
astropy is not needed.
"""

import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "ring_weights.npz")
_cache = {}


def nrings(nside):
    return 4 * nside - 1


def npix(nside):
    return 12 * nside * nside


def read_ring_weight(nside):
    """The 2*nside ring-weight corrections of HEALPix (cuhpx/sht_tools.py:34-44)."""
    if nside not in _cache:
        with np.load(_DATA) as d:
            key = f"n{nside}"
            if key not in d:
                avail = sorted(int(k[1:]) for k in d.files)
                raise ValueError(f"no 'ring' quadrature weights for nside={nside}; available: {avail}")
            _cache[nside] = np.array(d[key], dtype=np.float64)
    return _cache[nside]


def healpix_weights(nside, quad_weights="ring"):
    """(z, w): cos(theta) of each ring (south to north, as the reference returns it)
    and the per-ring quadrature weights (cuhpx/sht_tools.py:114-140)."""
    t = np.arange(4 * nside - 1)
    z = np.zeros(t.shape)
    m1 = t < nside - 1
    m2 = (t >= nside - 1) & (t <= 3 * nside - 1)
    m3 = t > 3 * nside - 1
    z[m1] = 1 - ((t[m1] + 1) ** 2) / (3 * nside**2)
    z[m2] = 4 / 3 - 2 * (t[m2] + 1) / (3 * nside)
    z[m3] = ((4 * nside - 1 - t[m3]) ** 2) / (3 * nside**2) - 1
    if quad_weights == "ring":
        corr = read_ring_weight(nside)
        north = np.where(t + 1 > 2 * nside, 4 * nside - (t + 1), t + 1)
        w = 4.0 * np.pi / npix(nside) * (1.0 + corr[north - 1])
    else:
        w = np.full(t.shape, 4.0 * np.pi / npix(nside))
    return np.flip(z).copy(), w


def nphi_ring(t, nside):
    if 0 <= t < nside - 1:
        return 4 * (t + 1)
    if nside - 1 <= t <= 3 * nside - 1:
        return 4 * nside
    if 3 * nside - 1 < t <= 4 * nside - 2:
        return 4 * (4 * nside - t - 1)
    raise ValueError(f"Ring t={t} not contained by nside={nside}")


def cumulative_nphi_ring(t, nside):
    if 0 <= t < nside:
        return 2 * t * (t + 1)
    if t < 3 * nside:
        return 2 * nside * (nside + 1) + (t - nside) * 4 * nside
    if t < 4 * nside:
        r = 4 * nside - t - 1
        return 12 * nside * nside - 2 * r * (r + 1)
    return -1


def p2phi_ring(t, p, nside):
    shift = 0.5
    if nside <= t + 1 <= 3 * nside:
        shift *= (t - nside + 2) % 2
        return np.pi / (2 * nside) * (p + shift)
    if t + 1 > 3 * nside:
        return np.pi / (2 * (4 * nside - t - 1)) * (p + shift)
    return np.pi / (2 * (t + 1)) * (p + shift)
