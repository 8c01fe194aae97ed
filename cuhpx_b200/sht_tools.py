"""HEALPix ring quadrature weights on the host.

The ``'ring'`` weights of cuHPX's ``cuhpx/sht_tools.py:34-44`` come from the
HEALPix FITS tables; here they are read from ``data/ring_weights.npz``
(converted once from those tables by ``data/make_ring_weights.py``), so
astropy is not needed.  The ring geometry itself lives in the CUDA plan.
"""

import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "ring_weights.npz")
_cache = {}


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
