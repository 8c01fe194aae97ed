"""healpy a_lm packing on the GPU (``hpx_alm_to_healpy`` / ``hpx_healpy_to_alm``).

``SHTCUDA`` returns dense ``[..., lmax, mmax]`` coefficients with zeros for
m > l, as cuHPX does; healpy keeps the m <= l triangle in one vector per map,
order by order, at index ``m (2 lmax - 1 - m) / 2 + l`` (healpy's own lmax is
``lmax - 1``).  cuHPX states this map in
``tests/reproduce_difference_between_healpy_cuhpx.py:58-81``.  ``csphase``
multiplies order m by (-1)^m: the Condon-Shortley factor between this
library's phase convention (cuHPX's: no such factor) and healpy's.
"""

import ctypes

import torch

from . import _lib


def healpy_size(lmax, mmax=None):
    """Length of the packed vector for degrees l < lmax and orders m < min(mmax, lmax)."""
    M = min(lmax if mmax is None else mmax, lmax)
    return M * lmax - M * (M - 1) // 2


def healpy_index(lmax, l, m):
    """Position of (l, m) in the packed vector."""
    return m * (2 * lmax - 1 - m) // 2 + l


def _elem(dtype):
    if dtype == torch.complex64:
        return 8
    if dtype == torch.complex128:
        return 16
    raise ValueError("coefficients must be complex64 or complex128")


def alm_to_healpy(alm: torch.Tensor, csphase: bool = False) -> torch.Tensor:
    """Dense [..., lmax, mmax] complex CUDA tensor -> packed [..., healpy_size(lmax, mmax)]."""
    if not alm.is_cuda:
        raise ValueError("alm_to_healpy expects a CUDA tensor")
    lib = _lib.load()
    L, M = alm.shape[-2], alm.shape[-1]
    lead = alm.shape[:-2]
    x = alm.resolve_conj().reshape(-1, L, M).contiguous()
    out = torch.empty(x.shape[0], healpy_size(L, M), dtype=alm.dtype, device=alm.device)
    stream = torch.cuda.current_stream(alm.device).cuda_stream
    _lib.check(lib.hpx_alm_to_healpy(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), x.shape[0], L, M,
                                     _elem(alm.dtype), 1 if csphase else 0, ctypes.c_void_p(stream)))
    return out.reshape(*lead, out.shape[-1])


def healpy_to_alm(packed: torch.Tensor, lmax: int, mmax: int = None, csphase: bool = False) -> torch.Tensor:
    """Packed [..., healpy_size(lmax, mmax)] complex CUDA tensor -> dense [..., lmax, mmax] (zeros for m > l)."""
    if not packed.is_cuda:
        raise ValueError("healpy_to_alm expects a CUDA tensor")
    mmax = lmax if mmax is None else mmax
    n = healpy_size(lmax, mmax)
    if packed.shape[-1] != n:
        raise ValueError(f"packed length must be {n} for lmax={lmax}, mmax={mmax}, got {packed.shape[-1]}")
    lib = _lib.load()
    lead = packed.shape[:-1]
    x = packed.resolve_conj().reshape(-1, n).contiguous()
    out = torch.empty(x.shape[0], lmax, mmax, dtype=packed.dtype, device=packed.device)
    stream = torch.cuda.current_stream(packed.device).cuda_stream
    _lib.check(lib.hpx_healpy_to_alm(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), x.shape[0], lmax,
                                     mmax, _elem(packed.dtype), 1 if csphase else 0, ctypes.c_void_p(stream)))
    return out.reshape(*lead, lmax, mmax)
