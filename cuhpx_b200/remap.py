"""HEALPix pixel-order remapping on the GPU: RING, NEST and per-face flat (XY).

Drop-in for cuHPX's ``cuhpx/hpx_remap.py:24-102`` (``ring2nest``,
``nest2ring``, ``nest2flat``, ``flat2nest``, ``ring2flat``, ``flat2ring``,
``flat2flat``), with the same arguments, results and errors:

* ``nside`` not a power of two -> ``ValueError("nside must be a power of two")``;
* last dimension not ``12 * nside**2`` -> ``RuntimeError`` (the reference's
  ``TORCH_CHECK`` in ``src/data_remapping/hpx_remapping.cpp:21-239``);
* an origin other than "S", "E", "N", "W" -> ``RuntimeError``.

A 1-D tensor is one map; any leading dimensions are a batch of maps, remapped
in one call.  Every dtype is accepted (the bytes are moved, not read).  The
result is a new tensor of the input's shape, computed on the current CUDA
stream by ``hpx_remap`` of ``libhpx_b200.so``, which allocates nothing beyond
it.  There is no CPU fallback: a CPU tensor raises.
"""

import ctypes

import torch

from . import _lib

RING, NEST, XY = 0, 1, 2
_ORIGINS = {"S": 0, "E": 1, "N": 2, "W": 3}


def is_power_of_two(n):
    return (n > 0) and (n & (n - 1)) == 0


def _origin(origin, what="The origin"):
    if origin not in _ORIGINS:
        raise RuntimeError(f"{what} must be one from S, E, N, W. Stop")
    return _ORIGINS[origin]


def remap(data: torch.Tensor, nside: int, src=(RING, 0, False), dst=(NEST, 0, False)) -> torch.Tensor:
    """Remap ``data[..., 12*nside**2]`` from layout ``src`` to layout ``dst``.

    A layout is ``(order, origin, clockwise)`` with order RING, NEST or XY;
    origin (0..3 = S, E, N, W) and clockwise only matter for XY.
    """
    if not is_power_of_two(nside):
        raise ValueError("nside must be a power of two")
    if not isinstance(data, torch.Tensor) or not data.is_cuda:
        raise RuntimeError("hpx_b200 remapping needs a CUDA tensor (there is no CPU path)")
    npix = 12 * nside * nside
    if data.dim() == 0 or data.size(-1) != npix:
        raise RuntimeError("The number of elements in the input array is not equal to the number of HEALPix grid "
                           "at current nside. Stop.")
    x = data.contiguous()
    out = torch.empty_like(x)
    batch = x.numel() // npix
    lib = _lib.load()
    with torch.cuda.device(x.device):
        stream = torch.cuda.current_stream(x.device).cuda_stream
        st = lib.hpx_remap(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(out.data_ptr()), int(batch), int(nside),
                           int(x.element_size()), int(src[0]), int(src[1]), int(bool(src[2])), int(dst[0]),
                           int(dst[1]), int(bool(dst[2])), ctypes.c_void_p(stream))
    _lib.check(st)
    return out


def _power_of_two(nside):
    if not is_power_of_two(nside):
        raise ValueError("nside must be a power of two")


def ring2nest(data: torch.Tensor, nside: int) -> torch.Tensor:
    return remap(data, nside, (RING, 0, False), (NEST, 0, False))


def nest2ring(data: torch.Tensor, nside: int) -> torch.Tensor:
    return remap(data, nside, (NEST, 0, False), (RING, 0, False))


def nest2flat(data: torch.Tensor, origin: str, clockwise: bool, nside: int) -> torch.Tensor:
    _power_of_two(nside)
    return remap(data, nside, (NEST, 0, False), (XY, _origin(origin), clockwise))


def flat2nest(data: torch.Tensor, origin: str, clockwise: bool, nside: int) -> torch.Tensor:
    _power_of_two(nside)
    return remap(data, nside, (XY, _origin(origin), clockwise), (NEST, 0, False))


def ring2flat(data: torch.Tensor, origin: str, clockwise: bool, nside: int) -> torch.Tensor:
    _power_of_two(nside)
    return remap(data, nside, (RING, 0, False), (XY, _origin(origin), clockwise))


def flat2ring(data: torch.Tensor, origin: str, clockwise: bool, nside: int) -> torch.Tensor:
    _power_of_two(nside)
    return remap(data, nside, (XY, _origin(origin), clockwise), (RING, 0, False))


def flat2flat(data: torch.Tensor, src_origin: str, src_clockwise: bool, dest_origin: str, dest_clockwise: bool,
              nside: int) -> torch.Tensor:
    _power_of_two(nside)
    so = _origin(src_origin, "The src origin")
    do = _origin(dest_origin, "The dest origin")
    return remap(data, nside, (XY, so, src_clockwise), (XY, do, dest_clockwise))
