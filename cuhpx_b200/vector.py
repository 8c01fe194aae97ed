"""Spin-1 (vector) transforms: drop-ins for cuHPX's ``VectorSHT`` / ``VectoriSHT``.

Mirrors cuhpx/hpx_sht.py:286-444: ``VectorSHTCUDA(nside, lmax=None,
mmax=None, grid="healpix", quad_weights="ring", norm="ortho", csphase=True)``
maps a real ``[..., 2, 12*nside**2]`` tangent field (two components) to
complex ``[..., 2, lmax, mmax]`` spheroidal and toroidal coefficients;
``VectoriSHTCUDA`` maps them back.  Defaults as the reference: ``lmax =
4*nside-1``, ``mmax = 2*nside+1``, ``csphase=True`` (odd orders negated).
float32 data run the FP32 path, float64 the FP64 path; the contractions run
in ``libhpx_b200.so`` (``hpx_vsht_*``) on a plan with one more degree and
order than the transform, which the derivative table needs.  Gradients are
the exact adjoints (the reference differentiates its einsums by autograd).
"""

import ctypes

import torch
import torch.nn as nn

from . import _lib
from .hpx_sht import get_plan


def _call(fn, plan, src, dst, batch, csphase):
    ws, nbytes = plan._ws(batch, src.device)
    stream = torch.cuda.current_stream(src.device).cuda_stream
    _lib.check(fn(plan._h, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), int(batch),
                  int(csphase), ctypes.c_void_p(ws.data_ptr()), nbytes, ctypes.c_void_p(stream)), plan._h)
    return dst


def _analysis(plan, x, L, M, csphase, adjoint=False):
    B = x.shape[0]
    out = torch.empty((B, 2, L, M), dtype=plan.cdtype, device=x.device)
    fn = plan._lib.hpx_vsht_inverse_adjoint if adjoint else plan._lib.hpx_vsht_forward
    _call(fn, plan, x, torch.view_as_real(out), B, csphase)
    return out


def _synthesis(plan, a, csphase, adjoint=False):
    B = a.shape[0]
    out = torch.empty((B, 2, plan.npix), dtype=plan.dtype, device=a.device)
    fn = plan._lib.hpx_vsht_forward_adjoint if adjoint else plan._lib.hpx_vsht_inverse
    _call(fn, plan, torch.view_as_real(a.resolve_conj().contiguous()), out, B, csphase)
    return out


class VectorSHTFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, plan, L, M, csphase):
        ctx.plan, ctx.csphase = plan, csphase
        return _analysis(plan, x, L, M, csphase)

    @staticmethod
    def backward(ctx, g):
        return _synthesis(ctx.plan, g.contiguous(), ctx.csphase, adjoint=True), None, None, None, None


class VectoriSHTFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, a, plan, L, M, csphase):
        ctx.plan, ctx.csphase, ctx.L, ctx.M = plan, csphase, L, M
        return _synthesis(plan, a, csphase)

    @staticmethod
    def backward(ctx, g):
        return _analysis(ctx.plan, g.contiguous(), ctx.L, ctx.M, ctx.csphase, adjoint=True), None, None, None, None


class _VBase(nn.Module):
    def __init__(self, nside, lmax, mmax, grid, quad_weights, norm, csphase):
        super().__init__()
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA device is not available. This class requires a GPU.")
        if grid != "healpix":
            raise ValueError("Unknown quadrature mode")
        self.nside = nside
        self.grid = grid
        self.norm = norm
        self.csphase = csphase
        self.nlat = 4 * nside - 1
        self.nlon = 4 * nside
        self.quad_weights = quad_weights
        self.lmax = lmax or self.nlat
        self.mmax = mmax or (self.nlon // 2 + 1)
        _lib.load()

    def _plan(self, dtype, device):
        prec = "fp64" if dtype in (torch.float64, torch.complex128) else "fp32"
        idx = device.index if device.index is not None else torch.cuda.current_device()
        return get_plan(self.nside, self.lmax + 1, self.mmax + 1, self.quad_weights, prec, idx)


class VectorSHTCUDA(_VBase):
    """[..., 2, npix] real -> [..., 2, lmax, mmax] complex (spheroidal, toroidal)."""

    def __init__(self, nside, lmax=None, mmax=None, grid="healpix", quad_weights="ring", norm="ortho", csphase=True,
                 use_bluestein=False):
        super().__init__(nside, lmax, mmax, grid, quad_weights, norm, csphase)

    def forward(self, x):
        if torch.is_complex(x):
            raise ValueError("Input tensor must be real.")
        if not x.is_cuda:
            raise ValueError("VectorSHTCUDA expects a CUDA tensor")
        if x.dtype not in (torch.float32, torch.float64):
            x = x.to(torch.float32)
        npix = 12 * self.nside * self.nside
        if x.dim() < 2 or x.shape[-2:] != (2, npix):
            raise ValueError(f"input must be [..., 2, {npix}], got {tuple(x.shape)}")
        lead = x.shape[:-2]
        xf = x.reshape(-1, 2, npix).contiguous()
        plan = self._plan(x.dtype, x.device)
        a = VectorSHTFunction.apply(xf, plan, self.lmax, self.mmax, self.csphase)
        return a.reshape(*lead, 2, self.lmax, self.mmax)


class VectoriSHTCUDA(_VBase):
    """[..., 2, lmax, mmax] complex -> [..., 2, npix] real."""

    def __init__(self, nside, lmax=None, mmax=None, grid="healpix", norm="ortho", csphase=True, use_bluestein=False):
        super().__init__(nside, lmax, mmax, grid, "ring", norm, csphase)

    def forward(self, a):
        if not a.is_cuda:
            raise ValueError("VectoriSHTCUDA expects a CUDA tensor")
        if not torch.is_complex(a):
            raise ValueError("Input tensor must be complex [..., 2, lmax, mmax].")
        if a.dtype not in (torch.complex64, torch.complex128):
            a = a.to(torch.complex64)
        if a.dim() < 3 or a.shape[-3:] != (2, self.lmax, self.mmax):
            raise ValueError(f"input must be [..., 2, {self.lmax}, {self.mmax}], got {tuple(a.shape)}")
        lead = a.shape[:-3]
        af = a.reshape(-1, 2, self.lmax, self.mmax).contiguous()
        plan = self._plan(a.dtype, a.device)
        f = VectoriSHTFunction.apply(af, plan, self.lmax, self.mmax, self.csphase)
        return f.reshape(*lead, 2, f.shape[-1])
