"""Spherical-harmonic transforms on latitude-longitude grids, on the GPU.

cuHPX's ``Regridding`` (cuhpx/hpx_regrid.py:21-91) hands these grids to
``torch_harmonics.RealSHT`` / ``InverseRealSHT``.  ``RealSHT`` and
``InverseRealSHT`` here take the same arguments (``nlat, nlon, lmax=None,
mmax=None, grid="equiangular", norm="ortho", csphase=True``) and run on the
hpx_b200 library (``hpx_plan_create_latlon``): the same ring FFTs and
Legendre contraction kernels as the HEALPix transforms, over nlat rings of
nlon samples, with quadrature

* ``"equiangular"``: theta_j = pi j / (nlat - 1), poles included, Clenshaw-Curtis weights;
* ``"legendre-gauss"``: Gauss-Legendre nodes and weights;
* ``"lobatto"``: Gauss-Lobatto nodes and weights (poles included).

Layouts: maps ``[..., nlat, nlon]`` (north to south, phi_k = 2 pi k / nlon),
coefficients ``[..., lmax, mmax]`` complex, as torch_harmonics.  Analysis is
a_lm = sum_j w_j Pbar_l^m(cos theta_j) (2 pi / nlon) sum_k f_jk e^{-i m phi_k}
with the orthonormal Pbar; ``csphase=True`` multiplies the coefficients by
the Condon-Shortley phase (-1)^m (the HEALPix transforms, like cuHPX's CUDA
path, carry none).  Only ``norm="ortho"`` is provided.  Gradients are the
exact adjoints, as for ``SHTCUDA``.
"""

import torch
import torch.nn as nn

from . import _lib
from .hpx_sht import SHTFunction, _device_index, get_latlon_plan, iSHTFunction


def default_lmax(nlat, grid):
    return nlat - 1 if grid == "lobatto" else nlat


class _LatLonBase(nn.Module):
    def __init__(self, nlat, nlon, lmax, mmax, grid, norm, csphase, precision, refine_iters, batch_chunk,
                 legendre_table):
        super().__init__()
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA device is not available. This class requires a GPU.")
        if grid not in _lib.GRIDS:
            raise ValueError(f"unknown grid {grid!r}; expected one of {sorted(_lib.GRIDS)}")
        if norm != "ortho":
            raise NotImplementedError("only norm='ortho' is provided")
        if precision not in ("fp32", "bf16x3", "f16x3"):
            raise ValueError("precision must be 'fp32', 'f16x3' or 'bf16x3' (float64 data select fp64 automatically)")
        self.nlat, self.nlon, self.grid = int(nlat), int(nlon), grid
        self.lmax = int(lmax or default_lmax(self.nlat, grid))
        self.mmax = int(mmax or (self.nlon // 2 + 1))
        self.norm, self.csphase = norm, bool(csphase)
        self.precision = precision
        self.refine_iters = int(refine_iters)
        self.batch_chunk = int(batch_chunk)
        self.legendre_table = bool(legendre_table)
        _lib.load()

    def _plan(self, dtype, device_index):
        prec = "fp64" if dtype == torch.float64 else self.precision
        return get_latlon_plan(self.nlat, self.nlon, self.lmax, self.mmax, self.grid, prec, device_index,
                               self.batch_chunk, self.legendre_table)

    def _phase(self, a):
        if not self.csphase:
            return a
        sign = 1.0 - 2.0 * (torch.arange(self.mmax, device=a.device) & 1).to(a.real.dtype)
        return a * sign


class RealSHT(_LatLonBase):
    """Analysis: real ``[..., nlat, nlon]`` -> complex ``[..., lmax, mmax]``."""

    def __init__(self, nlat, nlon, lmax=None, mmax=None, grid="equiangular", norm="ortho", csphase=True, *,
                 precision="fp32", refine_iters=0, batch_chunk=64, legendre_table=True):
        super().__init__(nlat, nlon, lmax, mmax, grid, norm, csphase, precision, refine_iters, batch_chunk,
                         legendre_table)

    def forward(self, x):
        if torch.is_complex(x):
            raise ValueError("Input tensor must be real.")
        if not x.is_cuda:
            raise ValueError("RealSHT expects a CUDA tensor")
        if tuple(x.shape[-2:]) != (self.nlat, self.nlon):
            raise ValueError(f"trailing dimensions must be (nlat, nlon)=({self.nlat}, {self.nlon})")
        if x.dtype not in (torch.float32, torch.float64):
            x = x.to(torch.float32)
        lead = x.shape[:-2]
        xf = x.reshape(-1, self.nlat * self.nlon).contiguous()
        plan = self._plan(x.dtype, _device_index(x))
        a = SHTFunction.apply(xf, plan, self.refine_iters)
        return self._phase(a.reshape(*lead, self.lmax, self.mmax))


class InverseRealSHT(_LatLonBase):
    """Synthesis: complex ``[..., lmax, mmax]`` -> real ``[..., nlat, nlon]``."""

    def __init__(self, nlat, nlon, lmax=None, mmax=None, grid="equiangular", norm="ortho", csphase=True, *,
                 precision="fp32", batch_chunk=64, legendre_table=True):
        super().__init__(nlat, nlon, lmax, mmax, grid, norm, csphase, precision, 0, batch_chunk, legendre_table)

    def forward(self, a):
        if not a.is_cuda:
            raise ValueError("InverseRealSHT expects a CUDA tensor")
        if not torch.is_complex(a):
            raise ValueError("Input tensor must be complex [..., lmax, mmax].")
        if tuple(a.shape[-2:]) != (self.lmax, self.mmax):
            raise ValueError(f"trailing dimensions must be (lmax, mmax)=({self.lmax}, {self.mmax})")
        if a.dtype not in (torch.complex64, torch.complex128):
            a = a.to(torch.complex64)
        lead = a.shape[:-2]
        af = self._phase(a).reshape(-1, self.lmax, self.mmax).contiguous()
        dt = torch.float64 if af.dtype == torch.complex128 else torch.float32
        plan = self._plan(dt, _device_index(a))
        f = iSHTFunction.apply(af, plan)
        return f.reshape(*lead, self.nlat, self.nlon)
