"""``Grid`` and ``Regridding``: drop-ins for cuhpx/hpx_regrid.py:21-91.

``Regridding(src_grid, dest_grid, lmax=None, mmax=None, device=None,
enable_cuda=True).execute(f)`` = synthesis on the destination grid of the
analysis on the source grid, with the reference's rules for the default
lmax / mmax.  HEALPix sides use ``SHTCUDA`` / ``iSHTCUDA``; latitude-longitude
sides ('equiangular', 'legendre-gauss', 'lobatto') use this package's
``RealSHT`` / ``InverseRealSHT`` on the GPU instead of torch_harmonics.

Deliberate differences from the reference:

* the latitude-longitude transforms use the grid the ``Grid`` names (the
  reference constructs torch_harmonics transforms without passing it, so
  they always fall back to torch_harmonics' default grid);
* both transforms use one phase convention (no Condon-Shortley phase when a
  side is HEALPix, whose transforms carry none; the grids' own ``csphase``
  when both sides are latitude-longitude, where it cancels), so the result is
  the band-limited resampling of the input;
* there is no CPU path: ``enable_cuda=False`` raises.
"""

import torch

from .hpx_sht import SHTCUDA, iSHTCUDA
from .latlon import InverseRealSHT, RealSHT

LATLON = ("legendre-gauss", "lobatto", "equiangular")


class Grid:
    def __init__(self, grid, grid_size, norm="ortho", csphase=True):
        self.grid = grid
        self.nside = None
        self.nlat = None
        self.nlon = None
        self.norm = norm
        self.csphase = csphase
        if grid == "healpix":
            self.nside = grid_size
        elif grid in LATLON:
            self.nlat, self.nlon = grid_size
        else:
            raise ValueError("Unknown quadrature mode")


class Regridding(torch.nn.Module):
    def __init__(self, src_grid, dest_grid, lmax=None, mmax=None, device=None, enable_cuda=True, *,
                 precision="fp32", refine_iters=0):
        super().__init__()
        if not enable_cuda:
            raise NotImplementedError("hpx_b200 runs on the GPU only (enable_cuda=False selects the reference's CPU path)")
        self.lmax = lmax or self._determine_lmax(src_grid, dest_grid)
        self.mmax = mmax or self._determine_mmax(src_grid, dest_grid)
        self.device = device
        self.enable_cuda = enable_cuda
        hp = src_grid.grid == "healpix" or dest_grid.grid == "healpix"
        self.sht = self._sht(src_grid, hp, precision, refine_iters)
        self.isht = self._isht(dest_grid, hp, precision)

    @staticmethod
    def _determine_lmax(src_grid, dest_grid):
        src = 2 * src_grid.nside + 1 if src_grid.nside else src_grid.nlat
        dst = 2 * dest_grid.nside + 1 if dest_grid.nside else dest_grid.nlat
        return min(src, dst)

    @staticmethod
    def _determine_mmax(src_grid, dest_grid):
        src = 2 * src_grid.nside + 1 if src_grid.nside else src_grid.nlon // 2 + 1
        dst = 2 * dest_grid.nside + 1 if dest_grid.nside else dest_grid.nlon // 2 + 1
        return min(src, dst)

    def _sht(self, g, hp, precision, refine_iters):
        if g.grid == "healpix":
            return SHTCUDA(g.nside, lmax=self.lmax, mmax=self.mmax, norm=g.norm, csphase=g.csphase,
                           precision=precision, refine_iters=refine_iters)
        if g.grid in LATLON:
            return RealSHT(g.nlat, g.nlon, lmax=self.lmax, mmax=self.mmax, grid=g.grid, norm=g.norm,
                           csphase=False if hp else g.csphase, precision=precision, refine_iters=refine_iters)
        raise ValueError("Unknown quadrature mode")

    def _isht(self, g, hp, precision):
        if g.grid == "healpix":
            return iSHTCUDA(g.nside, lmax=self.lmax, mmax=self.mmax, norm=g.norm, csphase=g.csphase,
                            precision=precision)
        if g.grid in LATLON:
            return InverseRealSHT(g.nlat, g.nlon, lmax=self.lmax, mmax=self.mmax, grid=g.grid, norm=g.norm,
                                  csphase=False if hp else g.csphase, precision=precision)
        raise ValueError("Unknown quadrature mode")

    def execute(self, f):
        return self.isht(self.sht(f))

    def forward(self, f):
        return self.execute(f)
