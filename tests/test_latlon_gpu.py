"""Latitude-longitude transforms (RealSHT / InverseRealSHT) and Regridding on the GPU,
against the latitude-longitude oracle and the HEALPix oracle.

Tolerances (rel-L2): FP32 paths 1e-5, FP64 1e-10, f16x3 2e-6, bf16x3 3e-5.
"""

import numpy as np
import pytest
import torch

from oracle import hpx_oracle as O
from oracle import latlon_oracle as LO

pytestmark = pytest.mark.gpu

GRIDS = ["equiangular", "legendre-gauss", "lobatto"]
TOL = {"fp32": 1e-5, "f16x3": 2e-6, "bf16x3": 3e-5}


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rand_alm(rng, L, M, batch=(), nlon=None):
    a = rng.standard_normal(batch + (L, M)) + 1j * rng.standard_normal(batch + (L, M))
    a = np.where(np.arange(M)[None, :] <= np.arange(L)[:, None], a, 0)
    a[..., 0] = a[..., 0].real
    if nlon is not None and M > nlon // 2:
        a[..., nlon // 2] = a[..., nlon // 2].real
    return a


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


# nlon = 36 and 90 give non-power-of-two rings (Bluestein kernel only; h = 45 is odd)
CASES = [(16, 32, None, None), (17, 32, 12, 10), (33, 64, None, None), (64, 128, 48, 40), (8, 16, 12, 12),
         (18, 36, None, None), (45, 90, 30, 28)]


@pytest.mark.parametrize("grid", GRIDS)
@pytest.mark.parametrize("nlat,nlon,L,M", CASES)
def test_latlon_forward_inverse(hpx, cuda, grid, nlat, nlon, L, M):
    rng = np.random.default_rng(nlat * 7 + nlon)
    sht = hpx.RealSHT(nlat, nlon, lmax=L, mmax=M, grid=grid, csphase=False)
    L, M = sht.lmax, sht.mmax
    f = rng.standard_normal((3, nlat, nlon))
    a = sht(torch.from_numpy(f).float().to(cuda))
    assert a.shape == (3, L, M)
    assert rel(a, LO.latlon_sht(f, L, M, grid)) < 1e-5
    a64 = sht(torch.from_numpy(f).to(cuda))
    assert a64.dtype == torch.complex128
    assert rel(a64, LO.latlon_sht(f, L, M, grid)) < 1e-10
    alm = rand_alm(rng, L, M, (2,), nlon)
    isht = hpx.InverseRealSHT(nlat, nlon, lmax=L, mmax=M, grid=grid, csphase=False)
    g = isht(torch.from_numpy(alm).to(torch.complex64).to(cuda))
    assert g.shape == (2, nlat, nlon)
    assert rel(g, LO.latlon_isht(alm, nlat, nlon, grid)) < 1e-5
    g64 = isht(torch.from_numpy(alm).to(cuda))
    assert rel(g64, LO.latlon_isht(alm, nlat, nlon, grid)) < 1e-10


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
@pytest.mark.parametrize("grid", GRIDS)
def test_latlon_tensor_cores(hpx, cuda, prec, grid):
    rng = np.random.default_rng(3)
    nlat, nlon = 96, 192
    f = rng.standard_normal((4, nlat, nlon))
    sht = hpx.RealSHT(nlat, nlon, grid=grid, csphase=False, precision=prec)
    a = sht(torch.from_numpy(f).float().to(cuda))
    assert rel(a, LO.latlon_sht(f, sht.lmax, sht.mmax, grid)) < TOL[prec]
    alm = rand_alm(rng, sht.lmax, sht.mmax, (4,), nlon)
    g = hpx.InverseRealSHT(nlat, nlon, grid=grid, csphase=False, precision=prec)(
        torch.from_numpy(alm).to(torch.complex64).to(cuda))
    assert rel(g, LO.latlon_isht(alm, nlat, nlon, grid)) < TOL[prec]


def test_gauss_round_trip_exact(hpx, cuda):
    rng = np.random.default_rng(5)
    nlat, nlon = 40, 80
    alm = rand_alm(rng, nlat, nlon // 2 + 1, (2,), nlon)
    a = torch.from_numpy(alm).to(cuda)
    f = hpx.InverseRealSHT(nlat, nlon, grid="legendre-gauss")(a)
    b = hpx.RealSHT(nlat, nlon, grid="legendre-gauss")(f)
    assert rel(b, alm) < 1e-12


def test_csphase(hpx, cuda):
    rng = np.random.default_rng(6)
    f = torch.from_numpy(rng.standard_normal((2, 16, 32))).to(cuda)
    a0 = hpx.RealSHT(16, 32, csphase=False)(f)
    a1 = hpx.RealSHT(16, 32, csphase=True)(f)
    sign = torch.tensor([(-1.0) ** m for m in range(a0.shape[-1])], device=cuda)
    assert torch.allclose(a1, a0 * sign)
    g0 = hpx.InverseRealSHT(16, 32, csphase=False)(a0)
    g1 = hpx.InverseRealSHT(16, 32, csphase=True)(a1)
    assert torch.allclose(g0, g1)


def test_latlon_gradients(hpx, cuda):
    """<SHT f, a> and <f, SHT^T a> agree (exact adjoint), FP64."""
    rng = np.random.default_rng(8)
    nlat, nlon = 12, 24
    sht = hpx.RealSHT(nlat, nlon, grid="equiangular", csphase=False)
    f = torch.from_numpy(rng.standard_normal((2, nlat, nlon))).to(cuda).requires_grad_(True)
    c = torch.from_numpy(rand_alm(rng, sht.lmax, sht.mmax, (2,))).to(cuda)
    out = sht(f)
    loss = (out.conj() * c).real.sum()
    loss.backward()
    lhs = loss.item()
    rhs = float((f.detach() * f.grad).sum())
    assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs))


def test_latlon_errors(hpx, cuda):
    with pytest.raises(ValueError):
        hpx.RealSHT(16, 32, grid="gauss")
    with pytest.raises(NotImplementedError):
        hpx.RealSHT(16, 32, norm="schmidt")
    sht = hpx.RealSHT(16, 32)
    with pytest.raises(ValueError):
        sht(torch.zeros(2, 16, 31, device=cuda))


@pytest.mark.parametrize("dest", ["legendre-gauss", "equiangular"])
def test_regrid_healpix_to_latlon(hpx, cuda, dest):
    """Regridding = the oracle's HEALPix analysis followed by its lat-lon synthesis."""
    rng = np.random.default_rng(9)
    nside, nlat, nlon = 16, 48, 96
    src = hpx.Grid("healpix", nside)
    dst = hpx.Grid(dest, (nlat, nlon))
    rg = hpx.Regridding(src, dst)
    assert (rg.lmax, rg.mmax) == (2 * nside + 1, 2 * nside + 1)
    f = rng.standard_normal((2, 12 * nside * nside))
    out = rg.execute(torch.from_numpy(f).float().to(cuda))
    assert out.shape == (2, nlat, nlon)
    ref = LO.latlon_isht(O.sht(f, nside, rg.lmax, rg.mmax), nlat, nlon, dest)
    assert rel(out, ref) < 1e-5


def test_regrid_band_limited_field(hpx, cuda):
    """A band-limited HEALPix field regridded with Jacobi-refined analysis equals
    the same field synthesised directly on the Gauss grid."""
    rng = np.random.default_rng(10)
    nside, nlat, nlon, L = 32, 40, 80, 25
    alm = rand_alm(rng, L, L, (2,))
    f = O.isht(alm, nside)
    rg = hpx.Regridding(hpx.Grid("healpix", nside), hpx.Grid("legendre-gauss", (nlat, nlon)), lmax=L, mmax=L,
                        refine_iters=4)
    out = rg.execute(torch.from_numpy(f).to(cuda))
    assert rel(out, LO.latlon_isht(alm, nlat, nlon, "legendre-gauss")) < 1e-6


def test_regrid_latlon_to_healpix_and_backward(hpx, cuda):
    rng = np.random.default_rng(11)
    nlat, nlon, nside = 33, 64, 8
    rg = hpx.Regridding(hpx.Grid("equiangular", (nlat, nlon)), hpx.Grid("healpix", nside))
    f = torch.from_numpy(rng.standard_normal((2, nlat, nlon))).to(cuda).requires_grad_(True)
    out = rg(f)
    assert out.shape == (2, 12 * nside * nside)
    ref = O.isht(LO.latlon_sht(f.detach().cpu().numpy(), rg.lmax, rg.mmax, "equiangular"), nside)
    assert rel(out, ref) < 1e-10
    out.pow(2).sum().backward()
    assert f.grad is not None and torch.isfinite(f.grad).all()


def test_regrid_latlon_to_latlon(hpx, cuda):
    rng = np.random.default_rng(12)
    src = hpx.Grid("legendre-gauss", (24, 48))
    dst = hpx.Grid("lobatto", (31, 62))
    rg = hpx.Regridding(src, dst)
    f = rng.standard_normal((1, 24, 48))
    out = rg.execute(torch.from_numpy(f).float().to(cuda))
    ref = LO.latlon_isht(LO.latlon_sht(f, rg.lmax, rg.mmax, "legendre-gauss"), 31, 62, "lobatto")
    assert rel(out, ref) < 1e-5


def test_regrid_cpu_path_refused(hpx, cuda):
    with pytest.raises(NotImplementedError):
        hpx.Regridding(hpx.Grid("healpix", 8), hpx.Grid("equiangular", (16, 32)), enable_cuda=False)
