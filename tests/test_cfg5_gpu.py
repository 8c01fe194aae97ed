"""Training-style uses at full size: a weighted power-spectrum loss through the
SHT of 16 maps at nside 512 (L = M = 1023), and HEALPix 256 -> equiangular
512 x 1024 regridding (L = M = 511), both with backward.  Gradients are checked
as directional derivatives against FP64 central differences (rel 1e-6)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


def _dir_check(fn, x, v, eps):
    x = x.detach().requires_grad_(True)
    y = fn(x)
    y.backward()
    g = float((x.grad * v).sum())
    with torch.no_grad():
        fd = (float(fn(x + eps * v)) - float(fn(x - eps * v))) / (2 * eps)
    return g, fd


def test_power_spectrum_loss_nside512(hpx, cuda):
    nside, L = 512, 1023
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L)
    w = (1.0 / (torch.arange(L, device=cuda, dtype=torch.float64) + 1.0))[:, None]
    gen = torch.Generator(device=cuda)
    gen.manual_seed(5)
    f = torch.randn((16, 12 * nside * nside), generator=gen, device=cuda)
    # FP32 forward + backward at full size
    x = f.clone().requires_grad_(True)
    a = sht(x)
    loss = (w.float() * a.abs() ** 2).sum()
    loss.backward()
    assert torch.isfinite(x.grad).all() and x.grad.abs().max() > 0
    # FP64 directional derivative
    f64 = f[:2].double()
    v = torch.randn(f64.shape, generator=gen, device=cuda, dtype=torch.float64)
    g, fd = _dir_check(lambda y: (w * sht(y).abs() ** 2).sum(), f64, v, 1e-4)
    assert abs(g - fd) <= 1e-6 * abs(fd)


def test_regrid_healpix256_to_equiangular_backward(hpx, cuda):
    rg = hpx.Regridding(hpx.Grid("healpix", 256), hpx.Grid("equiangular", (512, 1024)), lmax=511, mmax=511)
    gen = torch.Generator(device=cuda)
    gen.manual_seed(6)
    f = torch.randn((2, 12 * 256 * 256), generator=gen, device=cuda)
    out = rg(f)
    assert out.shape == (2, 512, 1024)
    x = f.clone().requires_grad_(True)
    rg(x).pow(2).mean().backward()
    assert torch.isfinite(x.grad).all()
    f64 = f[:1].double()
    v = torch.randn(f64.shape, generator=gen, device=cuda, dtype=torch.float64)
    tgt = torch.randn((1, 512, 1024), generator=gen, device=cuda, dtype=torch.float64)
    g, fd = _dir_check(lambda y: ((rg(y) - tgt) ** 2).sum(), f64, v, 1e-3)
    assert abs(g - fd) <= 1e-6 * abs(fd)
