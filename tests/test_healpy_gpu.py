"""healpy a_lm packing through the C ABI: bit-exact against the oracle."""

import numpy as np
import pytest
import torch

from oracle import healpy_oracle as H

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L,M", [(1, 1), (7, 7), (33, 33), (65, 17), (17, 40), (300, 300), (2047, 2047)])
@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_pack_and_unpack_vs_oracle(cuda, L, M, dtype):
    import cuhpx_b200 as hpx

    rng = np.random.default_rng(L + M)
    B = 3 if L < 1000 else 1
    a = rng.standard_normal((B, L, M)) + 1j * rng.standard_normal((B, L, M))
    a = np.where(np.arange(M)[None, None, :] <= np.arange(L)[None, :, None], a, 0)
    at = torch.from_numpy(a).to(cuda, dtype)
    host = at.cpu().numpy()
    for cs in (False, True):
        p = hpx.alm_to_healpy(at, csphase=cs)
        assert p.shape == (B, hpx.healpy_size(L, M)) and p.dtype == dtype
        want = H.alm_to_healpy(host, cs) if L < 1000 else None
        if want is not None:
            assert np.array_equal(p.cpu().numpy(), want)
        back = hpx.healpy_to_alm(p, L, M, csphase=cs)
        assert torch.equal(back, at)
    # entries are where the reference's index map puts them
    p = hpx.alm_to_healpy(at).cpu().numpy()
    for l, m in [(0, 0), (L - 1, 0), (L - 1, min(M, L) - 1), (L // 2, min(M, L) // 3)]:
        if m <= l:
            assert p[0, hpx.healpy_index(L, l, m)] == host[0, l, m]


def test_unpack_writes_zeros_everywhere_else(cuda):
    import cuhpx_b200 as hpx

    L, M = 40, 50
    p = torch.randn(2, hpx.healpy_size(L, M), dtype=torch.complex64, device=cuda)
    a = hpx.healpy_to_alm(p, L, M)
    mask = torch.from_numpy(np.arange(M)[None, :] > np.arange(L)[:, None]).to(cuda)
    assert torch.count_nonzero(a[:, mask]) == 0


def test_round_trip_with_the_transform(cuda):
    # healpy-packed coefficients -> dense -> iSHT -> SHT -> packed
    import cuhpx_b200 as hpx

    # band limit within what nside 16 resolves; two Jacobi iterations remove
    # the quadrature error
    nside, L = 16, 17
    rng = np.random.default_rng(1)
    a = rng.standard_normal((2, L, L)) + 1j * rng.standard_normal((2, L, L))
    a = np.where(np.arange(L)[None, None, :] <= np.arange(L)[None, :, None], a, 0)
    a[..., 0] = a[..., 0].real
    p = hpx.alm_to_healpy(torch.from_numpy(a).to(cuda), csphase=True)
    f = hpx.iSHTCUDA(nside, lmax=L, mmax=L)(hpx.healpy_to_alm(p, L, L, csphase=True))
    back = hpx.alm_to_healpy(hpx.SHTCUDA(nside, lmax=L, mmax=L, refine_iters=2)(f), csphase=True)
    assert float((back - p).abs().norm() / p.abs().norm()) < 1e-6


def test_argument_errors(cuda):
    import cuhpx_b200 as hpx

    with pytest.raises(ValueError, match="complex64 or complex128"):
        hpx.alm_to_healpy(torch.zeros(3, 3, device=cuda))
    with pytest.raises(ValueError, match="packed length"):
        hpx.healpy_to_alm(torch.zeros(5, dtype=torch.complex64, device=cuda), 3)
