"""Mixed-precision (tcgen05, bf16 3-term split) transforms against the oracle.

Tolerances (rel-L2):
  one bf16x3 transform vs float64 oracle          <= 3e-5
  bf16x3 refined analysis vs float64 oracle with the same number of Jacobi
  iterations                                        <= 1e-5
"""

import numpy as np
import pytest
import torch

from oracle import hpx_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rand_alm(rng, L, M, batch=(), decay=0.0):
    a = rng.standard_normal(batch + (L, M)) + 1j * rng.standard_normal(batch + (L, M))
    l = np.arange(L)[:, None]
    a = a / (l + 1.0) ** decay
    m = np.arange(M)[None, :]
    a = np.where(m <= l, a, 0)
    a[..., 0] = a[..., 0].real
    return a


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


TC_CASES = [(4, 9, 9), (8, 17, 17), (8, 31, 17), (8, 9, 17), (8, 17, 5), (16, 33, 33), (32, 65, 65), (64, 127, 127),
            (128, 255, 255), (64, 257, 129)]


@pytest.mark.parametrize("nside,L,M", TC_CASES)
def test_tc_forward(hpx, cuda, nside, L, M):
    rng = np.random.default_rng(nside + L + M)
    f = rng.standard_normal((3, 12 * nside * nside))
    ref = O.sht(f, nside, L, M)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=M, precision="bf16x3")
    a = sht(torch.from_numpy(f).float().to(cuda))
    hpx.get_plan(nside, L, M, "ring", "bf16x3", 0).check()
    e = rel(a, ref)
    print(f"bf16x3 forward nside={nside} L={L} M={M}: {e:.2e}")
    assert e < 3e-5
    mask = np.arange(M)[None, :] > np.arange(L)[:, None]
    assert torch.count_nonzero(a[:, torch.from_numpy(mask).to(cuda)]) == 0


@pytest.mark.parametrize("nside,L,M", TC_CASES)
def test_tc_inverse(hpx, cuda, nside, L, M):
    rng = np.random.default_rng(7 * nside + L + M)
    a = rand_alm(rng, L, M, (3,))
    ref = O.isht(a, nside)
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=M, precision="bf16x3")
    f = isht(torch.from_numpy(a).to(torch.complex64).to(cuda))
    hpx.get_plan(nside, L, M, "ring", "bf16x3", 0).check()
    e = rel(f, ref)
    print(f"bf16x3 inverse nside={nside} L={L} M={M}: {e:.2e}")
    assert e < 3e-5


def test_tc_batch_not_multiple_of_64(hpx, cuda):
    rng = np.random.default_rng(1)
    nside, L = 16, 33
    f = rng.standard_normal((70, 12 * nside * nside))
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="bf16x3")
    a = sht(torch.from_numpy(f).float().to(cuda))
    assert rel(a, O.sht(f, nside, L, L)) < 3e-5


@pytest.mark.parametrize("k", [1, 2])
def test_tc_refined_matches_fp64_refined(hpx, cuda, k):
    nside, L = 32, 63
    rng = np.random.default_rng(10 + k)
    a_true = rand_alm(rng, L, L, (2,), decay=1.0)
    fmap = O.isht(a_true, nside) + 1e-3 ** 0.5 * rng.standard_normal((2, 12 * nside * nside))
    ref = O.sht(fmap, nside, L, L)
    for _ in range(k):
        ref = ref + O.sht(fmap - O.isht(ref, nside), nside, L, L)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="bf16x3", refine_iters=k)
    out = sht(torch.from_numpy(fmap).float().to(cuda))
    e = rel(out, ref)
    print(f"bf16x3 refined k={k}: {e:.2e}")
    assert e < 1e-5


def test_tc_matches_fp32_plain(hpx, cuda):
    rng = np.random.default_rng(3)
    nside, L = 64, 127
    f = torch.from_numpy(rng.standard_normal((4, 12 * nside * nside))).float().to(cuda)
    a32 = hpx.SHTCUDA(nside, lmax=L, mmax=L)(f)
    atc = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="bf16x3")(f)
    assert rel(atc, a32.cpu().numpy()) < 3e-5
