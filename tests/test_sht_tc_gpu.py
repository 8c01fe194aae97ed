"""Mixed-precision (tcgen05, bf16 or fp16 3-term split) transforms against the oracle.

Tolerances (rel-L2):
  one bf16x3 transform vs float64 oracle          <= 3e-5
  one f16x3 transform vs float64 oracle           <= 2e-6
  refined analysis vs float64 oracle with the same number of Jacobi
  iterations                                        <= 1e-5 (bf16x3), 2e-6 (f16x3)
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


TOL = {"bf16x3": 3e-5, "f16x3": 2e-6}
TOL_REFINED = {"bf16x3": 1e-5, "f16x3": 2e-6}
PRECS = ["bf16x3", "f16x3"]

TC_CASES = [(4, 9, 9), (8, 17, 17), (8, 31, 17), (8, 9, 17), (8, 17, 5), (16, 33, 33), (32, 65, 65), (64, 127, 127),
            (128, 255, 255), (64, 257, 129)]


@pytest.mark.parametrize("tab", [True, False], ids=["table", "otf"])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("nside,L,M", TC_CASES)
def test_tc_forward(hpx, cuda, nside, L, M, prec, tab):
    rng = np.random.default_rng(nside + L + M)
    f = rng.standard_normal((3, 12 * nside * nside))
    ref = O.sht(f, nside, L, M)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=M, precision=prec, legendre_table=tab)
    a = sht(torch.from_numpy(f).float().to(cuda))
    plan = hpx.get_plan(nside, L, M, "ring", prec, 0, 64, tab)
    plan.check()
    assert (plan.table_bytes > 0) == tab
    e = rel(a, ref)
    print(f"{prec} forward nside={nside} L={L} M={M}: {e:.2e}")
    assert e < TOL[prec]
    mask = np.arange(M)[None, :] > np.arange(L)[:, None]
    assert torch.count_nonzero(a[:, torch.from_numpy(mask).to(cuda)]) == 0


@pytest.mark.parametrize("tab", [True, False], ids=["table", "otf"])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("nside,L,M", TC_CASES)
def test_tc_inverse(hpx, cuda, nside, L, M, prec, tab):
    rng = np.random.default_rng(7 * nside + L + M)
    a = rand_alm(rng, L, M, (3,))
    ref = O.isht(a, nside)
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=M, precision=prec, legendre_table=tab)
    f = isht(torch.from_numpy(a).to(torch.complex64).to(cuda))
    hpx.get_plan(nside, L, M, "ring", prec, 0, 64, tab).check()
    e = rel(f, ref)
    print(f"{prec} inverse nside={nside} L={L} M={M}: {e:.2e}")
    assert e < TOL[prec]


@pytest.mark.parametrize("prec", PRECS)
def test_tc_batch_not_multiple_of_64(hpx, cuda, prec):
    rng = np.random.default_rng(1)
    nside, L = 16, 33
    f = rng.standard_normal((70, 12 * nside * nside))
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec)
    a = sht(torch.from_numpy(f).float().to(cuda))
    assert rel(a, O.sht(f, nside, L, L)) < TOL[prec]


@pytest.mark.parametrize("tab", [True, False], ids=["table", "otf"])
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("k", [1, 2])
def test_tc_refined_matches_fp64_refined(hpx, cuda, k, prec, tab):
    nside, L = 32, 63
    rng = np.random.default_rng(10 + k)
    a_true = rand_alm(rng, L, L, (2,), decay=1.0)
    fmap = O.isht(a_true, nside) + 1e-3 ** 0.5 * rng.standard_normal((2, 12 * nside * nside))
    ref = O.sht(fmap, nside, L, L)
    for _ in range(k):
        ref = ref + O.sht(fmap - O.isht(ref, nside), nside, L, L)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec, refine_iters=k, legendre_table=tab)
    out = sht(torch.from_numpy(fmap).float().to(cuda))
    e = rel(out, ref)
    print(f"{prec} refined k={k}: {e:.2e}")
    assert e < TOL_REFINED[prec]


@pytest.mark.parametrize("prec", PRECS)
def test_tc_matches_fp32_plain(hpx, cuda, prec):
    rng = np.random.default_rng(3)
    nside, L = 64, 127
    f = torch.from_numpy(rng.standard_normal((4, 12 * nside * nside))).float().to(cuda)
    a32 = hpx.SHTCUDA(nside, lmax=L, mmax=L)(f)
    atc = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec)(f)
    assert rel(atc, a32.cpu().numpy()) < TOL[prec]


def test_f16x3_per_map_scale(hpx, cuda):
    """Maps (and coefficient sets) many decades apart in one batch, and an all-zero
    one: each keeps the accuracy of an unscaled map (the fp16 operands carry a
    power-of-two scale per map)."""
    rng = np.random.default_rng(5)
    nside, L = 32, 65
    base = rng.standard_normal((5, 12 * nside * nside))
    scales = np.array([1.0, 1e-30, 1e30, 3e-8, 0.0])
    f = base * scales[:, None]
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="f16x3")
    a = sht(torch.from_numpy(f).float().to(cuda)).cpu().numpy()
    ref = O.sht(base, nside, L, L)
    for i, s in enumerate(scales):
        if s == 0.0:
            assert np.count_nonzero(a[i]) == 0
        else:
            assert rel(a[i] / s, ref[i]) < 2e-6, i
    alm = rand_alm(rng, L, L, (5,))
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision="f16x3")
    g = isht(torch.from_numpy(alm * scales[:, None, None]).to(torch.complex64).to(cuda)).cpu().numpy()
    gref = O.isht(alm, nside)
    for i, s in enumerate(scales):
        if s == 0.0:
            assert np.count_nonzero(g[i]) == 0
        else:
            assert rel(g[i] / s, gref[i]) < 2e-6, i
    hpx.get_plan(nside, L, L, "ring", "f16x3", 0).check()


@pytest.mark.parametrize("prec", PRECS)
def test_table_matches_on_the_fly(hpx, cuda, prec):
    """Resident-table and on-the-fly Pbar give the same transforms up to the
    FP32 rounding of Pbar (the two round at different points)."""
    rng = np.random.default_rng(11)
    nside, L = 64, 127
    f = torch.from_numpy(rng.standard_normal((3, 12 * nside * nside))).float().to(cuda)
    at = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec, legendre_table=True)(f)
    ao = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec, legendre_table=False)(f)
    assert rel(at, ao.cpu().numpy()) < 1e-6
    gt = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision=prec, legendre_table=True)(at)
    go = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision=prec, legendre_table=False)(at)
    assert rel(gt, go.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
def test_table_stream_bytes(hpx, cuda, prec):
    """A table plan streams at most its box-granular table per pass and skips
    all-zero blocks (more of them with fp16, whose smallest subnormal is far
    above bf16's); an on-the-fly plan reports (0, 0)."""
    nside, L = 256, 511
    p = hpx.get_plan(nside, L, L, "ring", prec, cuda.index, legendre_table=True)
    fwd, inv = p.table_stream_bytes
    assert p.table_bytes > 0 and 0 < fwd and 0 < inv
    # box-granular bound: every analysis tile's full ring range, every synthesis tile's full degree range
    assert fwd <= 2 * p.table_bytes and inv <= 2 * p.table_bytes
    q = hpx.get_plan(nside, L, L, "ring", prec, cuda.index, legendre_table=False)
    assert q.table_stream_bytes == (0, 0)
    if prec == "f16x3":
        b = hpx.get_plan(nside, L, L, "ring", "bf16x3", cuda.index, legendre_table=True)
        bf, bi = b.table_stream_bytes
        assert fwd <= bf and inv <= bi
