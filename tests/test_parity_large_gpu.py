"""Parity with the CPU oracle at the survey's large configurations.

cfg2: synthesis -> analysis round trip at nside 256, L = M = 511, 8 maps whose
a_lm are complex Gaussian with variance C_l ~ (l+1)^-2 (m <= l, Im a_l0 = 0),
against the full float64 oracle (its per-order form, pinned to the full
transforms on the CPU).  Bars (rel-L2):
  FP64 path                       <= 1e-10
  plain FP32 path                 <= 1e-5
  f16x3 / bf16x3 with 1 Jacobi iteration vs the oracle with 1 iteration <= 1e-5
  f16x3 / bf16x3 synthesis        <= 1e-5

cfg3: nside 1024, L = M = 2047, maps of the benchmark's recipe (band-limited
field plus N(0, 1e-3) noise):
  * spot oracle (orders 0, 1, 2, 511, 1023, 2046; one Legendre column at a
    time) on 2 maps, at the plan's ring nodes with the recurrence in extended
    precision: FP64 path <= 1e-10, FP32 and f16x3 <= 1e-5.  The reference's
    own FP64 recurrence (the spot oracle's reference form) loses bits there
    (subnormal diagonals of high orders near the poles); on these orders the
    FP64 path is within 1e-7 of it;
  * the whole coefficient set of one map against the C port of the
    reference's CPU transform (oracle/ref_cpu.c) run in extended precision at
    the same nodes (pinned to the oracle on the CPU): FP64 analysis and
    synthesis <= 1e-10, FP32 <= 1e-5, f16x3 with 1 Jacobi iteration vs the
    port with 1 iteration <= 1e-5, f16x3 synthesis <= 1e-5.  The reference's
    own FP64 recurrence is off by far more than 1e-5 there: for orders near
    1200 its subnormal diagonal makes the recurrence diverge.
"""

import numpy as np
import pytest
import torch

from oracle import hpx_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    b = b.detach().cpu().numpy() if torch.is_tensor(b) else np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def cl_alm(rng, L, batch):
    """complex Gaussian a_lm with variance (l+1)^-2, m <= l, Im a_l0 = 0"""
    sig = 1.0 / (np.arange(L) + 1.0)[:, None]
    a = (rng.standard_normal((batch, L, L)) + 1j * rng.standard_normal((batch, L, L))) * sig / np.sqrt(2.0)
    a = np.where(np.arange(L)[None, :] <= np.arange(L)[:, None], a, 0)
    a[..., 0] = a[..., 0].real
    return a


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


# --------------------------------------------------------------------------- cfg2
N2, L2, B2 = 256, 511, 8


@pytest.fixture(scope="module")
def cfg2():
    rng = np.random.default_rng(1)
    a = cl_alm(rng, L2, B2)
    f = O.isht_by_m(a, N2)  # band-limited maps
    a0 = O.sht_by_m(f, N2, L2, L2)
    # one Jacobi iteration in float64: a1 = a0 + SHT(f - iSHT(a0))
    a1 = a0 + O.sht_by_m(f - O.isht_by_m(a0, N2), N2, L2, L2)
    return dict(a=a, f=f, a0=a0, a1=a1)


def test_cfg2_fp64(hpx, cuda, cfg2):
    sht = hpx.SHTCUDA(N2, lmax=L2, mmax=L2)
    isht = hpx.iSHTCUDA(N2, lmax=L2, mmax=L2)
    assert rel(isht(torch.from_numpy(cfg2["a"]).to(cuda)), cfg2["f"]) < 1e-10
    assert rel(sht(torch.from_numpy(cfg2["f"]).to(cuda)), cfg2["a0"]) < 1e-10


def test_cfg2_plain_fp32(hpx, cuda, cfg2):
    sht = hpx.SHTCUDA(N2, lmax=L2, mmax=L2, precision="fp32")
    isht = hpx.iSHTCUDA(N2, lmax=L2, mmax=L2, precision="fp32")
    assert rel(isht(torch.from_numpy(cfg2["a"]).to(cuda, torch.complex64)), cfg2["f"]) < 1e-5
    assert rel(sht(torch.from_numpy(cfg2["f"]).to(cuda, torch.float32)), cfg2["a0"]) < 1e-5


@pytest.mark.parametrize("prec", ["f16x3", "bf16x3"])
def test_cfg2_mixed(hpx, cuda, cfg2, prec):
    f32 = torch.from_numpy(cfg2["f"]).to(cuda, torch.float32)
    isht = hpx.iSHTCUDA(N2, lmax=L2, mmax=L2, precision=prec)
    assert rel(isht(torch.from_numpy(cfg2["a"]).to(cuda, torch.complex64)), cfg2["f"]) < 1e-5
    sht1 = hpx.SHTCUDA(N2, lmax=L2, mmax=L2, precision=prec, refine_iters=1)
    assert rel(sht1(f32), cfg2["a1"]) < 1e-5
    # without refinement the error is reported, not bounded by 1e-5; keep it in its known range
    sht0 = hpx.SHTCUDA(N2, lmax=L2, mmax=L2, precision=prec, refine_iters=0)
    assert rel(sht0(f32), cfg2["a0"]) < 3e-5


# ------------------------------------------------------ Bluestein lengths 3 * 2^k
@pytest.mark.parametrize("nside", [600, 768])
def test_bluestein_3x2k_lengths(hpx, cuda, nside):
    """Rings whose Bluestein convolution runs at 3072 points instead of 4096.

    Polar ring i carries h = 2i complex points and needs a convolution of at
    least 2h - 1 points: 3072 for i = 513..768.  At nside 600 the rings
    513..599 and the equatorial rings (h = 1200) run at 3072; at nside 768 the
    rings 513..767 and the equatorial rings, whose h = 1536 puts 2h - 1 = 3071
    at the top of the range.  Band-limited maps, 2 of them, L = M = nside + 1,
    uniform quadrature weights (ring weights exist for powers of two only),
    against the float64 oracle.
    """
    L = nside + 1
    rng = np.random.default_rng(nside)
    a = cl_alm(rng, L, 2)
    f = O.isht_by_m(a, nside)
    a0 = O.sht_by_m(f, nside, L, L, quad_weights="none")
    kw = dict(lmax=L, mmax=L, quad_weights="none")
    with torch.no_grad():
        at, ft = torch.from_numpy(a).to(cuda), torch.from_numpy(f).to(cuda)
        assert rel(hpx.iSHTCUDA(nside, **kw)(at), f) < 1e-10
        assert rel(hpx.SHTCUDA(nside, **kw)(ft), a0) < 1e-10
        assert rel(hpx.iSHTCUDA(nside, precision="fp32", **kw)(at.to(torch.complex64)), f) < 1e-5
        assert rel(hpx.SHTCUDA(nside, precision="fp32", **kw)(ft.float()), a0) < 1e-5
        assert rel(hpx.iSHTCUDA(nside, precision="f16x3", **kw)(at.to(torch.complex64)), f) < 2e-5
        assert rel(hpx.SHTCUDA(nside, precision="f16x3", refine_iters=0, **kw)(ft.float()), a0) < 2e-5


# --------------------------------------------------------------------------- cfg3
N3, L3 = 1024, 2047
SPOT = [0, 1, 2, 511, 1023, 2046]


@pytest.fixture(scope="module")
def cfg3_maps(hpx, cuda):
    """2 maps of the benchmark recipe, synthesised on the device in FP64."""
    rng = np.random.default_rng(3)
    a = torch.from_numpy(cl_alm(rng, L3, 2)).to(cuda)
    with torch.no_grad():
        f = hpx.iSHTCUDA(N3, lmax=L3, mmax=L3)(a)
    del a
    f = f.cpu().numpy() + rng.standard_normal(f.shape) * np.sqrt(1e-3)
    torch.cuda.empty_cache()
    return f


def test_cfg3_spot_oracle(hpx, cuda, cfg3_maps):
    f = cfg3_maps
    exact = O.sht_spot(f, N3, L3, L3, SPOT, nodes="exact")
    ref = O.sht_spot(f, N3, L3, L3, SPOT)
    x = torch.from_numpy(f).to(cuda)
    with torch.no_grad():
        a64 = hpx.SHTCUDA(N3, lmax=L3, mmax=L3)(x)[..., SPOT]
        assert rel(a64, exact) < 1e-10
        assert rel(a64, ref) < 1e-7
        a32 = hpx.SHTCUDA(N3, lmax=L3, mmax=L3, precision="fp32")(x.float())[..., SPOT]
        assert rel(a32, exact) < 1e-5
        amx = hpx.SHTCUDA(N3, lmax=L3, mmax=L3, precision="f16x3", refine_iters=0)(x.float())[..., SPOT]
        assert rel(amx, exact) < 1e-5
    torch.cuda.empty_cache()


@pytest.fixture(scope="module")
def ref_cpu():
    from oracle import ref_cpu as RC

    try:
        RC.load()
    except Exception as e:
        pytest.skip(f"CPU port not built: {e}")
    return RC


def test_cfg3_full_vs_extended_port(hpx, cuda, cfg3_maps, ref_cpu):
    f = cfg3_maps[0]
    a0 = ref_cpu.sht_extended(f, N3, L3, L3)
    g0 = ref_cpu.isht_extended(a0, N3)
    a1 = a0 + ref_cpu.sht_extended(f - g0, N3, L3, L3)
    x = torch.from_numpy(f).to(cuda)
    a0c = torch.from_numpy(a0).to(cuda)
    with torch.no_grad():
        assert rel(hpx.SHTCUDA(N3, lmax=L3, mmax=L3)(x), a0) < 1e-10
        assert rel(hpx.iSHTCUDA(N3, lmax=L3, mmax=L3)(a0c), g0) < 1e-10
        assert rel(hpx.SHTCUDA(N3, lmax=L3, mmax=L3, precision="fp32")(x.float()), a0) < 1e-5
        assert rel(hpx.iSHTCUDA(N3, lmax=L3, mmax=L3, precision="fp32")(a0c.to(torch.complex64)), g0) < 1e-5
        got = hpx.SHTCUDA(N3, lmax=L3, mmax=L3, precision="f16x3", refine_iters=1)(x.float())
        assert rel(got, a1) < 1e-5
        g = hpx.iSHTCUDA(N3, lmax=L3, mmax=L3, precision="f16x3")(a0c.to(torch.complex64))
        assert rel(g, g0) < 1e-5
    # the reference's own FP64 recurrence is far from these values at this size
    # (its subnormal diagonals make the recurrence diverge in orders near 1200)
    assert rel(ref_cpu.sht(f, N3, L3, L3), a0) > 1e-5
    torch.cuda.empty_cache()
