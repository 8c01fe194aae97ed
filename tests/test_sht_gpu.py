"""Parity of the CUDA transforms with the CPU oracle and with the reference's goldens.

Tolerances (rel-L2):
  FP64 plan vs float64 oracle          <= 1e-11
  FP32 plan vs float64 oracle          <= 1e-5  (the plain FP32 bar; typically ~1e-7)
  FP32 plan vs reference float32 output<= 1e-5
  adjoint dot-product identities (FP64) <= 1e-12
"""

import os

import numpy as np
import pytest
import torch

from oracle import hpx_oracle as O

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    b = b.detach().cpu().numpy() if torch.is_tensor(b) else np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rand_alm(rng, L, M, batch=()):
    a = rng.standard_normal(batch + (L, M)) + 1j * rng.standard_normal(batch + (L, M))
    l = np.arange(L)[:, None]
    m = np.arange(M)[None, :]
    a = np.where(m <= l, a, 0)
    a[..., 0] = a[..., 0].real
    return a


CASES = [
    (1, 3, 3),
    (3, 7, 7),
    (5, 11, 9),
    (2, 7, 5),
    (4, 9, 9),
    (8, 17, 17),
    (8, 31, 17),
    (8, 9, 17),
    (8, 17, 5),
    (16, 33, 33),
    (32, 65, 65),
    (32, 127, 65),
    (64, 129, 129),
]


def qw_for(nside):
    # 'ring' weights exist for power-of-two nside >= 2; other nside use uniform weights
    return "ring" if nside >= 2 and nside & (nside - 1) == 0 else "none"


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


@pytest.mark.parametrize("nside,L,M", CASES)
def test_forward_vs_oracle(hpx, cuda, nside, L, M):
    rng = np.random.default_rng(nside * 1000 + L)
    qw = qw_for(nside)
    f = rng.standard_normal((2, 12 * nside * nside))
    ref = O.sht(f, nside, L, M, quad_weights=qw)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=M, quad_weights=qw)
    a64 = sht(torch.from_numpy(f).to(cuda))
    assert a64.dtype == torch.complex128 and a64.shape == (2, L, M)
    assert rel(a64, ref) < 1e-11
    a32 = sht(torch.from_numpy(f).float().to(cuda))
    assert a32.dtype == torch.complex64
    assert rel(a32, ref) < 1e-5
    # entries with m > l are exactly zero
    mask = np.arange(M)[None, :] > np.arange(L)[:, None]
    assert torch.count_nonzero(a32[:, torch.from_numpy(mask).to(cuda)]) == 0


@pytest.mark.parametrize("nside,L,M", CASES)
def test_inverse_vs_oracle(hpx, cuda, nside, L, M):
    rng = np.random.default_rng(nside * 7 + M)
    a = rand_alm(rng, L, M, (3,))
    ref = O.isht(a, nside)
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=M, quad_weights=qw_for(nside))
    f64 = isht(torch.from_numpy(a).to(cuda))
    assert f64.dtype == torch.float64 and f64.shape == (3, 12 * nside * nside)
    assert rel(f64, ref) < 1e-11
    f32 = isht(torch.from_numpy(a).to(torch.complex64).to(cuda))
    assert rel(f32, ref) < 1e-5


def test_inverse_ignores_imag_of_m0(hpx, cuda):
    rng = np.random.default_rng(3)
    a = rand_alm(rng, 17, 17)
    b = a.copy()
    b[:, 0] += 1j * rng.standard_normal(17)
    isht = hpx.iSHTCUDA(8, lmax=17, mmax=17)
    fa = isht(torch.from_numpy(a).to(cuda))
    fb = isht(torch.from_numpy(b).to(cuda))
    assert rel(fb, fa) < 1e-14


def test_reference_goldens_cfg1(hpx, cuda):
    d = np.load(os.path.join(G, "cfg1_n32.npz"))
    sht = hpx.SHTCUDA(32, lmax=65, mmax=65)
    isht = hpx.iSHTCUDA(32, lmax=65, mmax=65)
    f = torch.from_numpy(d["f"]).to(cuda)
    assert rel(sht(f.float()), d["alm32"]) < 1e-5
    assert rel(sht(f), d["alm64"]) < 1e-7  # reference rounds its phases to complex64
    a = torch.from_numpy(d["alm64"]).to(cuda)
    assert rel(isht(a.to(torch.complex64)), d["map32"]) < 1e-5
    assert rel(isht(a), d["map64"]) < 1e-7


@pytest.mark.parametrize("name", ["small_n2", "small_n4", "small_n8", "small_n16"])
def test_reference_goldens_defaults(hpx, cuda, name):
    d = np.load(os.path.join(G, name + ".npz"))
    nside = int(d["default_nside"])
    # constructor defaults: lmax = 4*nside-1, mmax = 2*nside+1
    sht = hpx.SHTCUDA(nside)
    isht = hpx.iSHTCUDA(nside)
    assert (sht.lmax, sht.mmax) == (int(d["default_lmax"]), int(d["default_mmax"]))
    f = torch.from_numpy(d["default_f"]).to(cuda)
    assert rel(sht(f.float()), d["default_alm32"]) < 1e-5
    assert rel(isht(torch.from_numpy(d["default_alm64"]).to(cuda)), d["default_map64"]) < 1e-7


def test_reference_goldens_uniform_weights(hpx, cuda):
    d = np.load(os.path.join(G, "none_n8.npz"))
    sht = hpx.SHTCUDA(8, lmax=17, mmax=17, quad_weights="none")
    assert rel(sht(torch.from_numpy(d["f"]).float().to(cuda)), d["alm32"]) < 1e-5


def test_batch_shapes_and_1d(hpx, cuda):
    rng = np.random.default_rng(11)
    nside, L = 16, 33
    f = torch.from_numpy(rng.standard_normal((2, 3, 12 * nside * nside))).float().to(cuda)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L)
    a = sht(f)
    assert a.shape == (2, 3, L, L)
    for i in range(2):
        for j in range(3):
            a1 = sht(f[i, j])
            assert a1.shape == (L, L)
            assert rel(a1, a[i, j]) < 1e-6
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L)
    g = isht(a)
    assert g.shape == f.shape
    assert rel(isht(a[1, 2]), g[1, 2]) < 1e-6


def test_batch_larger_than_chunk(hpx, cuda):
    rng = np.random.default_rng(12)
    nside, L = 8, 17
    f = torch.from_numpy(rng.standard_normal((11, 12 * nside * nside))).to(cuda)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, batch_chunk=4)
    ref = O.sht(f.cpu().numpy(), nside, L, L)
    assert rel(sht(f), ref) < 1e-11
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L, batch_chunk=4)
    a = rand_alm(rng, L, L, (11,))
    assert rel(isht(torch.from_numpy(a).to(cuda)), O.isht(a, nside)) < 1e-11


def test_errors(hpx, cuda):
    sht = hpx.SHTCUDA(8, lmax=17, mmax=17)
    with pytest.raises(ValueError):
        sht(torch.zeros(12 * 64, dtype=torch.complex64, device=cuda))
    with pytest.raises(ValueError):
        sht(torch.zeros(100, device=cuda))
    isht = hpx.iSHTCUDA(8, lmax=17, mmax=17)
    with pytest.raises(ValueError):
        isht(torch.zeros(16, 17, dtype=torch.complex64, device=cuda))
    with pytest.raises(ValueError):
        hpx.SHTCUDA(3)(torch.zeros(12 * 9, device=cuda))  # no 'ring' weights for nside=3


def test_deterministic(hpx, cuda):
    rng = np.random.default_rng(5)
    f = torch.from_numpy(rng.standard_normal((4, 12 * 32 * 32))).float().to(cuda)
    sht = hpx.SHTCUDA(32, lmax=65, mmax=65)
    a1, a2 = sht(f), sht(f)
    assert torch.equal(a1, a2)


def test_one_plan_two_streams_two_threads(hpx, cuda):
    """Two host threads drive the same plan on two streams at once: each call's
    ring FFT forks onto the plan's own stream and joins back, and the results
    equal those of serial calls."""
    import threading

    rng = np.random.default_rng(11)
    nside, L = 64, 127
    fs = [torch.from_numpy(rng.standard_normal((8, 12 * nside * nside))).float().to(cuda) for _ in range(2)]
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="f16x3", refine_iters=0)
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision="f16x3")
    ref = [isht(sht(f)) for f in fs]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(cuda) for _ in range(2)]
    out = [[None] * 6, [None] * 6]

    def work(i):
        with torch.cuda.stream(streams[i]):
            for r in range(6):
                out[i][r] = isht(sht(fs[i]))

    ths = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    torch.cuda.synchronize()
    for i in range(2):
        for r in range(6):
            assert torch.equal(out[i][r], ref[i])


# ------------------------------------------------------------------ adjoints
def _dot_alm(a, b):
    return float(torch.sum(a.real * b.real + a.imag * b.imag))


@pytest.mark.parametrize("nside,L,M", [(4, 9, 9), (8, 17, 17), (8, 31, 17), (16, 20, 33)])
def test_adjoint_identities(hpx, cuda, nside, L, M):
    rng = np.random.default_rng(21)
    plan = hpx.get_plan(nside, L, M, "ring", "fp64", 0)
    f = torch.from_numpy(rng.standard_normal((2, 12 * nside * nside))).to(cuda)
    g = torch.from_numpy(rng.standard_normal((2, L, M)) + 1j * rng.standard_normal((2, L, M))).to(cuda)
    # <S f, g> = <f, S^T g>
    lhs = _dot_alm(plan.forward(f), g)
    rhs = float(torch.sum(f * plan.forward_adjoint(g)))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # <I a, h> = <a, I^T h>
    a = g
    h = torch.from_numpy(rng.standard_normal((2, 12 * nside * nside))).to(cuda)
    lhs = float(torch.sum(plan.inverse(a) * h))
    rhs = _dot_alm(a, plan.inverse_adjoint(h))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_grad_matches_reference_autograd(hpx, cuda):
    d = np.load(os.path.join(G, "grad_n8.npz"))
    nside, L = int(d["nside"]), int(d["lmax"])
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L)
    f = torch.from_numpy(d["f"]).to(cuda).requires_grad_(True)
    wl = 1.0 / (torch.arange(L, dtype=torch.float64, device=cuda) + 1.0)
    loss = (wl[:, None] * sht(f).abs() ** 2).sum()
    loss.backward()
    # the reference's float64 path rounds its ring phases to complex64 (~1e-8 relative)
    assert abs(loss.item() - float(d["loss"])) < 1e-7 * abs(float(d["loss"]))
    assert rel(f.grad, d["grad_f"]) < 1e-6
    # float32 path, same gradient to FP32 accuracy
    f32 = torch.from_numpy(d["f"]).float().to(cuda).requires_grad_(True)
    (wl.float()[:, None] * sht(f32).abs() ** 2).sum().backward()
    assert rel(f32.grad, d["grad_f"]) < 1e-5
    # inverse: loss = sum f^2
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L)
    a = torch.from_numpy(d["alm"]).to(cuda).requires_grad_(True)
    loss2 = (isht(a) ** 2).sum()
    loss2.backward()
    assert abs(loss2.item() - float(d["loss2"])) < 1e-7 * abs(float(d["loss2"]))
    # the reference's autograd gradient w.r.t. a complex leaf includes the
    # imaginary part of m=0, which the transform ignores; compare the rest
    ga, gr = a.grad.detach().cpu().numpy(), d["grad_alm"].copy()
    ga[:, 0] = ga[:, 0].real
    gr[:, 0] = gr[:, 0].real
    assert rel(ga, gr) < 1e-6


def test_grad_finite_differences_fp64(hpx, cuda):
    nside, L = 16, 33
    rng = np.random.default_rng(99)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L)
    wl = 1.0 / (torch.arange(L, dtype=torch.float64, device=cuda) + 1.0)

    def loss_fn(x):
        return (wl[:, None] * sht(x).abs() ** 2).sum()

    f = torch.from_numpy(rng.standard_normal(12 * nside * nside)).to(cuda).requires_grad_(True)
    loss_fn(f).backward()
    g = f.grad.detach()
    eps = 1e-5
    for _ in range(4):
        v = torch.from_numpy(rng.standard_normal(12 * nside * nside)).to(cuda)
        with torch.no_grad():
            fd = (loss_fn(f + eps * v) - loss_fn(f - eps * v)) / (2 * eps)
        an = torch.sum(g * v)
        assert abs(fd.item() - an.item()) <= 1e-6 * abs(an.item()) + 1e-12


def test_refined_matches_oracle(hpx, cuda):
    nside, L = 16, 31
    rng = np.random.default_rng(4)
    a_true = rand_alm(rng, L, L) / (np.arange(L)[:, None] + 1.0)
    fmap = O.isht(a_true, nside)
    # oracle Jacobi iterations
    ref = [O.sht(fmap, nside, L, L)]
    for _ in range(3):
        ref.append(ref[-1] + O.sht(fmap - O.isht(ref[-1], nside), nside, L, L))
    x = torch.from_numpy(fmap).to(cuda)
    for k in (0, 1, 3):
        sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, refine_iters=k)
        out = sht(x)
        assert rel(out, ref[k]) < 1e-10
    # refinement converges towards the band-limited truth
    e0 = rel(ref[0], a_true)
    e3 = rel(ref[3], a_true)
    assert e3 < 0.1 * e0


def test_refined_gradient_fd(hpx, cuda):
    nside, L = 8, 17
    rng = np.random.default_rng(31)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, refine_iters=2)
    f = torch.from_numpy(rng.standard_normal(12 * nside * nside)).to(cuda).requires_grad_(True)
    loss = (sht(f).abs() ** 2).sum()
    loss.backward()
    v = torch.from_numpy(rng.standard_normal(12 * nside * nside)).to(cuda)
    eps = 1e-5
    with torch.no_grad():
        fd = ((sht(f + eps * v).abs() ** 2).sum() - (sht(f - eps * v).abs() ** 2).sum()) / (2 * eps)
    an = torch.sum(f.grad * v)
    assert abs(fd.item() - an.item()) <= 1e-6 * abs(an.item())


def test_conjugated_inputs_and_cotangents(cuda):
    """Lazily conjugated tensors (from .conj()) are accepted as coefficients and
    as incoming gradients."""
    import cuhpx_b200 as hpx

    rng = np.random.default_rng(21)
    nside, L = 8, 17
    f = torch.from_numpy(rng.standard_normal((2, 12 * nside * nside))).to(cuda).requires_grad_(True)
    c = torch.from_numpy(rng.standard_normal((2, L, L)) + 1j * rng.standard_normal((2, L, L))).to(cuda)
    a = hpx.SHTCUDA(nside, lmax=L, mmax=L)(f)
    loss = (a.conj() * c).real.sum()
    loss.backward()
    assert abs(loss.item() - float((f.detach() * f.grad).sum())) < 1e-10 * max(1.0, abs(loss.item()))
    g = hpx.iSHTCUDA(nside, lmax=L, mmax=L)(a.detach().conj())
    g2 = hpx.iSHTCUDA(nside, lmax=L, mmax=L)(a.detach().conj().resolve_conj())
    assert torch.equal(g, g2)


@pytest.mark.parametrize("prec,tol", [("fp32", 5e-6), ("f16x3", 1e-5)])
def test_nside_2048_band_limited_round_trip(hpx, cuda, prec, tol):
    """nside 2048: Bluestein lengths up to 8192 (their FP64 chirp spectra are
    precomputed in a global scratch) and shared-memory ring kernels near the
    per-block limit; synthesis then analysis of band-limited coefficients
    returns them."""
    nside, L = 2048, 255
    rng = np.random.default_rng(2048)
    a = (rng.standard_normal((1, L, L)) + 1j * rng.standard_normal((1, L, L))) / np.sqrt(np.arange(1, L + 1))[None, :, None]
    a = np.tril(a)
    a[:, :, 0] = a[:, :, 0].real
    at = torch.from_numpy(a).to(cuda, torch.complex64)
    f = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision=prec)(at)
    b = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec, refine_iters=0)(f)
    assert rel(b, a) < tol
