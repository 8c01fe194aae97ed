"""Spin-1 (vector) transforms on the GPU against the oracle and the reference's goldens.

Tolerances (rel-L2): FP64 vs the float64 oracle <= 1e-11; FP32 <= 1e-5; vs
the reference's own float64 outputs <= 1e-6 (it rounds its ring phases to
complex64); adjoint dot-product identities (FP64) <= 1e-12; gradients vs the
reference's autograd (FP64) <= 1e-6.
"""

import os

import numpy as np
import pytest
import torch

from oracle import vector_oracle as V

pytestmark = pytest.mark.gpu

G = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    b = b.detach().cpu().numpy() if torch.is_tensor(b) else np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


def vec_alm(rng, L, M, batch=()):
    a = rng.standard_normal(batch + (2, L, M)) + 1j * rng.standard_normal(batch + (2, L, M))
    a = np.where(np.arange(M)[None, :] <= np.arange(L)[:, None], a, 0)
    a[..., 0] = a[..., 0].real
    return a


@pytest.mark.parametrize("name", ["n8", "n8_nocs", "n4_mlt", "n4_mgt"])
def test_reference_goldens(hpx, cuda, name):
    d = np.load(os.path.join(G, "vector_small.npz"))
    nside, L, M, cs = (int(v) for v in d[name + "_cfg"])
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=M, csphase=bool(cs))
    vi = hpx.VectoriSHTCUDA(nside, lmax=L, mmax=M, csphase=bool(cs))
    f = torch.from_numpy(d[name + "_f"]).to(cuda)
    a = torch.from_numpy(d[name + "_a"]).to(cuda)
    assert rel(vs(f), d[name + "_alm"]) < 1e-6
    assert rel(vi(a), d[name + "_map"]) < 1e-6
    assert rel(vs(f.float()), d[name + "_alm"]) < 1e-5
    assert rel(vi(a.to(torch.complex64)), d[name + "_map"]) < 1e-5


CASES = [(2, 5, 5), (8, 17, 17), (8, 17, 6), (8, 9, 13), (16, 33, 33), (32, 65, 40), (64, 129, 129)]


@pytest.mark.parametrize("nside,L,M", CASES)
def test_vs_oracle(hpx, cuda, nside, L, M):
    rng = np.random.default_rng(nside * 100 + L + M)
    f = rng.standard_normal((3, 2, 12 * nside * nside))
    a = vec_alm(rng, L, M, (2,))
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=M)
    vi = hpx.VectoriSHTCUDA(nside, lmax=L, mmax=M)
    ref_a = V.vsht(f, nside, L, M)
    ref_f = V.visht(a, nside)
    got_a = vs(torch.from_numpy(f).to(cuda))
    got_f = vi(torch.from_numpy(a).to(cuda))
    assert got_a.shape == (3, 2, L, M) and got_a.dtype == torch.complex128
    assert got_f.shape == (2, 2, 12 * nside * nside)
    assert rel(got_a, ref_a) < 1e-11
    assert rel(got_f, ref_f) < 1e-11
    assert rel(vs(torch.from_numpy(f).float().to(cuda)), ref_a) < 1e-5
    assert rel(vi(torch.from_numpy(a).to(cuda, torch.complex64)), ref_f) < 1e-5


def test_vs_oracle_nside256(hpx, cuda):
    """The size the benchmark times (nside 256, L = M = 511): FP64 and FP32
    analysis and synthesis of 2 tangent fields against the float64 oracle."""
    nside, L = 256, 511
    rng = np.random.default_rng(256)
    f = rng.standard_normal((2, 2, 12 * nside * nside))
    a = vec_alm(rng, L, L, (2,))
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=L)
    vi = hpx.VectoriSHTCUDA(nside, lmax=L, mmax=L)
    ref_a = V.vsht(f, nside, L, L)
    ref_f = V.visht(a, nside)
    with torch.no_grad():
        assert rel(vs(torch.from_numpy(f).to(cuda)), ref_a) < 1e-10
        assert rel(vi(torch.from_numpy(a).to(cuda)), ref_f) < 1e-10
        assert rel(vs(torch.from_numpy(f).float().to(cuda)), ref_a) < 1e-5
        assert rel(vi(torch.from_numpy(a).to(cuda, torch.complex64)), ref_f) < 1e-5


def test_shapes_and_many_chunks(hpx, cuda):
    nside, L = 8, 17
    rng = np.random.default_rng(7)
    f = rng.standard_normal((70, 2, 12 * nside * nside))  # three passes of 32 vector maps
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=L)
    ref = V.vsht(f, nside, L, L)
    assert rel(vs(torch.from_numpy(f).to(cuda)), ref) < 1e-11
    one = vs(torch.from_numpy(f[0]).to(cuda))  # a single vector map [2, npix]
    assert one.shape == (2, L, L) and rel(one, ref[0]) < 1e-11
    with pytest.raises(ValueError, match="real"):
        vs(torch.zeros(2, 768, dtype=torch.complex64, device=cuda))
    with pytest.raises(ValueError, match=r"\[\.\.\., 2, 768\]"):
        vs(torch.zeros(3, 768, device=cuda))


def test_adjoint_identities(hpx, cuda):
    from cuhpx_b200.vector import _analysis, _synthesis

    nside, L, M = 16, 33, 21
    rng = np.random.default_rng(9)
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=M)
    plan = vs._plan(torch.float64, cuda)
    x = torch.from_numpy(rng.standard_normal((2, 2, 12 * nside * nside))).to(cuda)
    y = torch.from_numpy(vec_alm(rng, L, M, (2,))).to(cuda)
    for cs in (True, False):
        # <S x, y> = <x, S^T y>  and  <I y, x> = <y, I^T x> (real inner products)
        lhs = torch.sum((_analysis(plan, x, L, M, cs).conj() * y).real)
        rhs = torch.sum(x * _synthesis(plan, y, cs, adjoint=True))
        assert abs(float(lhs - rhs)) < 1e-12 * float(lhs.abs() + rhs.abs())
        lhs = torch.sum(_synthesis(plan, y, cs) * x)
        rhs = torch.sum((y.conj() * _analysis(plan, x, L, M, cs, adjoint=True)).real)
        assert abs(float(lhs - rhs)) < 1e-12 * float(lhs.abs() + rhs.abs())


def test_gradients_vs_reference_autograd(hpx, cuda):
    d = np.load(os.path.join(G, "vector_small.npz"))
    nside, L, M, cs = (int(v) for v in d["n8_cfg"])
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=M, csphase=bool(cs))
    vi = hpx.VectoriSHTCUDA(nside, lmax=L, mmax=M, csphase=bool(cs))
    f = torch.from_numpy(d["n8_f"]).to(cuda).requires_grad_(True)
    wl = 1.0 / (torch.arange(L, dtype=torch.float64, device=cuda) + 1.0)[:, None]
    (vs(f).abs() ** 2 * wl).sum().backward()
    assert rel(f.grad, d["n8_grad_f"]) < 1e-6
    a = torch.from_numpy(d["n8_a"]).to(cuda).requires_grad_(True)
    (vi(a) ** 2).sum().backward()
    assert rel(a.grad, d["n8_grad_a"]) < 1e-6
