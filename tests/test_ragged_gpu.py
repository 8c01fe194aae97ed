"""Ragged batches (several resolutions in one call) and their CUDA-graph replay."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import hpx_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


def rand_maps(rng, nsides, counts, cuda, dtype=torch.float32):
    return [torch.from_numpy(rng.standard_normal((c, 12 * n * n))).to(cuda, dtype) for n, c in zip(nsides, counts)]


@pytest.mark.parametrize("prec", ["fp32", "f16x3"])
def test_ragged_forward_matches_per_group(hpx, cuda, prec):
    rng = np.random.default_rng(1)
    nsides, counts = [4, 16, 8, 32], [3, 5, 1, 2]
    maps = rand_maps(rng, nsides, counts, cuda)
    out = hpx.RaggedSHT(nsides, precision=prec)(maps)
    for x, a, n in zip(maps, out, nsides):
        ref = hpx.SHTCUDA(n, lmax=2 * n - 1, mmax=2 * n - 1, precision=prec)(x)
        assert a.shape == ref.shape
        assert torch.equal(a, ref)
    # and against the oracle
    a0 = out[1].cpu().numpy()
    assert np.linalg.norm(a0 - O.sht(maps[1].cpu().numpy().astype(np.float64), 16, 31, 31)) / np.linalg.norm(a0) < 3e-5


def test_ragged_inverse_matches_per_group(hpx, cuda):
    rng = np.random.default_rng(2)
    nsides, counts = [8, 4, 16], [2, 3, 4]
    alms = []
    for n, c in zip(nsides, counts):
        L = 2 * n - 1
        a = rng.standard_normal((c, L, L)) + 1j * rng.standard_normal((c, L, L))
        a = np.where(np.arange(L)[None, :] <= np.arange(L)[:, None], a, 0)
        alms.append(torch.from_numpy(a).to(cuda, torch.complex64))
    out = hpx.RaggedISHT(nsides)(alms)
    for a, f, n in zip(alms, out, nsides):
        assert torch.equal(f, hpx.iSHTCUDA(n, lmax=2 * n - 1, mmax=2 * n - 1)(a))


@pytest.mark.parametrize("prec", ["fp32", "f16x3"])
def test_ragged_graph_replay(hpx, cuda, prec):
    rng = np.random.default_rng(3)
    nsides, counts = [8, 32, 16], [2, 3, 4]
    eager = hpx.RaggedSHT(nsides, precision=prec)
    graphed = hpx.RaggedSHT(nsides, precision=prec, graph=True)
    for it in range(3):  # capture on the first call, replay with new inputs after
        maps = rand_maps(rng, nsides, counts, cuda)
        ref = eager(maps)
        got = graphed(maps)
        torch.cuda.synchronize()
        for a, b in zip(got, ref):
            assert torch.equal(a, b), it


def test_split_by_offsets(hpx, cuda):
    rng = np.random.default_rng(4)
    nsides = [4, 4, 8, 8, 8, 4]
    sizes = [12 * n * n for n in nsides]
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    flat = torch.from_numpy(rng.standard_normal(offsets[-1])).float().to(cuda)
    groups, gns = hpx.split_by_offsets(flat, offsets, nsides)
    assert gns == [4, 8, 4]
    assert [g.shape[0] for g in groups] == [2, 3, 1]
    assert groups[1].data_ptr() == flat[offsets[2]:].data_ptr()  # a view, no copy
    out = hpx.RaggedSHT(gns)(groups)
    assert torch.equal(out[1][2], hpx.SHTCUDA(8, lmax=15, mmax=15)(flat[offsets[4]:offsets[5]]))
    with pytest.raises(ValueError):
        hpx.split_by_offsets(flat, offsets, [4, 4, 8, 8, 4, 4])


def test_ragged_abi_errors(hpx, cuda):
    from cuhpx_b200 import _lib

    lib = _lib.load()
    plan = hpx.get_plan(4, 7, 7, "ring", "fp32", 0)
    ph = (ctypes.c_void_p * 2)(plan._h.value, None)
    pb = (ctypes.c_int64 * 2)(1, 1)
    need = ctypes.c_size_t()
    assert lib.hpx_ragged_workspace_size(ph, 2, pb, ctypes.byref(need)) == 1
    ph1 = (ctypes.c_void_p * 1)(plan._h.value)
    pb1 = (ctypes.c_int64 * 1)(-1)
    assert lib.hpx_ragged_workspace_size(ph1, 1, pb1, ctypes.byref(need)) == 1
    pb1 = (ctypes.c_int64 * 1)(2)
    assert lib.hpx_ragged_workspace_size(ph1, 1, pb1, ctypes.byref(need)) == 0
    nul = (ctypes.c_void_p * 1)(None)
    assert lib.hpx_ragged_forward(ph1, 1, nul, nul, pb1, None, 0, None) == 1


def test_ragged_concurrent_and_sequential_workspaces(hpx, cuda):
    """The groups run concurrently when the workspace holds all of them (the size
    hpx_ragged_workspace_size returns) and one after another in a workspace of the
    largest group's size; both give the per-group results bit for bit."""
    from cuhpx_b200 import _lib

    lib = _lib.load()
    rng = np.random.default_rng(6)
    nsides, counts = [16, 8, 32, 8], [3, 2, 5, 1]  # two groups share a plan
    maps = rand_maps(rng, nsides, counts, cuda)
    plans = [hpx.get_plan(n, 2 * n - 1, 2 * n - 1, "ring", "f16x3", 0) for n in nsides]
    outs = [torch.empty(c, 2 * n - 1, 2 * n - 1, dtype=torch.complex64, device=cuda) for n, c in zip(nsides, counts)]
    k = len(nsides)
    ph = (ctypes.c_void_p * k)(*[p._h.value for p in plans])
    pi = (ctypes.c_void_p * k)(*[m.data_ptr() for m in maps])
    po = (ctypes.c_void_p * k)(*[o.data_ptr() for o in outs])
    pb = (ctypes.c_int64 * k)(*counts)
    need = ctypes.c_size_t()
    assert lib.hpx_ragged_workspace_size(ph, k, pb, ctypes.byref(need)) == 0
    largest = max(p.workspace_bytes(c) for p, c in zip(plans, counts))
    assert need.value >= sum(p.workspace_bytes(c) for p, c in zip(plans, counts)) > largest
    refs = [hpx.SHTCUDA(n, lmax=2 * n - 1, mmax=2 * n - 1, precision="f16x3")(m) for n, m in zip(nsides, maps)]
    stream = torch.cuda.current_stream(cuda).cuda_stream
    for size in (need.value, largest):
        ws = torch.empty(size + 256, dtype=torch.uint8, device=cuda)
        base = (ws.data_ptr() + 255) & ~255
        for o in outs:
            o.fill_(float("nan"))
        st = lib.hpx_ragged_forward(ph, k, pi, po, pb, base, size, stream)
        assert st == 0, lib.hpx_last_error(None)
        torch.cuda.synchronize()
        for o, r in zip(outs, refs):
            assert torch.equal(o, r), size
    ws = torch.empty(largest - 256, dtype=torch.uint8, device=cuda)
    assert lib.hpx_ragged_forward(ph, k, pi, po, pb, (ws.data_ptr() + 255) & ~255, largest - 512, stream) == 6
