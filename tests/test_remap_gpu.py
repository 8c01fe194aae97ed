"""Pixel-order remapping through the C ABI (``hpx_remap``), bit-exact.

Checked against the CPU oracle (oracle/remap_oracle.py) for every function of
cuhpx/hpx_remap.py:24-102 and every flat orientation, against the reference's
own kernels when ``oracle/_ref/cuhpx_remap.so`` was built
(``python -m oracle.build_ref_remap``), and at the largest nside by
round trips.
"""

import itertools

import numpy as np
import pytest
import torch

from oracle import remap_oracle as R

pytestmark = pytest.mark.gpu

ORIGINS = "SENW"
ORIENTS = [(o, cw) for o in ORIGINS for cw in (False, True)]


@pytest.fixture(scope="module")
def rm(cuda):
    from cuhpx_b200 import remap

    return remap


def oracle_call(name, x, nside, *args):
    return getattr(R, name)(x, *args, nside) if args else getattr(R, name)(x, nside)


def gpu_call(rm, name, x, nside, *args):
    return getattr(rm, name)(x, *args, nside) if args else getattr(rm, name)(x, nside)


CASES = ([("ring2nest",), ("nest2ring",)] + [(f, o, cw) for f in ("nest2flat", "flat2nest", "ring2flat", "flat2ring")
                                              for o, cw in ORIENTS])


@pytest.mark.parametrize("nside", [1, 2, 4, 8, 16, 32, 64, 128])
def test_all_functions_vs_oracle(rm, cuda, nside):
    rng = np.random.default_rng(nside)
    npix = 12 * nside * nside
    for case in CASES:
        name, args = case[0], case[1:]
        for shape in [(npix,), (2, 3, npix)]:
            x = rng.integers(-2**31, 2**31 - 1, size=shape, dtype=np.int64).astype(np.int32)
            want = oracle_call(name, x, nside, *args)
            got = gpu_call(rm, name, torch.from_numpy(x).to(cuda), nside, *args)
            assert got.shape == x.shape and got.dtype == torch.int32
            assert np.array_equal(got.cpu().numpy(), want), (name, args, shape)


@pytest.mark.parametrize("nside", [1, 4, 32, 64])
def test_flat2flat_all_orientations(rm, cuda, nside):
    npix = 12 * nside * nside
    x = np.arange(2 * npix, dtype=np.int64).reshape(2, npix)
    xd = torch.from_numpy(x).to(cuda)
    for (so, scw), (do, dcw) in itertools.product(ORIENTS, ORIENTS):
        want = R.flat2flat(x, so, scw, do, dcw, nside)
        got = rm.flat2flat(xd, so, scw, do, dcw, nside)
        assert np.array_equal(got.cpu().numpy(), want), (so, scw, do, dcw)


@pytest.mark.parametrize("dtype", [torch.bool, torch.uint8, torch.int16, torch.float16, torch.bfloat16, torch.int32,
                                   torch.float32, torch.int64, torch.float64, torch.complex64, torch.complex128])
def test_every_element_width(rm, cuda, dtype):
    nside = 64
    npix = 12 * nside * nside
    g = torch.Generator().manual_seed(3)
    x = torch.randn(3, npix, generator=g, dtype=torch.float64)
    if dtype == torch.bool:
        x = x > 0
    elif dtype.is_complex:
        x = torch.complex(x, torch.randn(3, npix, generator=g, dtype=torch.float64)).to(dtype)
    else:
        x = (x * 100).to(dtype)
    xd = x.to(cuda)
    host = x.view(torch.int16).numpy() if dtype == torch.bfloat16 else x.numpy()
    for name, args in [("nest2ring", ()), ("ring2flat", ("N", True)), ("flat2nest", ("E", False))]:
        want = torch.from_numpy(oracle_call(name, host, nside, *args))
        got = gpu_call(rm, name, xd, nside, *args).cpu()
        if dtype == torch.bfloat16:
            got = got.view(torch.int16)
        assert torch.equal(got, want), (dtype, name)


def test_reference_kernels_agree(rm, cuda):
    """The reference's own cuhpx_remap, compiled from its sources, gives the same bytes."""
    from oracle import build_ref_remap

    ref = build_ref_remap.load()
    if ref is None:
        pytest.skip("oracle/_ref/cuhpx_remap.so not built")
    ours = {"nest2xy": "nest2flat", "xy2nest": "flat2nest", "ring2xy": "ring2flat", "xy2ring": "flat2ring"}
    for nside in (1, 2, 8, 32, 64):
        npix = 12 * nside * nside
        x1 = torch.arange(npix, dtype=torch.int64, device=cuda)
        xb = torch.randn(4, npix, device=cuda)
        for name, args in [("ring2nest", ()), ("nest2ring", ())] + [(f, a) for f in ours for a in ORIENTS]:
            for x in (x1, xb):
                fn = getattr(ref, name if x.dim() == 1 else name + "_batch")
                want = fn(x, *args, nside, npix)
                got = gpu_call(rm, ours.get(name, name), x, nside, *args)
                torch.cuda.synchronize()
                assert torch.equal(got, want), (nside, name, args, x.dim())
        for (so, scw), (do, dcw) in itertools.product(ORIENTS, ORIENTS):
            want = ref.xy2xy_batch(xb, so, scw, do, dcw, nside, npix)
            assert torch.equal(rm.flat2flat(xb, so, scw, do, dcw, nside), want), (nside, so, scw, do, dcw)


def test_nside_1024_batch(rm, cuda):
    nside, B = 1024, 8
    npix = 12 * nside * nside
    g = torch.Generator(device=cuda).manual_seed(5)
    x = torch.randn(B, npix, device=cuda, generator=g)
    y = rm.nest2ring(x, nside)
    want = R.nest2ring(x[1].cpu().numpy(), nside)
    assert np.array_equal(y[1].cpu().numpy(), want)
    assert torch.equal(rm.ring2nest(y, nside), x)
    z = rm.ring2flat(y, "W", True, nside)
    assert torch.equal(rm.flat2nest(z, "W", True, nside), x)


def test_largest_nside_round_trip(rm, cuda):
    """nside 8192: 805,306,368 pixels, offsets up to 2**29.6."""
    nside = 8192
    npix = 12 * nside * nside
    x = torch.arange(npix, dtype=torch.int32, device=cuda)
    r = rm.nest2ring(x, nside)
    idx = np.array([0, 1, 12345, npix // 2, npix - 2, npix - 1], dtype=np.int64)
    ring_of = R.xyf2ring(*R.nest2xyf(idx, nside), nside)
    assert np.array_equal(r[torch.from_numpy(ring_of).to(cuda)].cpu().numpy(), idx)
    assert torch.equal(rm.ring2nest(r, nside), x)
    del r


def test_layout_and_stream_semantics(rm, cuda):
    nside = 16
    npix = 12 * nside * nside
    x = torch.randn(npix, 5, device=cuda).t()  # non-contiguous batch of 5 maps
    want = R.nest2ring(x.cpu().numpy(), nside)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        y = rm.nest2ring(x, nside)
    s.synchronize()
    assert np.array_equal(y.cpu().numpy(), want)
    empty = rm.ring2nest(torch.empty(0, npix, device=cuda), nside)
    assert empty.shape == (0, npix)
    same = rm.flat2flat(x, "N", True, "N", True, nside)
    assert torch.equal(same, x)


def test_argument_errors(rm, cuda):
    with pytest.raises(ValueError, match="power of two"):
        rm.ring2nest(torch.zeros(12 * 9, device=cuda), 3)
    with pytest.raises(RuntimeError, match="number of elements"):
        rm.nest2ring(torch.zeros(49, device=cuda), 2)
    with pytest.raises(RuntimeError, match="S, E, N, W"):
        rm.nest2flat(torch.zeros(48, device=cuda), "X", False, 2)
    with pytest.raises(RuntimeError, match="dest origin"):
        rm.flat2flat(torch.zeros(48, device=cuda), "S", False, "Q", False, 2)
    with pytest.raises(RuntimeError, match="CUDA tensor"):
        rm.ring2nest(torch.zeros(48), 2)


@pytest.mark.parametrize("dtype", [torch.float32, torch.int64, torch.complex64])
def test_unaligned_buffers_vs_oracle(cuda, dtype):
    """Buffers that start one element past a 16-byte boundary take the
    per-element staging path of the kernel (no 16-byte accesses); called
    through the C ABI on views, since the Python wrappers pass fresh tensors.
    (16-byte elements are always 16-byte aligned, so they never take it.)"""
    import ctypes

    from cuhpx_b200 import _lib

    lib = _lib.load()
    RING, NEST, XY = 0, 1, 2
    nside, B = 64, 3
    npix = 12 * nside * nside
    g = torch.Generator().manual_seed(11)
    x = torch.randn(B, npix, generator=g, dtype=torch.float64)
    if dtype.is_complex:
        x = torch.complex(x, torch.randn(B, npix, generator=g, dtype=torch.float64))
    x = (x * 1000).to(dtype)
    src_buf = torch.zeros(B * npix + 1, dtype=dtype, device=cuda)
    dst_buf = torch.zeros(B * npix + 1, dtype=dtype, device=cuda)
    src = src_buf[1:]
    dst = dst_buf[1:]
    src.copy_(x.reshape(-1).to(cuda))
    assert src.data_ptr() % 16 != 0 and dst.data_ptr() % 16 != 0
    host = x.numpy()
    pairs = [
        ((NEST, 0, 0), (XY, 1, 1), lambda h: R.nest2flat(h, "E", True, nside)),
        ((XY, 2, 0), (NEST, 0, 0), lambda h: R.flat2nest(h, "N", False, nside)),
        ((XY, 0, 1), (XY, 3, 0), lambda h: R.flat2flat(h, "S", True, "W", False, nside)),
        ((NEST, 0, 0), (RING, 0, 0), lambda h: R.nest2ring(h, nside)),
        ((RING, 0, 0), (XY, 2, 1), lambda h: R.ring2flat(h, "N", True, nside)),
    ]
    stream = torch.cuda.current_stream(cuda).cuda_stream
    for (so, sorg, scw), (do, dorg, dcw), ref in pairs:
        st = lib.hpx_remap(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), B, nside,
                           src.element_size(), so, sorg, scw, do, dorg, dcw, ctypes.c_void_p(stream))
        assert st == 0, lib.hpx_last_error(None)
        torch.cuda.synchronize()
        got = dst.reshape(B, npix).cpu().numpy()
        assert np.array_equal(got, ref(host)), (so, do)
    assert dst_buf[0].item() == 0  # nothing written before the view
