"""hpx_sht_forward_noalloc: the analysis entry point that allocates nothing.

Called through the C ABI (ctypes) and compared, element for element, with
hpx_sht_forward given its own workspace.  Two calls in a row with different
maps check that nothing one call leaves in the shared static scratch reaches
the next.  The file sorts last so it also runs after every other GPU test has
used the library on the same device.
"""

import ctypes

import numpy as np
import pytest
import torch

from cuhpx_b200 import _lib
from cuhpx_b200.sht_tools import read_ring_weight

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 32 << 20
HPX_OK, HPX_ERR_INVALID_ARG, HPX_ERR_WORKSPACE = 0, 1, 6


@pytest.fixture(scope="module")
def lib(cuda):
    return _lib.load()


def make_plan(lib, nside, L, M, precision, weights=True):
    d = _lib.HpxDesc()
    d.nside, d.lmax, d.mmax, d.precision = nside, L, M, precision
    d.refine_iters, d.batch_chunk, d.device, d.flags = 0, 0, 0, 0
    w = None
    if weights:
        w = np.ascontiguousarray(read_ring_weight(nside), dtype=np.float64)
        d.ring_weights = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    h = ctypes.c_void_p()
    _lib.check(lib.hpx_plan_create(ctypes.byref(d), ctypes.byref(h)))
    return h


def forward_ws(lib, plan, f, alm, stream):
    need = ctypes.c_size_t()
    _lib.check(lib.hpx_workspace_size(plan, f.shape[0], ctypes.byref(need)), plan)
    ws = torch.empty(need.value + 256, dtype=torch.uint8, device=f.device)
    base = (ws.data_ptr() + 255) & ~255
    _lib.check(lib.hpx_sht_forward(plan, f.data_ptr(), alm.data_ptr(), f.shape[0], base, need.value, stream), plan)


# (nside, L, M, precision, batch): FP32, BF16X3, F16X3 and FP64 plans; batches of one
# chunk, a partial chunk and two chunks (the second one partial)
CASES = [
    (16, 33, 33, 0, 5),
    (32, 64, 64, 0, 64),
    (32, 65, 65, 2, 70),
    (64, 128, 128, 2, 64),
    (32, 65, 65, 4, 70),
    (16, 33, 33, 1, 3),
    (32, 64, 64, 1, 66),
]


@pytest.mark.parametrize("nside,L,M,prec,batch", CASES)
def test_noalloc_matches_forward_twice(lib, cuda, nside, L, M, prec, batch):
    dt = torch.float64 if prec == 1 else torch.float32
    plan = make_plan(lib, nside, L, M, prec)
    try:
        stream = torch.cuda.current_stream(cuda).cuda_stream
        g = torch.Generator(device="cpu").manual_seed(nside * 1000 + L + prec)
        maps = [torch.randn(batch, 12 * nside * nside, generator=g, dtype=torch.float64).to(cuda, dt) for _ in range(2)]
        for f in maps:
            ref = torch.empty(batch, L, M, 2, dtype=dt, device=cuda)
            forward_ws(lib, plan, f, ref, stream)
            out = torch.full((batch, L, M, 2), float("nan"), dtype=dt, device=cuda)
            _lib.check(lib.hpx_sht_forward_noalloc(plan, f.data_ptr(), out.data_ptr(), batch, stream), plan)
            _lib.check(lib.hpx_plan_check(plan, stream), plan)
            torch.cuda.synchronize()
            assert torch.isfinite(out).all()
            assert torch.equal(out, ref), float((out - ref).abs().max())
    finally:
        lib.hpx_plan_destroy(plan)


def make_latlon_plan(lib, nlat, nlon, L, M, precision, grid=0):
    d = _lib.HpxLatLonDesc()
    d.nlat, d.nlon, d.lmax, d.mmax, d.grid, d.precision = nlat, nlon, L, M, grid, precision
    d.batch_chunk, d.device, d.flags, d.reserved = 0, 0, 0, 0
    h = ctypes.c_void_p()
    _lib.check(lib.hpx_plan_create_latlon(ctypes.byref(d), ctypes.byref(h)))
    return h


# latitude-longitude plans take the same scratch layout: (nlat, nlon, L, M, precision, batch, grid)
LATLON = [(32, 64, 32, 32, 0, 5, 0), (32, 64, 32, 32, 2, 70, 0), (33, 64, 30, 20, 4, 3, 1)]


@pytest.mark.parametrize("nlat,nlon,L,M,prec,batch,grid", LATLON)
def test_noalloc_latlon_matches_forward_twice(lib, cuda, nlat, nlon, L, M, prec, batch, grid):
    plan = make_latlon_plan(lib, nlat, nlon, L, M, prec, grid)
    try:
        stream = torch.cuda.current_stream(cuda).cuda_stream
        g = torch.Generator(device="cpu").manual_seed(nlat * 100 + prec)
        for _ in range(2):
            f = torch.randn(batch, nlat * nlon, generator=g).to(cuda)
            ref = torch.empty(batch, L, M, 2, device=cuda)
            forward_ws(lib, plan, f, ref, stream)
            out = torch.full((batch, L, M, 2), float("nan"), device=cuda)
            _lib.check(lib.hpx_sht_forward_noalloc(plan, f.data_ptr(), out.data_ptr(), batch, stream), plan)
            _lib.check(lib.hpx_plan_check(plan, stream), plan)
            torch.cuda.synchronize()
            assert torch.equal(out, ref), float((out - ref).abs().max())
    finally:
        lib.hpx_plan_destroy(plan)


def test_noalloc_refuses_plans_above_scratch(lib, cuda):
    # FP32, nside 64, lmax = mmax = 192: about 36 MiB per chunk of 64 maps
    plan = make_plan(lib, 64, 192, 192, 0)
    try:
        f = torch.zeros(1, 12 * 64 * 64, device=cuda)
        alm = torch.zeros(1, 192, 192, 2, device=cuda)
        st = lib.hpx_sht_forward_noalloc(plan, f.data_ptr(), alm.data_ptr(), 1, None)
        assert st == HPX_ERR_WORKSPACE
        msg = lib.hpx_last_error(plan).decode()
        assert str(SCRATCH_BYTES) in msg and "hpx_sht_forward" in msg
        assert torch.count_nonzero(alm) == 0
        # the same plan still works through the workspace entry point
        forward_ws(lib, plan, f, alm, torch.cuda.current_stream(cuda).cuda_stream)
    finally:
        lib.hpx_plan_destroy(plan)


def test_noalloc_argument_errors(lib, cuda):
    plan = make_plan(lib, 8, 17, 17, 0)
    try:
        assert lib.hpx_sht_forward_noalloc(None, 1, 1, 1, None) == HPX_ERR_INVALID_ARG
        assert lib.hpx_sht_forward_noalloc(plan, None, 1, 1, None) == HPX_ERR_INVALID_ARG
        assert lib.hpx_sht_forward_noalloc(plan, 1, 1, -1, None) == HPX_ERR_INVALID_ARG
        assert lib.hpx_sht_forward_noalloc(plan, None, None, 0, None) == HPX_OK
    finally:
        lib.hpx_plan_destroy(plan)
