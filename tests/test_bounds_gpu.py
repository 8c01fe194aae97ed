"""The bounds-checked build: every checked access stays inside its buffer.

``libhpx_b200_bounds.so`` (``cuhpx_b200.build.build_variant("bounds")``,
``-DHPX_CHECK_BOUNDS``) checks the global accesses of the ring, fold/unfold,
layout, contraction-epilogue and spin-1 kernels against the extents of the
current chunk's buffers and reports a skipped access through
``hpx_plan_check`` (``HPX_ERR_BOUNDS``).  Small transforms of every kind run
through it here and must match the oracle with no access reported; then one
extent is shrunk by an element (``HPX_TEST_SHRINK_EXTENT``, read by the
checker build only) and the kernel's last access to that buffer must be
reported -- the check skips it, so nothing is read or written outside.
"""

import ctypes
import os

import numpy as np
import pytest
import torch

from cuhpx_b200 import _lib
from cuhpx_b200.build import VARIANTS
from cuhpx_b200.sht_tools import read_ring_weight
from oracle import hpx_oracle as O

pytestmark = pytest.mark.gpu

HPX_OK, HPX_ERR_BOUNDS = 0, 7
FP32, FP64, BF16X3, F16X3 = 0, 1, 2, 4
EXT_ALM = 3  # index of the coefficient extent (hpx_common.cuh HpxExtent)


@pytest.fixture(scope="module")
def blib(cuda):
    path = VARIANTS["bounds"][1]
    if not os.path.exists(path):
        pytest.skip("checker build libhpx_b200_bounds.so not built (cuhpx_b200.build.build_variant)")
    return _lib.load_path(path)


def make_plan(lib, nside, L, M, precision, flags=0):
    d = _lib.HpxDesc()
    d.nside, d.lmax, d.mmax, d.precision = nside, L, M, precision
    d.refine_iters, d.batch_chunk, d.device, d.flags = 0, 0, 0, flags
    w = np.ascontiguousarray(read_ring_weight(nside), dtype=np.float64)
    d.ring_weights = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    h = ctypes.c_void_p()
    assert lib.hpx_plan_create(ctypes.byref(d), ctypes.byref(h)) == HPX_OK, lib.hpx_last_error(None)
    return h


def call(lib, fn, plan, src, dst, batch, *extra):
    need = ctypes.c_size_t()
    assert lib.hpx_workspace_size(plan, batch, ctypes.byref(need)) == HPX_OK
    ws = torch.empty(need.value + 256, dtype=torch.uint8, device=src.device)
    base = (ws.data_ptr() + 255) & ~255
    stream = torch.cuda.current_stream(src.device).cuda_stream
    st = fn(plan, src.data_ptr(), dst.data_ptr(), batch, *extra, base, need.value, stream)
    assert st == HPX_OK, lib.hpx_last_error(plan)
    return lib.hpx_plan_check(plan, stream)


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# (nside, L, M, precision, flags, batch): SIMT, tensor-core table and on-the-fly, two chunks
CASES = [(8, 17, 17, FP32, 0, 3), (16, 33, 20, FP64, 0, 2), (16, 31, 31, F16X3, 0, 70), (32, 63, 63, BF16X3, 1, 5)]


@pytest.mark.parametrize("nside,L,M,prec,flags,batch", CASES)
def test_no_access_outside_buffers(blib, cuda, nside, L, M, prec, flags, batch):
    lib = blib
    plan = make_plan(lib, nside, L, M, prec, flags)
    try:
        dt = torch.float64 if prec == FP64 else torch.float32
        rng = np.random.default_rng(nside + L + prec)
        f = rng.standard_normal((batch, 12 * nside * nside))
        ref = O.sht(f[:2], nside, L, M)
        x = torch.from_numpy(f).to(cuda, dt)
        a = torch.zeros(batch, L, M, 2, dtype=dt, device=cuda)
        assert call(lib, lib.hpx_sht_forward, plan, x, a, batch) == HPX_OK
        got = torch.view_as_complex(a).cpu().numpy()[:2]
        assert rel(got, ref) < (1e-10 if prec == FP64 else 3e-5)
        g = torch.zeros_like(x)
        assert call(lib, lib.hpx_sht_inverse, plan, a, g, batch) == HPX_OK
        assert rel(g.cpu().numpy()[:2], O.isht(torch.view_as_complex(a).cpu().numpy()[:2].astype(np.complex128), nside)) < (
            1e-10 if prec == FP64 else 3e-5)
        assert call(lib, lib.hpx_sht_forward_refined, plan, x, a, batch, ctypes.c_int32(1)) == HPX_OK
        assert call(lib, lib.hpx_sht_forward_adjoint, plan, a, g, batch) == HPX_OK
        assert call(lib, lib.hpx_sht_inverse_adjoint, plan, x, a, batch) == HPX_OK
    finally:
        lib.hpx_plan_destroy(plan)


def test_spin1_no_access_outside_buffers(blib, cuda):
    from oracle import vector_oracle as V

    lib = blib
    nside, L, M, B = 8, 17, 13, 35  # two passes of vector maps
    plan = make_plan(lib, nside, L + 1, M + 1, FP64)
    try:
        rng = np.random.default_rng(3)
        f = rng.standard_normal((B, 2, 12 * nside * nside))
        x = torch.from_numpy(f).to(cuda)
        a = torch.zeros(B, 2, L, M, 2, dtype=torch.float64, device=cuda)
        assert call(lib, lib.hpx_vsht_forward, plan, x, a, B, ctypes.c_int32(1)) == HPX_OK
        assert rel(torch.view_as_complex(a).cpu().numpy()[:2], V.vsht(f[:2], nside, L, M)) < 1e-10
        g = torch.zeros_like(x)
        assert call(lib, lib.hpx_vsht_inverse, plan, a, g, B, ctypes.c_int32(1)) == HPX_OK
    finally:
        lib.hpx_plan_destroy(plan)


def test_shrunk_extent_is_reported(blib, cuda, monkeypatch):
    # one element less of the coefficient buffer: the last coefficient's store
    # is skipped and reported; everything else is written as usual
    lib = blib
    monkeypatch.setenv("HPX_TEST_SHRINK_EXTENT", str(EXT_ALM))
    plan = make_plan(lib, 8, 17, 17, FP32)
    try:
        x = torch.randn(2, 768, device=cuda)
        a = torch.zeros(2, 17, 17, 2, device=cuda)
        assert call(lib, lib.hpx_sht_forward, plan, x, a, 2) == HPX_ERR_BOUNDS
        assert b"out-of-bounds" in lib.hpx_last_error(plan)
        monkeypatch.delenv("HPX_TEST_SHRINK_EXTENT")
        assert lib.hpx_plan_check(plan, torch.cuda.current_stream(cuda).cuda_stream) == HPX_OK  # cleared
        assert call(lib, lib.hpx_sht_forward, plan, x, a, 2) == HPX_OK
    finally:
        lib.hpx_plan_destroy(plan)
