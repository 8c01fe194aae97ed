"""Failure detection on the GPU: a pipeline wait that runs out ends the call with a status.

Every wait of the tensor-core kernels on an mbarrier is bounded: past its
limit it records an error code in the plan's device flag, the kernel drains
what it issued and returns, and ``hpx_plan_check`` reports HPX_ERR_TIMEOUT.
This test makes such a wait run out without faulting or hanging anything: it
loads a checker build of the library (``libhpx_b200_waittest.so``, built by
``cuhpx_b200.build.build_variant("waittest")``) in which the limit is 1 ms and
the TMA thread announces each pipeline stage but issues none of its loads, so
the barrier the MMA thread waits on never completes.  The call must come back
with the timeout status, quickly, with the flag cleared afterwards, and the
device must stay usable: the same checker library's SIMT path and the product
library both give correct transforms on it afterwards.
"""

import ctypes
import os
import time

import numpy as np
import pytest
import torch

from cuhpx_b200 import _lib
from cuhpx_b200.build import VARIANTS
from oracle import hpx_oracle as O

pytestmark = pytest.mark.gpu

HPX_OK, HPX_ERR_TIMEOUT = 0, 4
FP32, BF16X3, F16X3 = 0, 2, 4
OTF = 1
NSIDE, L = 8, 17
NPIX = 12 * NSIDE * NSIDE


@pytest.fixture(scope="module")
def waitlib(cuda):
    path = VARIANTS["waittest"][1]
    if not os.path.exists(path):
        pytest.skip("checker build libhpx_b200_waittest.so not built (cuhpx_b200.build.build_variant)")
    return _lib.load_path(path)


def make_plan(lib, precision, flags=0):
    d = _lib.HpxDesc()
    d.nside, d.lmax, d.mmax, d.precision = NSIDE, L, L, precision
    d.refine_iters, d.batch_chunk, d.device, d.flags = 0, 0, 0, flags
    h = ctypes.c_void_p()
    st = lib.hpx_plan_create(ctypes.byref(d), ctypes.byref(h))
    assert st == HPX_OK, lib.hpx_last_error(None)
    return h


def call(lib, fn, plan, src, dst, batch, stream):
    need = ctypes.c_size_t()
    assert lib.hpx_workspace_size(plan, batch, ctypes.byref(need)) == HPX_OK
    ws = torch.empty(need.value + 256, dtype=torch.uint8, device=src.device)
    base = (ws.data_ptr() + 255) & ~255
    st = fn(plan, src.data_ptr(), dst.data_ptr(), batch, base, need.value, stream)
    return st, ws


@pytest.mark.parametrize("precision,flags", [(F16X3, 0), (BF16X3, 0), (F16X3, OTF)])
def test_tensor_core_wait_runs_out_with_a_status(waitlib, cuda, precision, flags):
    lib = waitlib
    plan = make_plan(lib, precision, flags)
    try:
        stream = torch.cuda.current_stream(cuda).cuda_stream
        f = torch.randn(3, NPIX, device=cuda)
        alm = torch.zeros(3, L, L, 2, device=cuda)
        for fn, src, dst in ((lib.hpx_sht_forward, f, alm), (lib.hpx_sht_inverse, alm, f)):
            t0 = time.perf_counter()
            st, ws = call(lib, fn, plan, src, dst, 3, stream)
            assert st == HPX_OK  # the launches themselves succeed
            st = lib.hpx_plan_check(plan, stream)
            elapsed = time.perf_counter() - t0
            assert st == HPX_ERR_TIMEOUT, lib.hpx_last_error(plan)
            assert b"timed out" in lib.hpx_last_error(plan)
            assert elapsed < 10.0
            # the flag was cleared by the check
            assert lib.hpx_plan_check(plan, stream) == HPX_OK
            del ws
        torch.cuda.synchronize()
    finally:
        lib.hpx_plan_destroy(plan)


def test_device_usable_after_timeouts(waitlib, cuda):
    rng = np.random.default_rng(5)
    f = rng.standard_normal((2, NPIX))
    stream = torch.cuda.current_stream(cuda).cuda_stream
    # the checker library's SIMT path has no pipeline waits and computes normally
    # (its plans here carry no ring weights: uniform quadrature)
    ref = O.sht(f, NSIDE, L, L, quad_weights="none")
    plan = make_plan(waitlib, FP32)
    try:
        x = torch.from_numpy(f).float().to(cuda)
        a = torch.zeros(2, L, L, 2, device=cuda)
        st, ws = call(waitlib, waitlib.hpx_sht_forward, plan, x, a, 2, stream)
        assert st == HPX_OK and waitlib.hpx_plan_check(plan, stream) == HPX_OK
        got = torch.view_as_complex(a).cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5
    finally:
        waitlib.hpx_plan_destroy(plan)
    # and the product library's tensor-core path on the same device
    import cuhpx_b200 as hpx

    ref = O.sht(f, NSIDE, L, L)

    got = hpx.SHTCUDA(NSIDE, lmax=L, mmax=L, precision="f16x3")(torch.from_numpy(f).float().to(cuda))
    err = np.linalg.norm(got.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < 2e-6
    torch.cuda.synchronize()
