"""The C ABI library: built for sm_100a, loadable, exports every declared symbol.

No compute calls here -- these run on a machine without a GPU.
"""

import ctypes
import os
import re
import subprocess

import pytest

from cuhpx_b200 import _lib
from cuhpx_b200 import build as hpx_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hpx_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"HPX_API\s+(?:const\s+)?\w+\*?\s+(hpx_\w+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    hpx_build.build()
    return _lib.load()


def test_header_declares_api():
    syms = declared_symbols()
    for s in ("hpx_plan_create", "hpx_plan_destroy", "hpx_workspace_size", "hpx_sht_forward", "hpx_sht_inverse",
              "hpx_sht_forward_adjoint", "hpx_sht_inverse_adjoint", "hpx_sht_forward_refined", "hpx_last_error"):
        assert s in syms


def test_every_declared_symbol_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s+(hpx_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in declared_symbols():
        assert hasattr(lib, s)
    # binding table covers the header
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_library_is_sm100a_only(lib):
    out = subprocess.run(["cuobjdump", "--list-elf", _lib.LIB_PATH], capture_output=True, text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_status_strings_and_version(lib):
    assert lib.hpx_status_string(0) == b"ok"
    assert lib.hpx_status_string(6) == b"workspace too small"
    assert b"sm_100a" in lib.hpx_version()


def _desc(**kw):
    d = _lib.HpxDesc()
    d.nside, d.lmax, d.mmax, d.precision = 8, 17, 17, 0
    d.refine_iters, d.batch_chunk, d.device, d.flags = 0, 0, 0, 0
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize(
    "kw",
    [dict(nside=0), dict(lmax=0), dict(mmax=-1), dict(precision=9), dict(flags=4), dict(batch_chunk=-2), dict(refine_iters=-1)],
)
def test_plan_create_rejects_bad_descriptors(lib, kw):
    h = ctypes.c_void_p()
    st = lib.hpx_plan_create(ctypes.byref(_desc(**kw)), ctypes.byref(h))
    assert st == 1  # HPX_ERR_INVALID_ARG, decided before any CUDA call
    assert not h.value
    assert lib.hpx_last_error(None)


def test_null_arguments(lib):
    assert lib.hpx_plan_create(None, None) == 1
    assert lib.hpx_plan_destroy(None) == 0
    n = ctypes.c_size_t()
    assert lib.hpx_workspace_size(None, 1, ctypes.byref(n)) == 1
    assert lib.hpx_sht_forward(None, None, None, 1, None, 0, None) == 1
    assert lib.hpx_sht_forward_refined(None, None, None, 1, 1, None, 0, None) == 1


def test_no_gpu_is_a_status_not_a_crash(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = ctypes.c_void_p()
    st = lib.hpx_plan_create(ctypes.byref(_desc()), ctypes.byref(h))
    assert st == 3 and not h.value


def test_remap_rejects_bad_arguments_before_any_cuda_call(lib):
    """hpx_remap validates everything on the host first; none of these reaches the GPU."""
    RING, NEST, XY = 0, 1, 2
    a, b = ctypes.c_void_p(0x10000), ctypes.c_void_p(0x90000000)

    def call(inp=a, out=b, batch=1, nside=4, elem=4, so=NEST, sorg=0, scw=0, do=RING, dorg=0, dcw=0):
        return lib.hpx_remap(inp, out, batch, nside, elem, so, sorg, scw, do, dorg, dcw, None)

    assert call(batch=0) == 0  # nothing to do
    assert call(batch=-1) == 1
    for bad in (0, 3, 12, 16384):
        assert call(nside=bad) == 1
    assert b"power of two" in lib.hpx_last_error(None)
    for bad in (0, 3, 32):
        assert call(elem=bad) == 1
    assert call(so=3) == 1
    assert call(so=XY, sorg=4) == 1
    assert b"src origin" in lib.hpx_last_error(None)
    assert call(do=XY, dorg=-1) == 1
    assert b"dest origin" in lib.hpx_last_error(None)
    assert call(inp=ctypes.c_void_p(0)) == 1
    assert call(inp=ctypes.c_void_p(0x10002)) == 1  # not 4-byte aligned
    assert b"aligned" in lib.hpx_last_error(None)
    assert call(out=ctypes.c_void_p(0x10000 + 64)) == 1  # overlapping buffers
    assert b"overlap" in lib.hpx_last_error(None)
    # a byte count that would wrap 64 bits is refused before the overlap test
    assert call(batch=2**62, nside=8192, elem=16) == 1
    assert b"batch too large" in lib.hpx_last_error(None)
