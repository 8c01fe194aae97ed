"""Multi-threaded CPU port of cuHPX's CPU SHT / iSHT -- TEST INFRASTRUCTURE AND CPU BASELINE ONLY.

cuHPX's CPU transforms (cuhpx/hpx_sht.py:173-283) run, per call, one
``rfft``/``irfft`` per ring (cuhpx/hpx_sht.py:37-76, restated by
``hpx_oracle.ring_rfft``/``ring_irfft``) and a dense einsum of the ring
spectra with the precomputed Legendre table.  This module does the same with
the contraction in C (``ref_cpu.c``, OpenMP over the orders), regenerating
the table's values per order by the reference's recurrence instead of holding
it (68.6 GB at nside 1024, L = M = 2047).  ``sht_extended``/``isht_extended``
run the same recurrence in 80-bit extended precision at the rings' exact
nodes: at nside 1024 the reference's FP64 diagonal goes subnormal for high
orders near the poles and its recurrence then diverges (values up to ~40
where the true ones are ~1e-35), so large-nside parity is checked against
those.  It is what ``bench.py`` times as
the reference's CPU implementation; ``tests/test_oracle_golden.py`` checks it
against the golden-pinned oracle.  The product never imports it.

The shared library is compiled with gcc into ``oracle/_build`` on first use
(x86-64-v3: AVX2 and FMA).
"""

import ctypes
import os
import subprocess
import time

import numpy as np

from . import hpx_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ref_cpu.c")
OUT = os.path.join(HERE, "_build", "libhpx_ref_cpu.so")
_lib = None


def build(force=False):
    """Compile ``ref_cpu.c`` (gcc -O3 -fopenmp); returns the library path."""
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC", "-o", OUT + ".tmp", SRC, "-lm"]
    subprocess.run(cmd, check=True, capture_output=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


def load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(build())
        dp = ctypes.POINTER(ctypes.c_double)
        lib.hpx_ref_sht_contract.argtypes = [dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        lib.hpx_ref_isht_contract.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        lib.hpx_ref_sht_contract_ext.argtypes = [dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        lib.hpx_ref_isht_contract_ext.argtypes = [dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
        lib.hpx_ref_threads.restype = ctypes.c_int
        lib.hpx_ref_set_threads.argtypes = [ctypes.c_int]
        _lib = lib
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def set_threads(n):
    load().hpx_ref_set_threads(int(n))


def threads():
    return load().hpx_ref_threads()


def sht(f, nside, lmax, mmax, quad_weights="ring"):
    """Forward SHT of one map (float64): [npix] -> [L, M] complex (cuhpx/hpx_sht.py:214-236)."""
    lib = load()
    ftm = np.ascontiguousarray(O.ring_rfft(np.asarray(f, dtype=np.float64), mmax, nside))
    w = np.ascontiguousarray(O.ring_weights(nside, quad_weights))
    x = np.ascontiguousarray(np.cos(O.ring_theta(nside)))
    alm = np.empty((lmax, mmax), dtype=np.complex128)
    if lib.hpx_ref_sht_contract(_ptr(ftm.view(np.float64)), _ptr(w), _ptr(x), x.size, lmax, mmax,
                                _ptr(alm.view(np.float64))):
        raise MemoryError("ref_cpu: allocation failed")
    return alm


def sht_extended(f, nside, lmax, mmax, quad_weights="ring"):
    """Forward SHT of one map with the Legendre recurrence in 80-bit extended
    precision at the rings' z_t (sin^2 from ``hpx_oracle.ring_sin2``): the
    accurate analysis at large nside, where the reference's FP64 diagonal
    underflows for high orders near the poles."""
    lib = load()
    ftm = np.ascontiguousarray(O.ring_rfft(np.asarray(f, dtype=np.float64), mmax, nside))
    w = np.ascontiguousarray(O.ring_weights(nside, quad_weights))
    x = np.ascontiguousarray(O.ring_z(nside))
    s2 = np.ascontiguousarray(O.ring_sin2(nside))
    alm = np.empty((lmax, mmax), dtype=np.complex128)
    if lib.hpx_ref_sht_contract_ext(_ptr(ftm.view(np.float64)), _ptr(w), _ptr(x), _ptr(s2), x.size, lmax, mmax,
                                    _ptr(alm.view(np.float64))):
        raise MemoryError("ref_cpu: allocation failed")
    return alm


def isht(alm, nside):
    """Inverse SHT of one coefficient set: [L, M] complex -> [npix] (cuhpx/hpx_sht.py:268-283)."""
    lib = load()
    alm = np.ascontiguousarray(alm, dtype=np.complex128)
    L, M = alm.shape
    x = np.ascontiguousarray(np.cos(O.ring_theta(nside)))
    ftm = np.empty((x.size, M), dtype=np.complex128)
    if lib.hpx_ref_isht_contract(_ptr(alm.view(np.float64)), _ptr(x), x.size, L, M, _ptr(ftm.view(np.float64))):
        raise MemoryError("ref_cpu: allocation failed")
    return O.ring_irfft(ftm, M, nside)


def isht_extended(alm, nside):
    """Inverse SHT of one coefficient set with the Legendre recurrence in 80-bit
    extended precision at the rings' z_t (see ``sht_extended``)."""
    lib = load()
    alm = np.ascontiguousarray(alm, dtype=np.complex128)
    L, M = alm.shape
    x = np.ascontiguousarray(O.ring_z(nside))
    s2 = np.ascontiguousarray(O.ring_sin2(nside))
    ftm = np.empty((x.size, M), dtype=np.complex128)
    if lib.hpx_ref_isht_contract_ext(_ptr(alm.view(np.float64)), _ptr(x), _ptr(s2), x.size, L, M,
                                     _ptr(ftm.view(np.float64))):
        raise MemoryError("ref_cpu: allocation failed")
    return O.ring_irfft(ftm, M, nside)


def time_sht_isht(nside, lmax, mmax, seed=0):
    """Seconds for one float64 map's SHT followed by the iSHT of its result."""
    f = np.random.default_rng(seed).standard_normal(O.npix(nside))
    t0 = time.perf_counter()
    a = sht(f, nside, lmax, mmax)
    isht(a, nside)
    return time.perf_counter() - t0
