"""ctypes binding of ``libhpx_b200.so`` (the C ABI in ``include/hpx_b200.h``).

The shared library is the product's compute path.  There is no fallback: if
the library is missing or cannot be loaded, every transform raises.
"""

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhpx_b200.so")

HPX_OK = 0
STATUS = {
    0: "ok",
    1: "invalid argument",
    2: "out of memory",
    3: "CUDA error",
    4: "timeout",
    5: "unsupported",
    6: "workspace too small",
    7: "out-of-bounds access",
}

FLAG_OTF_LEGENDRE = 1

PRECISIONS = {"fp32": 0, "fp64": 1, "bf16x3": 2, "tf32": 3, "f16x3": 4}

GRIDS = {"equiangular": 0, "legendre-gauss": 1, "lobatto": 2}


class HpxLatLonDesc(ctypes.Structure):
    _fields_ = [
        ("nlat", ctypes.c_int32),
        ("nlon", ctypes.c_int32),
        ("lmax", ctypes.c_int32),
        ("mmax", ctypes.c_int32),
        ("grid", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("batch_chunk", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


# exported symbols and their signatures (argtypes, restype)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_sz = ctypes.c_size_t


class HpxDesc(ctypes.Structure):
    _fields_ = [
        ("nside", ctypes.c_int32),
        ("lmax", ctypes.c_int32),
        ("mmax", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("refine_iters", ctypes.c_int32),
        ("batch_chunk", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("ring_weights", ctypes.POINTER(ctypes.c_double)),
    ]


class HpxSchedule(ctypes.Structure):
    _fields_ = [
        ("ring_maps_per_cta", ctypes.c_int32),
        ("fwd_deal", ctypes.c_int32),
        ("inv_deal", ctypes.c_int32),
        ("ctas", ctypes.c_int32),
        ("ring_streams", ctypes.c_int32),
    ]


DEALS = {"order_snake": 0, "tile_snake": 1, "greedy": 2, "contiguous": 3}


class HpxStageStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("launches", ctypes.c_int64), ("total_ms", ctypes.c_double)]


SIGNATURES = {
    "hpx_stats_enable": ([_vp, ctypes.c_int], ctypes.c_int),
    "hpx_plan_check": ([_vp, _vp], ctypes.c_int),
    "hpx_stats_read": ([_vp, ctypes.POINTER(HpxStageStat), ctypes.c_int, ctypes.POINTER(ctypes.c_int)], ctypes.c_int),
    "hpx_plan_create": ([ctypes.POINTER(HpxDesc), ctypes.POINTER(_vp)], ctypes.c_int),
    "hpx_plan_destroy": ([_vp], ctypes.c_int),
    "hpx_workspace_size": ([_vp, _i64, ctypes.POINTER(_sz)], ctypes.c_int),
    "hpx_sht_forward": ([_vp, _vp, _vp, _i64, _vp, _sz, _vp], ctypes.c_int),
    "hpx_sht_inverse": ([_vp, _vp, _vp, _i64, _vp, _sz, _vp], ctypes.c_int),
    "hpx_sht_forward_adjoint": ([_vp, _vp, _vp, _i64, _vp, _sz, _vp], ctypes.c_int),
    "hpx_sht_inverse_adjoint": ([_vp, _vp, _vp, _i64, _vp, _sz, _vp], ctypes.c_int),
    "hpx_sht_forward_refined": ([_vp, _vp, _vp, _i64, ctypes.c_int32, _vp, _sz, _vp], ctypes.c_int),
    "hpx_sht_forward_noalloc": ([_vp, _vp, _vp, _i64, _vp], ctypes.c_int),
    "hpx_vsht_forward": ([_vp, _vp, _vp, _i64, ctypes.c_int32, _vp, _sz, _vp], ctypes.c_int),
    "hpx_vsht_inverse": ([_vp, _vp, _vp, _i64, ctypes.c_int32, _vp, _sz, _vp], ctypes.c_int),
    "hpx_vsht_forward_adjoint": ([_vp, _vp, _vp, _i64, ctypes.c_int32, _vp, _sz, _vp], ctypes.c_int),
    "hpx_vsht_inverse_adjoint": ([_vp, _vp, _vp, _i64, ctypes.c_int32, _vp, _sz, _vp], ctypes.c_int),
    "hpx_plan_get_schedule": ([_vp, ctypes.POINTER(HpxSchedule)], ctypes.c_int),
    "hpx_plan_set_schedule": ([_vp, ctypes.POINTER(HpxSchedule)], ctypes.c_int),
    "hpx_plan_table_bytes": ([_vp, ctypes.POINTER(_sz)], ctypes.c_int),
    "hpx_plan_table_stream_bytes": ([_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz)], ctypes.c_int),
    "hpx_plan_create_latlon": ([ctypes.POINTER(HpxLatLonDesc), ctypes.POINTER(_vp)], ctypes.c_int),
    "hpx_ragged_workspace_size": ([ctypes.POINTER(_vp), ctypes.c_int32, ctypes.POINTER(_i64), ctypes.POINTER(_sz)],
                                  ctypes.c_int),
    "hpx_ragged_forward": ([ctypes.POINTER(_vp), ctypes.c_int32, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                            ctypes.POINTER(_i64), _vp, _sz, _vp], ctypes.c_int),
    "hpx_ragged_inverse": ([ctypes.POINTER(_vp), ctypes.c_int32, ctypes.POINTER(_vp), ctypes.POINTER(_vp),
                            ctypes.POINTER(_i64), _vp, _sz, _vp], ctypes.c_int),
    "hpx_remap": ([_vp, _vp, _i64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                   ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp], ctypes.c_int),
    "hpx_alm_to_healpy": ([_vp, _vp, _i64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp],
                          ctypes.c_int),
    "hpx_healpy_to_alm": ([_vp, _vp, _i64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _vp],
                          ctypes.c_int),
    "hpx_plan_info": (
        [_vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
        ctypes.c_int,
    ),
    "hpx_last_error": ([_vp], ctypes.c_char_p),
    "hpx_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "hpx_version": ([], ctypes.c_char_p),
}

_lock = threading.Lock()
_lib = None


class HpxError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"hpx_b200: {STATUS.get(status, status)}: {message}")
        self.status = status


def load():
    """Load the library once; raise if it is missing (no silent fallback)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cuhpx_b200.build` "
                "(the transforms have no CPU fallback)"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


def load_path(path):
    """A separate copy of the library from `path` (a checker build), with the
    same signatures; it shares no state with the one load() returns."""
    lib = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


def check(status, plan=None):
    if status != HPX_OK:
        lib = load()
        msg = lib.hpx_last_error(plan).decode(errors="replace")
        raise HpxError(status, msg)
