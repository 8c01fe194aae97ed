"""hpx_b200: HEALPix spherical-harmonic transforms for NVIDIA B200 (sm_100a).

Drop-in for the SHT path of cuHPX: ``SHTCUDA``, ``iSHTCUDA``, the spin-1
``VectorSHTCUDA`` / ``VectoriSHTCUDA``, ``Grid`` and ``Regridding``, and for its pixel-order remapping (``ring2nest``,
``nest2ring``, ``nest2flat``, ``flat2nest``, ``ring2flat``, ``flat2ring``,
``flat2flat``), with the healpy a_lm packing beside them (``alm_to_healpy``,
``healpy_to_alm``).  The transforms run in ``libhpx_b200.so`` (hand-written CUDA,
C ABI in ``include/hpx_b200.h``); there is no CPU fallback.
"""

from . import sht_tools
from .healpy_alm import alm_to_healpy, healpy_index, healpy_size, healpy_to_alm
from .hpx_sht import (LatLonPlan, Plan, SHTCUDA, SHTFunction, clear_plan_cache, get_latlon_plan, get_plan, iSHTCUDA,
                      iSHTFunction)
from .latlon import InverseRealSHT, RealSHT
from .ragged import RaggedISHT, RaggedSHT, split_by_offsets
from .regrid import Grid, Regridding
from .remap import flat2flat, flat2nest, flat2ring, nest2flat, nest2ring, ring2flat, ring2nest
from .vector import VectoriSHTCUDA, VectorSHTCUDA

__all__ = [
    "SHTCUDA",
    "iSHTCUDA",
    "VectorSHTCUDA",
    "VectoriSHTCUDA",
    "SHTFunction",
    "iSHTFunction",
    "Plan",
    "LatLonPlan",
    "get_latlon_plan",
    "RealSHT",
    "InverseRealSHT",
    "Grid",
    "Regridding",
    "RaggedSHT",
    "RaggedISHT",
    "split_by_offsets",
    "get_plan",
    "clear_plan_cache",
    "sht_tools",
    "ring2nest",
    "nest2ring",
    "nest2flat",
    "flat2nest",
    "ring2flat",
    "flat2ring",
    "flat2flat",
    "alm_to_healpy",
    "healpy_to_alm",
    "healpy_size",
    "healpy_index",
]
