"""Drop-in ``SHTCUDA`` / ``iSHTCUDA`` modules backed by the hpx_b200 CUDA library.

Mirrors the reference interface (cuhpx/hpx_sht.py:644-735):

* ``SHTCUDA(nside, lmax=None, mmax=None, quad_weights="ring", norm="ortho", csphase=True)``
  maps a real ``[..., 12*nside**2]`` CUDA tensor to complex ``[..., lmax, mmax]``
  (``lmax`` defaults to ``4*nside-1``, ``mmax`` to ``2*nside+1``).  Complex
  input raises ``ValueError``; a machine without CUDA raises ``RuntimeError``.
* ``iSHTCUDA(...)`` maps complex ``[..., lmax, mmax]`` back to a real map.
* float32 data run the FP32 path (or the requested mixed precision), float64
  data run the FP64 path; leading dimensions are batch dimensions and a 1-D
  input gives a 2-D output, as in the reference.
* ``norm`` and ``csphase`` are accepted and, as on the reference's CUDA path,
  do not change the result (orthonormal, no Condon-Shortley phase).

Differences from the reference, all deliberate:

* transforms run on the *current* CUDA stream at call time (the reference
  pins the stream that was current at construction);
* gradients are the exact adjoints of the transforms (the reference's
  hand-written backward is approximate, cuhpx/hpx_sht.py:565-583, 614-641);
* keyword-only extras: ``precision`` ('fp32'; 'f16x3' or 'bf16x3': tcgen05
  tensor cores with a three-term fp16 (per-map power-of-two scaled, ~22-bit)
  or bf16 (~16-bit) split and FP32 accumulation),
  ``refine_iters`` (Jacobi refinement of the analysis), ``batch_chunk``,
  ``legendre_table`` (tensor-core plans: keep the Legendre values resident on
  the device when they fit, default; False generates them on the fly),
  ``autotune`` (time the plan's launch schedules once and keep the fastest,
  cached on disk: ``cuhpx_b200.autotune``).
"""

import ctypes
import threading

import numpy as np
import torch
import torch.nn as nn

from . import _lib
from .sht_tools import read_ring_weight

_plan_lock = threading.Lock()
_plans = {}


class Plan:
    """One ``hpx_plan_t``: immutable, shareable between modules and streams."""

    def __init__(self, nside, lmax, mmax, quad_weights="ring", precision="fp32", device=0, batch_chunk=64, refine_iters=0,
                 legendre_table=True):
        lib = _lib.load()
        if precision not in _lib.PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}; expected one of {sorted(_lib.PRECISIONS)}")
        self.nside, self.lmax, self.mmax = int(nside), int(lmax), int(mmax)
        self.precision = precision
        self.device = int(device)
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.cdtype = torch.complex128 if precision == "fp64" else torch.complex64
        self.npix = 12 * self.nside * self.nside
        desc = _lib.HpxDesc()
        desc.nside = self.nside
        desc.lmax = self.lmax
        desc.mmax = self.mmax
        desc.precision = _lib.PRECISIONS[precision]
        desc.refine_iters = int(refine_iters)
        desc.batch_chunk = int(batch_chunk)
        desc.device = self.device
        desc.flags = 0 if legendre_table else _lib.FLAG_OTF_LEGENDRE
        self._w = None
        if quad_weights == "ring":
            self._w = np.ascontiguousarray(read_ring_weight(self.nside), dtype=np.float64)
            desc.ring_weights = self._w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        handle = ctypes.c_void_p()
        _lib.check(lib.hpx_plan_create(ctypes.byref(desc), ctypes.byref(handle)))
        self._h = handle
        self._lib = lib

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.hpx_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    def check(self, device=None):
        """Synchronise and raise if a kernel gave up on a bounded pipeline wait."""
        dev = torch.device("cuda", self.device) if device is None else device
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(self._lib.hpx_plan_check(self._h, ctypes.c_void_p(stream)), self._h)

    @property
    def table_bytes(self):
        """Bytes of the resident Legendre table (0: values generated on the fly)."""
        n = ctypes.c_size_t()
        _lib.check(self._lib.hpx_plan_table_bytes(self._h, ctypes.byref(n)), self._h)
        return n.value

    @property
    def table_stream_bytes(self):
        """(analysis, synthesis): table bytes one pass over a chunk of maps streams
        (all-zero table blocks are skipped); (0, 0) without a table."""
        f, i = ctypes.c_size_t(), ctypes.c_size_t()
        _lib.check(self._lib.hpx_plan_table_stream_bytes(self._h, ctypes.byref(f), ctypes.byref(i)), self._h)
        return f.value, i.value

    # ------------------------------------------------------------------ stats
    def stats_enable(self, on=True):
        _lib.check(self._lib.hpx_stats_enable(self._h, 1 if on else 0), self._h)

    def stats_read(self):
        """{stage: (launches, total_ms)} since the last read (synchronises on the events)."""
        arr = (_lib.HpxStageStat * 16)()
        n = ctypes.c_int()
        _lib.check(self._lib.hpx_stats_read(self._h, arr, 16, ctypes.byref(n)), self._h)
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(min(n.value, 16))}

    # ------------------------------------------------------------------ calls
    def workspace_bytes(self, batch):
        n = ctypes.c_size_t()
        _lib.check(self._lib.hpx_workspace_size(self._h, int(batch), ctypes.byref(n)), self._h)
        return n.value

    def _ws(self, batch, device):
        nbytes = self.workspace_bytes(batch)
        return torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device), nbytes

    def _call(self, fn, src, dst, batch, *extra):
        ws, nbytes = self._ws(batch, src.device)
        stream = torch.cuda.current_stream(src.device).cuda_stream
        st = fn(self._h, ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()), int(batch), *extra,
                ctypes.c_void_p(ws.data_ptr()), nbytes, ctypes.c_void_p(stream))
        _lib.check(st, self._h)
        return dst

    def _check_map(self, x):
        if x.shape[-1] != self.npix:
            raise ValueError(f"last dimension must be npix={self.npix} for nside={self.nside}, got {x.shape[-1]}")

    def _check_alm(self, a):
        if tuple(a.shape[-2:]) != (self.lmax, self.mmax):
            raise ValueError(f"trailing dimensions must be (lmax, mmax)=({self.lmax}, {self.mmax}), got {tuple(a.shape[-2:])}")

    def forward(self, x, iters=0):
        """map [B, npix] (contiguous, plan dtype) -> alm [B, L, M] complex."""
        self._check_map(x)
        B = x.shape[0]
        out = torch.empty((B, self.lmax, self.mmax), dtype=self.cdtype, device=x.device)
        dst = torch.view_as_real(out)
        if iters:
            self._call(self._lib.hpx_sht_forward_refined, x, dst, B, ctypes.c_int32(int(iters)))
        else:
            self._call(self._lib.hpx_sht_forward, x, dst, B)
        return out

    def inverse(self, a):
        """alm [B, L, M] complex (contiguous) -> map [B, npix]."""
        self._check_alm(a)
        B = a.shape[0]
        out = torch.empty((B, self.npix), dtype=self.dtype, device=a.device)
        self._call(self._lib.hpx_sht_inverse, torch.view_as_real(a.resolve_conj().contiguous()), out, B)
        return out

    def forward_adjoint(self, g):
        """alm-space cotangent [B, L, M] complex -> map-space cotangent [B, npix]."""
        self._check_alm(g)
        B = g.shape[0]
        out = torch.empty((B, self.npix), dtype=self.dtype, device=g.device)
        self._call(self._lib.hpx_sht_forward_adjoint, torch.view_as_real(g.resolve_conj().contiguous()), out, B)
        return out

    def inverse_adjoint(self, g):
        """map-space cotangent [B, npix] -> alm-space cotangent [B, L, M] complex."""
        self._check_map(g)
        B = g.shape[0]
        out = torch.empty((B, self.lmax, self.mmax), dtype=self.cdtype, device=g.device)
        self._call(self._lib.hpx_sht_inverse_adjoint, g, torch.view_as_real(out), B)
        return out


class LatLonPlan(Plan):
    """An ``hpx_plan_t`` over a latitude-longitude grid (hpx_plan_create_latlon):
    maps [B, nlat * nlon], rings north to south, same transform calls as Plan."""

    def __init__(self, nlat, nlon, lmax, mmax, grid="equiangular", precision="fp32", device=0, batch_chunk=64,
                 legendre_table=True):
        lib = _lib.load()
        if precision not in _lib.PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}; expected one of {sorted(_lib.PRECISIONS)}")
        if grid not in _lib.GRIDS:
            raise ValueError(f"unknown grid {grid!r}; expected one of {sorted(_lib.GRIDS)}")
        self.nside = 0
        self.nlat, self.nlon, self.grid = int(nlat), int(nlon), grid
        self.lmax, self.mmax = int(lmax), int(mmax)
        self.precision = precision
        self.device = int(device)
        self.dtype = torch.float64 if precision == "fp64" else torch.float32
        self.cdtype = torch.complex128 if precision == "fp64" else torch.complex64
        self.npix = self.nlat * self.nlon
        desc = _lib.HpxLatLonDesc()
        desc.nlat, desc.nlon, desc.lmax, desc.mmax = self.nlat, self.nlon, self.lmax, self.mmax
        desc.grid = _lib.GRIDS[grid]
        desc.precision = _lib.PRECISIONS[precision]
        desc.batch_chunk = int(batch_chunk)
        desc.device = self.device
        desc.flags = 0 if legendre_table else _lib.FLAG_OTF_LEGENDRE
        desc.reserved = 0
        handle = ctypes.c_void_p()
        _lib.check(lib.hpx_plan_create_latlon(ctypes.byref(desc), ctypes.byref(handle)))
        self._h = handle
        self._lib = lib


def get_latlon_plan(nlat, nlon, lmax, mmax, grid, precision, device, batch_chunk=64, legendre_table=True):
    key = ("latlon", int(nlat), int(nlon), int(lmax), int(mmax), grid, precision, int(device), int(batch_chunk),
           bool(legendre_table))
    with _plan_lock:
        p = _plans.get(key)
        if p is None:
            p = LatLonPlan(nlat, nlon, lmax, mmax, grid, precision, device, batch_chunk, legendre_table)
            _plans[key] = p
        return p


def get_plan(nside, lmax, mmax, quad_weights, precision, device, batch_chunk=64, legendre_table=True):
    key = (int(nside), int(lmax), int(mmax), quad_weights if quad_weights == "ring" else "none", precision, int(device),
           int(batch_chunk), bool(legendre_table))
    with _plan_lock:
        p = _plans.get(key)
        if p is None:
            p = Plan(nside, lmax, mmax, key[3], precision, device, batch_chunk, legendre_table=key[7])
            _plans[key] = p
        return p


def clear_plan_cache():
    with _plan_lock:
        _plans.clear()


# ---------------------------------------------------------------------- autograd
class SHTFunction(torch.autograd.Function):
    """Forward SHT (optionally Jacobi-refined) with its exact adjoint as backward."""

    @staticmethod
    def forward(ctx, x, plan, iters):
        ctx.plan = plan
        ctx.iters = iters
        return plan.forward(x, iters)

    @staticmethod
    def backward(ctx, g):
        plan, k = ctx.plan, ctx.iters
        g = g.contiguous()
        # a_k = a_{k-1} + S(f - I a_{k-1})  =>  R_k = S + (1 - S I) R_{k-1}
        #   =>  R_k^T g = S^T g + R_{k-1}^T (g - I^T S^T g)
        out = None
        h = g
        for _ in range(k):
            u = plan.forward_adjoint(h)
            out = u if out is None else out + u
            h = h - plan.inverse_adjoint(u)
        u = plan.forward_adjoint(h)
        out = u if out is None else out + u
        return out, None, None


class iSHTFunction(torch.autograd.Function):
    """Inverse SHT with its exact adjoint as backward."""

    @staticmethod
    def forward(ctx, a, plan):
        ctx.plan = plan
        return plan.inverse(a)

    @staticmethod
    def backward(ctx, g):
        return ctx.plan.inverse_adjoint(g.contiguous()), None


def _device_index(x):
    return x.device.index if x.device.index is not None else torch.cuda.current_device()


class _Base(nn.Module):
    def __init__(self, nside, lmax, mmax, quad_weights, norm, csphase, precision, refine_iters, batch_chunk,
                 legendre_table=True, autotune=False):
        super().__init__()
        if not torch.cuda.is_available():
            raise RuntimeError("CUDA device is not available. This class requires a GPU.")
        self.nside = nside
        self.norm = norm
        self.csphase = csphase
        self.nlat = 4 * nside - 1
        self.nlon = 4 * nside
        self.quad_weights = quad_weights
        self.lmax = lmax or self.nlat
        self.mmax = mmax or (self.nlon // 2 + 1)
        if precision not in ("fp32", "bf16x3", "f16x3"):
            raise ValueError("precision must be 'fp32', 'f16x3' or 'bf16x3' (float64 data select fp64 automatically)")
        self.precision = precision
        self.refine_iters = int(refine_iters)
        self.batch_chunk = int(batch_chunk)
        self.legendre_table = bool(legendre_table)
        self.autotune = bool(autotune)
        _lib.load()  # fail loudly at construction if the library is missing

    def _plan(self, dtype, device_index):
        prec = "fp64" if dtype == torch.float64 else self.precision
        plan = get_plan(self.nside, self.lmax, self.mmax, self.quad_weights, prec, device_index, self.batch_chunk,
                        self.legendre_table)
        if self.autotune and not getattr(plan, "_tuned", False):
            from .autotune import tune

            tune(plan, self.batch_chunk)
            plan._tuned = True
        return plan


class SHTCUDA(_Base):
    def __init__(self, nside, lmax=None, mmax=None, quad_weights="ring", norm="ortho", csphase=True, *,
                 precision="fp32", refine_iters=0, batch_chunk=64, legendre_table=True, autotune=False):
        super().__init__(nside, lmax, mmax, quad_weights, norm, csphase, precision, refine_iters, batch_chunk,
                         legendre_table, autotune)

    def forward(self, x):
        if torch.is_complex(x):
            raise ValueError("Input tensor must be real.")
        if not x.is_cuda:
            raise ValueError("SHTCUDA expects a CUDA tensor")
        if x.dtype not in (torch.float32, torch.float64):
            x = x.to(torch.float32)
        lead = x.shape[:-1]
        xf = x.reshape(-1, x.shape[-1]).contiguous()
        plan = self._plan(x.dtype, _device_index(x))
        a = SHTFunction.apply(xf, plan, self.refine_iters)
        return a.reshape(*lead, self.lmax, self.mmax)


class iSHTCUDA(_Base):
    def __init__(self, nside, lmax=None, mmax=None, quad_weights="ring", norm="ortho", csphase=True, *,
                 precision="fp32", refine_iters=0, batch_chunk=64, legendre_table=True, autotune=False):
        super().__init__(nside, lmax, mmax, quad_weights, norm, csphase, precision, refine_iters, batch_chunk,
                         legendre_table, autotune)

    def forward(self, x):
        if not x.is_cuda:
            raise ValueError("iSHTCUDA expects a CUDA tensor")
        if not torch.is_complex(x):
            raise ValueError("Input tensor must be complex [..., lmax, mmax].")
        if x.dtype not in (torch.complex64, torch.complex128):
            x = x.to(torch.complex64)
        lead = x.shape[:-2]
        af = x.reshape(-1, x.shape[-2], x.shape[-1]).contiguous()
        dt = torch.float64 if x.dtype == torch.complex128 else torch.float32
        plan = self._plan(dt, _device_index(x))
        f = iSHTFunction.apply(af, plan)
        return f.reshape(*lead, f.shape[-1])
