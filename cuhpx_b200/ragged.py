"""Ragged batches: maps of several HEALPix resolutions in one call.

``RaggedSHT(nsides, ...)(maps)`` analyses a list of map batches, one
``[B_g, 12 nside_g^2]`` tensor per resolution, through ``hpx_ragged_forward``
(one library call; the groups run at the same time on streams the library
forks from the current one) and returns the list of ``[B_g, L_g, M_g]``
coefficient tensors; ``RaggedISHT`` is the synthesis.  By default a group of
resolution N keeps L = M = 2N - 1.  ``autotune=True`` tunes each group's
launch schedule for its batch size on the first call (``cuhpx_b200.autotune``).

``graph=True`` records the whole sequence of launches once in a CUDA graph
(``torch.cuda.CUDAGraph``) for the batch sizes of the first call, and later
calls copy their inputs into the graph's buffers and replay it: the outputs
then live in the graph's buffers and are overwritten by the next call.

``split_by_offsets`` turns the flat form (one 1-D buffer of concatenated
maps, ``offsets[i]`` the first sample of map i, runs of equal nside kept
together) into the list form without copying.
"""

import ctypes

import torch
import torch.nn as nn

from . import _lib
from .hpx_sht import _device_index, get_plan


def split_by_offsets(flat, offsets, nsides):
    """Runs of consecutive maps with equal nside -> list of [B, npix] views, and their nsides."""
    groups, gns = [], []
    i, n = 0, len(nsides)
    while i < n:
        j = i
        while j + 1 < n and nsides[j + 1] == nsides[i]:
            j += 1
        npix = 12 * nsides[i] * nsides[i]
        start = int(offsets[i])
        for k in range(i, j + 1):
            if int(offsets[k + 1]) - int(offsets[k]) != npix:
                raise ValueError(f"map {k}: offsets span {int(offsets[k + 1]) - int(offsets[k])} samples, nside "
                                 f"{nsides[k]} needs {npix}")
        groups.append(flat[start:start + (j - i + 1) * npix].view(j - i + 1, npix))
        gns.append(nsides[i])
        i = j + 1
    return groups, gns


class _Ragged(nn.Module):
    def __init__(self, nsides, lmax, mmax, precision, graph, legendre_table, autotune=False):
        super().__init__()
        self.autotune = bool(autotune)
        self.nsides = [int(n) for n in nsides]
        self.lmax = [int(lmax(n)) if callable(lmax) else int(lmax or 2 * n - 1) for n in self.nsides]
        self.mmax = [int(mmax(n)) if callable(mmax) else int(mmax or 2 * n - 1) for n in self.nsides]
        self.precision = precision
        self.graph = bool(graph)
        self.legendre_table = legendre_table
        self._g = None
        _lib.load()

    def _plans(self, dtype, dev, batches=None):
        prec = "fp64" if dtype in (torch.float64, torch.complex128) else self.precision
        plans = [get_plan(n, L, M, "ring", prec, dev, 64, self.legendre_table)
                 for n, L, M in zip(self.nsides, self.lmax, self.mmax)]
        if self.autotune and batches is not None:
            from .autotune import tune

            for p, b in zip(plans, batches):
                if b > 0 and getattr(p, "_tuned_batch", None) != min(int(b), 64):
                    tune(p, min(int(b), 64))
                    p._tuned_batch = min(int(b), 64)
        return plans

    def _run(self, fn, plans, ins, outs):
        lib = _lib.load()
        n = len(plans)
        ph = (ctypes.c_void_p * n)(*[p._h.value for p in plans])
        pi = (ctypes.c_void_p * n)(*[t.data_ptr() for t in ins])
        po = (ctypes.c_void_p * n)(*[t.data_ptr() for t in outs])
        pb = (ctypes.c_int64 * n)(*[t.shape[0] for t in ins])
        need = ctypes.c_size_t()
        _lib.check(lib.hpx_ragged_workspace_size(ph, n, pb, ctypes.byref(need)))
        dev = ins[0].device
        ws = torch.empty(max(need.value, 1), dtype=torch.uint8, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(fn(ph, n, pi, po, pb, ctypes.c_void_p(ws.data_ptr()), need.value, ctypes.c_void_p(stream)))
        return ws

    def _keep(self, ws):
        # A captured graph reads its workspace at every replay, so graph mode
        # keeps it; an eager call may release it at once: the library joins
        # its group streams back into the caller's stream before returning,
        # so the allocator's stream-ordered reuse comes after the last kernel.
        self._ws = ws if self.graph else None

    def _call(self, xs):
        if len(xs) != len(self.nsides):
            raise ValueError(f"expected {len(self.nsides)} groups, got {len(xs)}")
        if not self.graph:
            return self._eager(xs)
        shapes = [tuple(x.shape) for x in xs]
        if self._g is None or self._g[0] != shapes:
            static_in = [x.clone() for x in xs]
            s = torch.cuda.Stream(xs[0].device)
            s.wait_stream(torch.cuda.current_stream(xs[0].device))
            with torch.cuda.stream(s):
                self._eager(static_in)  # warm-up: plans, allocator pools
            torch.cuda.current_stream(xs[0].device).wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                static_out = self._eager(static_in)
            self._g = (shapes, g, static_in, static_out)
        _, g, static_in, static_out = self._g
        for dst, src in zip(static_in, xs):
            dst.copy_(src)
        g.replay()
        return static_out


class RaggedSHT(_Ragged):
    """Analysis of a list of map batches of several resolutions (see module docstring)."""

    def __init__(self, nsides, lmax=None, mmax=None, *, precision="fp32", graph=False, legendre_table=True,
                 autotune=False):
        super().__init__(nsides, lmax, mmax, precision, graph, legendre_table, autotune)

    def _eager(self, xs):
        xs = [x.contiguous() for x in xs]
        dtype = xs[0].dtype
        plans = self._plans(dtype, _device_index(xs[0]), [x.shape[0] for x in xs])
        cdt = torch.complex128 if dtype == torch.float64 else torch.complex64
        outs = [torch.empty((x.shape[0], L, M), dtype=cdt, device=x.device)
                for x, L, M in zip(xs, self.lmax, self.mmax)]
        ws = self._run(_lib.load().hpx_ragged_forward, plans, xs, [torch.view_as_real(o) for o in outs])
        self._keep(ws)
        return outs

    def forward(self, maps):
        return self._call(list(maps))


class RaggedISHT(_Ragged):
    """Synthesis of a list of coefficient batches of several resolutions."""

    def __init__(self, nsides, lmax=None, mmax=None, *, precision="fp32", graph=False, legendre_table=True,
                 autotune=False):
        super().__init__(nsides, lmax, mmax, precision, graph, legendre_table, autotune)

    def _eager(self, alms):
        alms = [a.resolve_conj().contiguous() for a in alms]
        dt = torch.float64 if alms[0].dtype == torch.complex128 else torch.float32
        plans = self._plans(alms[0].dtype, _device_index(alms[0]), [a.shape[0] for a in alms])
        outs = [torch.empty((a.shape[0], 12 * n * n), dtype=dt, device=a.device) for a, n in zip(alms, self.nsides)]
        ws = self._run(_lib.load().hpx_ragged_inverse, plans, [torch.view_as_real(a) for a in alms], outs)
        self._keep(ws)
        return outs

    def forward(self, alms):
        return self._call(list(alms))
