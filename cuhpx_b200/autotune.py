"""Autotuner of the launch schedule (``hpx_plan_set_schedule``).

For one plan and batch size it times candidate schedules on random maps of
the plan's shape, on the device, and keeps the fastest: the maps each
ring-FFT CTA transforms (4, 8, 16, 32), whether the power-of-two and the
Bluestein ring launches overlap on two streams, and, for tensor-core plans, how the
analysis and the synthesis tiles are dealt to the persistent CTAs (the
m-to-CTA schedule: ``order_snake``, ``tile_snake``, ``greedy``,
``contiguous``).  The search is coordinate-wise: ring grouping and ring
streams on the whole SHT + iSHT step, then the analysis deal on the analysis, then the synthesis
deal on the synthesis; each candidate is the median of ``reps`` CUDA-event
timings after ``warmup`` calls.  Results are cached in a JSON file keyed by
GPU name, nside, lmax, mmax, batch, precision and whether the plan holds the
resident Legendre table (``$HPX_TUNE_CACHE``, default
``~/.cache/hpx_b200/schedules.json``), so later processes apply a tuned
schedule without measuring.  cuHPX has no counterpart (its contraction is a
torch einsum and its FFT cuFFT).
"""

import json
import os
import statistics
import tempfile
import threading

import torch

from . import _lib

RING_GROUPS = (4, 8, 16, 32)
DEALS = tuple(_lib.DEALS)
_lock = threading.Lock()


def cache_path():
    return os.environ.get("HPX_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "hpx_b200",
                                                            "schedules.json")


def _load_cache(path):
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _save_cache(path, data):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(path), prefix=".schedules.")
    with os.fdopen(fd, "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def get_schedule(plan):
    s = _lib.HpxSchedule()
    _lib.check(plan._lib.hpx_plan_get_schedule(plan._h, s), plan._h)
    inv = {v: k for k, v in _lib.DEALS.items()}
    return {"ring_maps_per_cta": s.ring_maps_per_cta, "fwd_deal": inv[s.fwd_deal], "inv_deal": inv[s.inv_deal],
            "ctas": s.ctas, "ring_streams": s.ring_streams}


def set_schedule(plan, sched):
    s = _lib.HpxSchedule()
    s.ring_maps_per_cta = int(sched["ring_maps_per_cta"])
    s.fwd_deal = _lib.DEALS[sched["fwd_deal"]]
    s.inv_deal = _lib.DEALS[sched["inv_deal"]]
    s.ctas = int(sched.get("ctas", 0))
    s.ring_streams = int(sched.get("ring_streams", 2))
    _lib.check(plan._lib.hpx_plan_set_schedule(plan._h, s), plan._h)


def key(plan, batch):
    dev = torch.cuda.get_device_name(plan.device)
    table = getattr(plan, "table_bytes", 0) > 0
    return f"{dev}|nside={plan.nside}|lmax={plan.lmax}|mmax={plan.mmax}|batch={int(batch)}|{plan.precision}|table={int(table)}"


def _time(fn, warmup, reps, device):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize(device)
    out = []
    stream = torch.cuda.current_stream(device)
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return statistics.median(out)


def tune(plan, batch, warmup=2, reps=3, cache=True, force=False):
    """Pick and apply the fastest schedule of `plan` for `batch` maps; returns
    ``{"schedule": ..., "ms": {candidate: ms}, "cached": bool}``."""
    device = torch.device("cuda", plan.device)
    path = cache_path()
    k = key(plan, batch)
    with _lock:
        if cache and not force:
            hit = _load_cache(path).get(k)
            if hit:
                set_schedule(plan, hit["schedule"])
                return {"schedule": hit["schedule"], "ms": hit.get("ms", {}), "cached": True}
        g = torch.Generator(device=device).manual_seed(0)
        x = torch.randn((int(batch), plan.npix), generator=g, device=device, dtype=plan.dtype)
        with torch.no_grad():
            a = plan.forward(x)

        def analysis():
            plan.forward(x)

        def synthesis():
            plan.inverse(a)

        def step():
            plan.inverse(plan.forward(x))

        best = get_schedule(plan)
        ms = {}

        def trial(name, sched, fn):
            set_schedule(plan, sched)
            t = _time(fn, warmup, reps, device)
            ms[name] = t
            return t

        with torch.no_grad():
            tc = plan.precision in ("f16x3", "bf16x3")
            cands = [(f"ring_maps_per_cta={gsz}", dict(best, ring_maps_per_cta=gsz)) for gsz in RING_GROUPS]
            best = min(cands, key=lambda c: trial(c[0], c[1], step))[1]
            cands = [(f"ring_streams={k}", dict(best, ring_streams=k)) for k in (2, 1)]
            best = min(cands, key=lambda c: trial(c[0], c[1], step))[1]
            if tc:
                cands = [(f"fwd_deal={d}", dict(best, fwd_deal=d)) for d in DEALS]
                best = min(cands, key=lambda c: trial(c[0], c[1], analysis))[1]
                cands = [(f"inv_deal={d}", dict(best, inv_deal=d)) for d in DEALS]
                best = min(cands, key=lambda c: trial(c[0], c[1], synthesis))[1]
        set_schedule(plan, best)
        if cache:
            data = _load_cache(path)
            data[k] = {"schedule": best, "ms": ms}
            _save_cache(path, data)
        return {"schedule": best, "ms": ms, "cached": False}
