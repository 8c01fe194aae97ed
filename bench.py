"""Throughput of the HEALPix SHT+iSHT on B200: maps/s at nside=1024, lmax=mmax=2047, batch 64.

One step = analysis (SHT, with the configured Jacobi refinement) of a batch of
64 float32 maps followed by synthesis (iSHT) of the resulting coefficients.
Inputs are band-limited Gaussian fields (C_l ~ (l+1)^-2) plus N(0, 1e-3)
white noise, generated on the device from a fixed seed; each batch is 3.2 GB,
larger than the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--precision f16x3|bf16x3|fp32] [--refine k]
  python bench.py --impl reference ...   # the reference's CPU algorithm (multi-threaded port) on the host

Under torchrun every rank runs its own batch (replicas, no collective on the
data path); the timed region is bracketed by barriers and the max over ranks
is reported.  Prints one JSON line on rank 0.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "SHT+iSHT maps/s nside1024 lmax2047 B64: mixed vs FP32 plain, err<=1e-5 vs FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hpx", choices=["hpx", "reference"])
    ap.add_argument("--precision", default="auto")
    ap.add_argument("--refine", type=int, default=-1, help="Jacobi iterations (-1: default for the precision)")
    ap.add_argument("--nside", type=int, default=1024)
    ap.add_argument("--lmax", type=int, default=2047)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-FP32 comparison run")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the error check against the FP64 path")
    ap.add_argument("--no-ragged", action="store_true", help="skip the ragged workload (96 maps of mixed nside)")
    ap.add_argument("--no-refined", action="store_true",
                    help="skip the refined variants (1 and 3 Jacobi iterations) of the mixed-precision analysis")
    ap.add_argument("--workload", default="sht_isht", choices=["sht_isht", "ragged", "remap", "next"],
                    help="sht_isht: the headline step; ragged: 96 maps of mixed nside; remap: NEST -> RING "
                         "reordering of a batch of maps (with the other layout pairs beside it); next: the rows "
                         "beside the headline (cfg5 loss and regridding with backward, spin-1, healpy packing)")
    ap.add_argument("--accuracy-maps", type=int, default=16)
    ap.add_argument("--spot-maps", type=int, default=2, help="maps checked against the CPU spot oracle")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL,
                text=True,
            )
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": smax,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ----------------------------------------------------------------- CPU baseline
def host_info():
    """CPU model, logical cores and RAM of this host (for the CPU timings)."""
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    ram = None
    try:
        ram = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 2**30
    except (ValueError, OSError):
        pass
    return {"cpu_model": model, "logical_cores": os.cpu_count(), "ram_gib": ram}


def _ref_port(threads=None):
    """The multi-threaded CPU port of the reference's SHT/iSHT (oracle/ref_cpu)."""
    from oracle import ref_cpu as RC

    RC.load()
    if threads:
        RC.set_threads(threads)
    return RC


PORT_SAMPLE = ("per map: the reference's CPU SHT then iSHT (cuhpx/hpx_sht.py:173-283) in float64 -- one rfft/irfft "
               "per ring (numpy) and the Legendre contraction over every order m < M and degree m <= l < L (C, "
               "OpenMP over the orders, the table's values regenerated per order by the reference's recurrence "
               "instead of held: 68.6 GB at nside 1024)")


def cpu_baseline(nside, lmax, min_seconds=10.0):
    """The CPU port timed on whole maps (all orders) for at least min_seconds."""
    RC = _ref_port(os.cpu_count())
    RC.time_sht_isht(nside, lmax, lmax, seed=99)  # warm-up (page-in, thread pool)
    secs, t0 = [], time.perf_counter()
    while len(secs) < 2 or time.perf_counter() - t0 < min_seconds:
        secs.append(RC.time_sht_isht(nside, lmax, lmax, seed=len(secs)))
    spm = statistics.median(secs)
    return {
        "value": 1.0 / spm,
        "unit": "maps/s",
        "cores": RC.threads(),
        "kind": "port",
        "sample": f"{len(secs)} maps at nside={nside}, L=M={lmax}, one at a time; " + PORT_SAMPLE,
        "seconds_per_map": spm,
        "host": host_info(),
    }


def run_reference(args):
    """The reference's CPU implementation (its port, every order) on the host:
    each step is one whole float64 map, SHT then iSHT, timed end to end."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lm = args.lmax
    RC = _ref_port(os.cpu_count())
    cores = RC.threads()
    for w in range(args.warmup):
        RC.time_sht_isht(args.nside, lm, lm, seed=100 + w)
    t0 = time.perf_counter()
    for s in range(args.steps):
        RC.time_sht_isht(args.nside, lm, lm, seed=s)
    total = time.perf_counter() - t0
    value = args.steps / total
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "maps/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"SHT+iSHT nside={args.nside} lmax=mmax={lm}, one whole map per step (a bounded "
                               f"sample of the batch of {args.batch})", "batch": 1, "nside": args.nside, "lmax": lm,
                   "mmax": lm},
        "cpu_baseline": {
            "value": value,
            "unit": "maps/s",
            "cores": cores,
            "kind": "port",
            "sample": "one map per step, every order and degree computed; " + PORT_SAMPLE,
        },
        "host": host_info(),
        "e2e": {"value": value, "unit": "maps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU arm
def make_inputs(torch, hpx, nside, L, B, device, seed=2):
    """cfg3 maps: band-limited a_lm with C_l ~ (l+1)^-2 synthesised, plus N(0, 1e-3) noise."""
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    l = torch.arange(L, device=device, dtype=torch.float32)
    sig = (1.0 / (l + 1.0))[:, None]
    re = torch.randn((B, L, L), generator=g, device=device) * sig
    im = torch.randn((B, L, L), generator=g, device=device) * sig
    tri = torch.tril(torch.ones(L, L, device=device, dtype=torch.bool))
    a = torch.complex(re, im) * tri
    a[..., 0] = a[..., 0].real.to(a.dtype)
    a = a / np.sqrt(2.0)
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L)
    with torch.no_grad():
        f = isht(a)
    del a
    f += torch.randn(f.shape, generator=g, device=device) * np.sqrt(1e-3)
    return f.contiguous()


def time_steps(torch, fn, steps, warmup, dist, stream):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        from cuhpx_b200.replicas import max_over_ranks

        ms = max_over_ranks(ms, device="cuda")
        dist.barrier()
    return ms


def run_gpu(args):
    import torch

    import cuhpx_b200 as hpx

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
        dist = tdist

    nside, L, B = args.nside, args.lmax, args.batch
    prec = args.precision
    if prec == "auto":
        prec = "f16x3" if _tc_available(hpx, dev) else "fp32"
    refine = args.refine if args.refine >= 0 else (1 if prec in ("bf16x3", "tf32") else 0)

    f = make_inputs(torch, hpx, nside, L, B, dev)
    sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec, refine_iters=refine)
    isht = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision=prec)
    stream = torch.cuda.current_stream(dev)
    out = {}

    def step():
        with torch.no_grad():
            a = sht(f)
            out["f2"] = isht(a)

    # plan creation (ring tables, Legendre seeds, chirp spectra and, for
    # tensor-core plans, the resident Legendre table) timed on its own
    torch.cuda.synchronize()
    t_plan = time.perf_counter()
    plan = hpx.get_plan(nside, L, L, "ring", prec, local)
    torch.cuda.synchronize()
    plan_create_s = time.perf_counter() - t_plan
    clocks = ClockSampler(local)
    # warm-up, then the timed region with per-kernel events and clock sampling
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    plan.stats_enable(True)
    clocks.start()
    ms = time_steps(torch, step, args.steps, 0, dist, stream)
    clk = clocks.stop()
    stats = plan.stats_read()
    plan.stats_enable(False)
    plan.check()  # raises if a tensor-core pipeline wait gave up during the timed steps
    # the timed result must be a real transform: compare one batch with the plain FP32 path
    with torch.no_grad():
        ref = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="fp32")(f[:4])
        got = sht(f[:4])
        plan.check()
        check_rel = float((got - ref).abs().pow(2).sum().sqrt() / ref.abs().pow(2).sum().sqrt())
    if not (check_rel < 1e-3):
        raise RuntimeError(f"timed transform disagrees with the FP32 path: rel-L2 {check_rel:.3e}")
    ms_step = ms / args.steps
    value = world * B * args.steps / (ms / 1000.0)
    launches_per_step = sum(v[0] * kernels_in_stage(k, prec, nside) for k, v in stats.items()) / args.steps

    # roofline of the dominant kernel
    roof = roofline(stats, args, prec, refine, nside, L, B, plan.table_bytes > 0, plan.table_stream_bytes)

    # plain FP32 comparison (the target is >= 2x this on the same GPU)
    plain = None
    if not args.no_plain and prec != "fp32":
        sht_p = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="fp32")
        isht_p = hpx.iSHTCUDA(nside, lmax=L, mmax=L, precision="fp32")

        def step_p():
            with torch.no_grad():
                isht_p(sht_p(f))

        ms_p = time_steps(torch, step_p, max(1, args.steps // 2), 1, dist, stream)
        plain = world * B * max(1, args.steps // 2) / (ms_p / 1000.0)

    # end to end through the public modules with host buffers
    e2e = None
    if not args.no_e2e:
        # the pipeline's fill (first upload) and drain (last download) do not
        # overlap anything: at least 60 steps amortise them to about 2% (about
        # 4 s; 30 steps measured 2% slower per step on the same box).  Cached
        # blocks of the earlier runs are returned first, so that the pipeline's
        # buffers do not have to displace them inside the timed region.
        torch.cuda.empty_cache()
        ms_e, ksteps = e2e_pipelined(torch, sht, isht, f, dev, max(args.steps, 60), args.warmup, dist)
        nb = f.numel() * f.element_size()
        e2e = {
            "value": world * B * ksteps / (ms_e / 1000.0),
            "unit": "maps/s",
            "h2d_bytes_per_step": nb,
            "d2h_bytes_per_step": nb,
            "steps": ksteps,
            "pipeline": "every step copies its 64 maps host->device (pinned), runs SHT+iSHT through "
            "SHTCUDA/iSHTCUDA and copies the maps back; upload of step i+1 and download of step i-1 "
            "overlap step i on three streams",
        }

    acc = None
    if not args.no_accuracy:
        acc = accuracy_vs_fp64(torch, hpx, sht, isht, f[: args.accuracy_maps], nside, L, refine, args.spot_maps)

    # the workload's refined variants: k Jacobi iterations in the analysis (each
    # one more synthesis and analysis of the residual), the same maps, and their
    # round-trip error against the FP64 path with the same k
    refined = None
    if not args.no_refined and prec in ("f16x3", "bf16x3") and world == 1:
        refined = {}
        for k in (1, 3):
            sht_k = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec, refine_iters=k)

            def step_k():
                with torch.no_grad():
                    out["fk"] = isht(sht_k(f))

            ms_k = time_steps(torch, step_k, max(2, args.steps // 2), args.warmup, dist, stream)
            e = {"maps_per_s": B * max(2, args.steps // 2) / (ms_k / 1000.0)}
            if not args.no_accuracy:
                a_k = accuracy_vs_fp64(torch, hpx, sht_k, isht, f[: args.accuracy_maps], nside, L, k)
                e["roundtrip_rel_l2"] = a_k["roundtrip_rel_l2"]
                e["alm_rel_l2"] = a_k["alm_rel_l2"]
            refined[str(k)] = e
            del sht_k
        out.pop("fk", None)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(nside, L)

    # the ragged workload (96 maps of mixed nside) beside the headline, so that
    # every run of the default line records it
    ragged = None
    if world == 1 and not args.no_ragged and prec in ("f16x3", "bf16x3") and nside == 1024:
        out.clear()
        torch.cuda.empty_cache()
        ragged = ragged_figures(torch, hpx, dev, prec, max(3, args.steps // 2), args.warmup)

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "maps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if prec == "fp32" else f"f32 io, {prec} contraction",
            "data": "synthetic",
            "config": {
                "workload": f"SHT(refine={refine})+iSHT nside={nside} lmax=mmax={L} batch={B} per GPU",
                "nside": nside,
                "lmax": L,
                "mmax": L,
                "batch_per_gpu": B,
                "precision": prec,
                "refine_iters": refine,
                "l2": "inputs larger than L2 (3.2 GB per batch); no flush",
                "parallelism": f"replicas x{world}",
            },
            "gpu_launches": int(round(launches_per_step * args.steps)),
            "plan": {"create_s": plan_create_s, "table_bytes": plan.table_bytes},
            "kernels_per_step": launches_per_step,
            "stage_ms_per_step": {k: v[1] / args.steps for k, v in stats.items() if v[0]},
            "roofline": roof,
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "plain_fp32_maps_per_s": plain,
            "check_rel_l2_vs_fp32": check_rel,
            "err_vs_fp64": acc,
            "refined": refined,
            "ragged": ragged,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def accuracy_vs_fp64(torch, hpx, sht, isht, f, nside, L, refine, spot_maps=0):
    """Rel-L2 of the timed modules against the FP64 path with the same Jacobi
    iterations, on the first maps of the timed batch: the analysis coefficients
    and the round trip iSHT(SHT(f)).  With spot_maps > 0 (no refinement), the
    orders 0, 1, 2, M/4, M/2 and M-1 of the first spot_maps maps are also
    compared with the CPU spot oracle (one float64 Legendre column at a time,
    oracle/hpx_oracle.py sht_spot), for the timed path and the FP64 path."""

    def rel(a, b):
        return float((a.to(b.dtype) - b).abs().pow(2).sum().sqrt() / b.abs().pow(2).sum().sqrt())

    with torch.no_grad():
        f64 = f.double()
        a64 = hpx.SHTCUDA(nside, lmax=L, mmax=L, refine_iters=refine)(f64)
        r64 = hpx.iSHTCUDA(nside, lmax=L, mmax=L)(a64)
        a = sht(f)
        r = isht(a)
        out = {
            "maps": int(f.shape[0]),
            "refine_iters": refine,
            "alm_rel_l2": rel(a, a64),
            "roundtrip_rel_l2": rel(r, r64),
            "tolerance": 1e-5,
            "reference": "this library's FP64 path (FP64 FFTs, FP64 Legendre recurrence and contraction), same "
                         "refine_iters",
        }
        if spot_maps > 0 and refine == 0:
            from oracle import hpx_oracle as O

            ms = sorted({0, 1, 2, L // 4, L // 2, L - 1})
            fs = f64[:spot_maps].cpu().numpy()
            ex = torch.from_numpy(O.sht_spot(fs, nside, L, L, ms, nodes="exact")).to(a.device)
            rf = torch.from_numpy(O.sht_spot(fs, nside, L, L, ms)).to(a.device)
            out["spot_oracle"] = {
                "maps": spot_maps,
                "orders": ms,
                "alm_rel_l2": rel(a[:spot_maps, :, ms], ex),
                "fp64_path_alm_rel_l2": rel(a64[:spot_maps, :, ms], ex),
                "reference_form_alm_rel_l2": rel(rf, ex),
                "reference": "CPU spot oracle: float64 ring rfft + one Legendre column per order by the "
                             "reference's recurrence (cuhpx/hpx_sht.py:214-236, cuhpx/sht_tools.py:204-214) in "
                             "80-bit extended precision at the plan's ring nodes; reference_form_alm_rel_l2 is the "
                             "reference's own FP64 recurrence against it (its diagonal goes subnormal for high "
                             "orders near the poles)",
            }
        del f64, a64, r64
    torch.cuda.empty_cache()
    return out


def e2e_pipelined(torch, sht, isht, f, dev, steps, warmup, dist):
    """Time `steps` end-to-end steps: host->device copy of the step's maps from
    pinned memory, SHT + iSHT through the public modules, device->host copy of
    the result.  Consecutive steps overlap on three streams with two device
    buffers each way (the copy engines of the two directions and the SMs work
    at the same time).  Returns (ms, steps), max over ranks."""
    s_in, s_c, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    hin = [torch.empty(f.shape, dtype=f.dtype, pin_memory=True) for _ in range(2)]
    hout = [torch.empty(f.shape, dtype=f.dtype, pin_memory=True) for _ in range(2)]
    for h in hin:
        h.copy_(f)
    din = [torch.empty_like(f) for _ in range(2)]
    ys = [None, None]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_c = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def run(n):
        for i in range(n):
            k = i & 1
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_c[k])  # step i-2 has finished reading din[k]
                din[k].copy_(hin[k], non_blocking=True)
                ev_in[k].record(s_in)
            if ys[k] is not None:
                # step i-2's result is released only once its download is done, so that the
                # allocator hands its block to the compute stream again (no record_stream,
                # whose deferred frees make the cache grow with every step)
                ev_out[k].synchronize()
                ys[k] = None
            with torch.cuda.stream(s_c):
                s_c.wait_event(ev_in[k])
                with torch.no_grad():
                    ys[k] = isht(sht(din[k]))
                ev_c[k].record(s_c)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_c[k])
                hout[k].copy_(ys[k], non_blocking=True)
                ev_out[k].record(s_out)

    run(warmup)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    run(steps)
    s_in.wait_stream(s_out)
    e1.record(s_in)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        from cuhpx_b200.replicas import max_over_ranks

        ms = max_over_ranks(ms, device="cuda")
        dist.barrier()
    return ms, steps


def _tc_available(hpx, dev):
    try:
        hpx.get_plan(8, 17, 17, "ring", "f16x3", dev.index)
        return True
    except Exception:
        return False


def algorithmic(nside, L, M):
    """Per map: useful FLOPs of one Legendre contraction direction (N/S folded,
    triangle l >= m, each order stopped at its ring's truncation) and the
    algorithmic HBM bytes of every stage of the step (each operand read once,
    each result written once).  The table-driven contractions also stream the
    part of the resident fp16 hi/lo Legendre table they use once per launch:
    4 bytes per (ring pair, m, l), which equals the FLOP count per map."""
    NP = 2 * nside

    def nphi(tn):
        return 4 * (tn + 1) if tn < nside - 1 else 4 * nside

    flops = 0
    kept_pairs = 0
    for p in range(NP):
        mt = min(M, nphi(p) // 2 + 1)
        kept_pairs += mt
        flops += 4 * int(np.sum(np.maximum(L - np.arange(mt), 0)))
    kept = 0
    for t in range(4 * nside - 1):
        kept += min(M, nphi(t if t < NP else 4 * nside - 2 - t) // 2 + 1)
    npix = 12 * nside * nside
    tri = sum(L - m for m in range(M))
    stage_bytes = {
        "ring_fft_forward": 4 * npix + 8 * kept,  # real rings in, ring spectra out
        "ring_fft_inverse": 8 * kept + 4 * npix,
        "fold": 8 * kept + 16 * kept_pairs,  # spectra in, fp16 hi/lo S and D per (m, ring pair) out
        "unfold": 16 * kept_pairs + 8 * kept,  # E and O per (m, ring pair) in, spectra out
        "legendre_forward": 16 * kept_pairs + 8 * tri,  # operand in, order-major rows out (+ table)
        "columns_to_alm": 8 * tri + 8 * L * M,  # rows in, dense alm out
        "alm_to_columns": 8 * tri + 8 * tri,  # alm (m <= l) in once, fp16 hi/lo operand out (the max scan reads it again)
        "legendre_inverse": 8 * tri + 16 * kept_pairs,  # operand in, E and O out (+ table)
    }
    return flops, stage_bytes


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per 64-map launch of
# each stage's kernels at nside 1024, lmax = mmax = 2047, f16x3 with the resident
# table, from one single-pass ncu capture of this script's default workload:
# stage -> bytes.  Used for (nside, lmax, precision, batch) = (1024, 2047, f16x3, 64) only.
MEASURED_TRAFFIC = {
    "ring_fft_forward": (2183413760 + 2138995712) + (1166255872 + 1030015488),
    "ring_fft_inverse": (2179128064 + 2158633472) + (1164670208 + 1028427776),
    "fold": 3223599360 + 3172154880,
    "legendre_forward": 19562228480 + 1066144256,
    "columns_to_alm": 1088439040 + 2098970624,
    "alm_to_columns": (1088928768 + 386304) + (1088931584 + 1077855744),
    "legendre_inverse": 17077325824 + 3179270656,
    "unfold": 3252765440 + 3185650688,
}

def ring_kernel_count(nside):
    """Kernels of a ring stage: one per ring list the plan has -- power-of-two
    rings, Bluestein rings of length 2^K, Bluestein rings of length 3072 (for
    2h - 1 in (2048, 3072], nside <= 1024) -- for the rings' h = 2i (polar
    ring i) and 2 nside (equatorial rings)."""
    kinds = set()
    for h in list(range(2, 2 * nside, 2)) + [2 * nside]:
        if h & (h - 1) == 0:
            kinds.add(0)
        else:
            p2 = 1 << (2 * h - 2).bit_length()
            kinds.add(2 if (nside <= 1024 and 2 * h - 1 <= 3072 < p2) else 1)
    return len(kinds)


# kernels behind each stage's timer: the ring stages launch one kernel per ring
# list, and the mixed path's alm_to_columns is a max scan plus the conversion
# when the operand carries a per-map fp16 scale
def kernels_in_stage(name, prec, nside):
    if name.startswith("ring_fft"):
        return ring_kernel_count(nside)
    return 2 if (name == "alm_to_columns" and prec == "f16x3") else 1


def load_peaks():
    """(HBM GB/s, bf16 TFLOP/s for kernels timed inside a long step, source).

    The tensor-core contractions are timed inside the timed loop of whole
    SHT+iSHT steps, where the GPU runs at its power cap: their denominator is
    the sustained cuBLAS bf16 figure of MEASURED_PEAKS.json (bf16_tflops_sustained,
    a seconds-long GEMM loop under the same cap), not the burst one."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        pk = json.load(open(path))
        tf = pk.get("bf16_tflops_sustained") or pk.get("bf16_tflops", 1590.0)
        which = "bf16_tflops_sustained" if pk.get("bf16_tflops_sustained") else "bf16_tflops"
        return (pk.get("hbm_gbs", 6650.0), tf,
                f"MEASURED_PEAKS.json (measured): hbm_gbs, {which} (kernels timed inside the step loop)")
    return 6650.0, 1400.0, ("fallback (no MEASURED_PEAKS.json): 6650 GB/s and 1400 TFLOP/s sustained bf16, an "
                            "earlier measurement on this pool")


def roofline(stats, args, prec, refine, nside, L, B, table, stream=(0, 0)):
    """Roofline of every timed stage and of the dominant one (largest time).
    Table-driven contractions stream their operands and the part of the
    resident table that holds nonzero entries (`stream`: bytes per pass in each
    direction, from the plan) and are HBM-bound; their executed tensor-core
    rate is reported beside it."""
    hbm, bf16, source = load_peaks()
    flops_map, stage_bytes = algorithmic(nside, L, L)
    chunk = min(B, 64)
    measured = nside == 1024 and L == 2047 and prec == "f16x3" and chunk == 64 and table
    stages = {}
    for name, (n, tot) in stats.items():
        if not n:
            continue
        ms = tot / n
        e = {"ms_per_launch": ms}
        if name.startswith("legendre") and not (prec in ("bf16x3", "f16x3") and table):
            useful = flops_map * chunk
            if prec in ("bf16x3", "f16x3"):
                e.update(bound="tensor", achieved=3 * useful / (ms * 1e-3) / 1e12, peak=bf16, unit="TFLOP/s")
            else:
                e.update(bound="fp32_simt", achieved=useful / (ms * 1e-3) / 1e12, peak=FP32_SIMT_PEAK_TFLOPS,
                         unit="TFLOP/s")
        else:
            byts = stage_bytes.get(name, 0) * chunk
            if name.startswith("legendre"):
                tb = stream[0] if name == "legendre_forward" else stream[1]
                tb = tb or flops_map
                byts += tb
                # executed: 3 products over the table blocks streamed
                e["tensor_tflops"] = 3 * tb * chunk / (ms * 1e-3) / 1e12
                e["tensor_frac"] = e["tensor_tflops"] / bf16
                e["table_bytes"] = tb
            e.update(bound="hbm", achieved=byts / (ms * 1e-3) / 1e9, peak=hbm, unit="GB/s", algorithmic_bytes=byts)
        e["frac"] = e["achieved"] / e["peak"]
        e["traffic"] = MEASURED_TRAFFIC.get(name) if measured else None
        stages[name] = e
    dom = max(stats.items(), key=lambda kv: kv[1][1])[0]
    d = stages[dom]
    out = {"kernel": dom, "bound": d["bound"], "achieved": d["achieved"], "peak": d["peak"], "unit": d["unit"],
           "frac": d["frac"], "traffic": d["traffic"], "peak_source": source, "stages": stages}
    return out


# FP32 CUDA-core peak of a B200 at its maximum SM clock
FP32_SIMT_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def ragged_figures(torch, hpx, dev, prec, steps, warmup, loop_steps=2):
    """cfg4: 96 maps, nside drawn uniformly from {64, 128, 256, 512, 1024}
    (seed 4), L = M = 2 nside - 1 each, N(0, 1) pixels; one step is the
    analysis then the synthesis of all of them, timed (a) as a loop of one
    SHTCUDA and one iSHTCUDA call per map, (b) as one ragged analysis and one
    ragged synthesis call (groups concurrent on forked streams), (c) as the
    replay of those calls captured in CUDA graphs, with the fixed default
    schedule and with the autotuned one.  Returns maps/s of each."""
    rng = np.random.default_rng(4)
    draw = rng.choice([64, 128, 256, 512, 1024], size=96)
    nsides = sorted(set(int(n) for n in draw))
    counts = [int((draw == n).sum()) for n in nsides]
    g = torch.Generator(device=dev)
    g.manual_seed(4)
    maps = [torch.randn((c, 12 * n * n), generator=g, device=dev) for n, c in zip(nsides, counts)]
    singles = {n: hpx.SHTCUDA(n, lmax=2 * n - 1, mmax=2 * n - 1, precision=prec) for n in nsides}
    singles_i = {n: hpx.iSHTCUDA(n, lmax=2 * n - 1, mmax=2 * n - 1, precision=prec) for n in nsides}
    eager = hpx.RaggedSHT(nsides, precision=prec)
    eager_i = hpx.RaggedISHT(nsides, precision=prec)
    graphed = hpx.RaggedSHT(nsides, precision=prec, graph=True)
    graphed_i = hpx.RaggedISHT(nsides, precision=prec, graph=True)
    stream = torch.cuda.current_stream(dev)

    def loop():
        with torch.no_grad():
            for n, x in zip(nsides, maps):
                for i in range(x.shape[0]):
                    singles_i[n](singles[n](x[i:i + 1]))

    def one_call():
        with torch.no_grad():
            eager_i(eager(maps))

    def replay():
        with torch.no_grad():
            graphed_i(graphed(maps))

    def replay_analysis():
        with torch.no_grad():
            graphed(maps)

    res = {"nsides": nsides, "counts": counts}
    for name, fn, k in (("loop", loop, loop_steps), ("ragged_call", one_call, steps), ("graph", replay, steps),
                        ("graph_analysis", replay_analysis, steps)):
        ms = time_steps(torch, fn, k, warmup if name != "loop" else 1, None, stream)
        res[name + "_maps_per_s"] = 96 * k / (ms / 1000.0)
    # the graphs hold their inputs, outputs and workspaces: release them before
    # the autotuned pair captures its own
    del graphed, graphed_i, eager, eager_i
    torch.cuda.empty_cache()
    # the same with each group's schedule autotuned for its batch (plans are
    # shared, so the fixed default is restored afterwards)
    from cuhpx_b200 import autotune as AT

    plans = [hpx.get_plan(n, 2 * n - 1, 2 * n - 1, "ring", prec, dev.index) for n in nsides]
    saved = [AT.get_schedule(p) for p in plans]
    tuned_f = hpx.RaggedSHT(nsides, precision=prec, graph=True, autotune=True)
    tuned_i = hpx.RaggedISHT(nsides, precision=prec, graph=True, autotune=True)

    def replay_tuned():
        with torch.no_grad():
            tuned_i(tuned_f(maps))

    ms = time_steps(torch, replay_tuned, steps, warmup, None, stream)
    res["graph_autotuned_maps_per_s"] = 96 * steps / (ms / 1000.0)
    res["autotuned_schedules"] = {str(n): AT.get_schedule(p) for n, p in zip(nsides, plans)}
    del tuned_f, tuned_i
    torch.cuda.empty_cache()
    for p, s0 in zip(plans, saved):
        AT.set_schedule(p, s0)
    return res


def run_ragged(args):
    """The ragged workload (cfg4) as its own line; see ragged_figures."""
    import torch

    import cuhpx_b200 as hpx

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prec = "f16x3" if args.precision == "auto" else args.precision
    res = ragged_figures(torch, hpx, dev, prec, args.steps, args.warmup)
    line = {
        "metric": "ragged SHT+iSHT maps/s: 96 maps, nside in {64..1024}, L=M=2N-1",
        "value": res["graph_maps_per_s"],
        "unit": "maps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 96 * 1000.0 / res["graph_maps_per_s"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": f"f32 io, {prec} contraction",
        "data": "synthetic",
        "config": {"workload": "ragged SHT+iSHT, 96 maps", "nsides": res["nsides"], "counts": res["counts"],
                   "precision": prec},
        "ragged": res,
    }
    print(json.dumps(line), flush=True)
    return 0


# DRAM bytes (read + write) per nside-1024 float32 map of k_remap_async, NEST ->
# RING, from one ncu capture of an 8-map launch (795.9 MB: dram__bytes_read.sum
# + dram__bytes_write.sum), scaled by the maps
REMAP_TRAFFIC_PER_MAP = 795.9e6 / 8


def run_remap(args):
    """nest2ring of a batch of float32 maps (default 64 maps at nside 1024,
    3.2 GB each way, larger than L2) per step, the operation the reference's
    tests/reproduce_data_reorder_timing.py times (ms per map of a batched
    call).  The roofline is HBM: every pixel is read once and written once.
    Beside it: the other layout pairs, an end-to-end step through the public
    API from and to pinned host memory, and the CPU restatement of the
    reference's index formulas on one map."""
    import torch

    import cuhpx_b200 as hpx

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nside, B = args.nside, args.batch
    npix = 12 * nside * nside
    g = torch.Generator(device=dev)
    g.manual_seed(6)
    x = torch.randn((B, npix), generator=g, device=dev)
    stream = torch.cuda.current_stream(dev)

    def bench(fn):
        return time_steps(torch, fn, args.steps, args.warmup, None, stream)

    pairs = {
        "nest2ring": lambda: hpx.nest2ring(x, nside),
        "ring2nest": lambda: hpx.ring2nest(x, nside),
        "nest2flat": lambda: hpx.nest2flat(x, "S", False, nside),
        "ring2flat": lambda: hpx.ring2flat(x, "N", True, nside),
        "flat2flat": lambda: hpx.flat2flat(x, "S", False, "E", True, nside),
    }
    sampler = ClockSampler(0)
    sampler.start()
    ms = bench(pairs["nest2ring"])
    clocks = sampler.stop()
    out = {name: (ms if name == "nest2ring" else bench(fn)) for name, fn in pairs.items()}
    byts = 2.0 * npix * x.element_size() * B
    hbm, _, source = load_peaks()
    per_step = ms / args.steps
    ach = byts / (per_step * 1e-3) / 1e9

    # end to end: pinned host maps -> device -> nest2ring -> pinned host
    host_in = torch.empty((B, npix), dtype=torch.float32, pin_memory=True)
    host_in.copy_(x)
    host_out = torch.empty_like(host_in, pin_memory=True)
    e2e_steps = max(3, min(args.steps, 10))

    def e2e():
        d = host_in.to(dev, non_blocking=True)
        host_out.copy_(hpx.nest2ring(d, nside), non_blocking=True)

    e2e_ms = time_steps(torch, e2e, e2e_steps, args.warmup, None, stream)
    cpu = None
    if not args.no_cpu:
        from oracle import remap_oracle as R

        one = x[0].cpu().numpy()
        reps, t0 = 0, time.perf_counter()
        while reps < 3 or time.perf_counter() - t0 < 10.0:
            R.nest2ring(one, nside)
            reps += 1
        cpu_ms = (time.perf_counter() - t0) / reps * 1e3
        cpu = {"value": 1e3 / cpu_ms, "unit": "maps/s", "cores": 1, "kind": "port",
               "sample": f"oracle nest2ring (numpy, the reference's index formulas) of one nside-{nside} map, "
                         f"{reps} repetitions"}
    line = {
        "metric": f"nest2ring maps/s nside{nside} B{B} float32",
        "value": B / (per_step * 1e-3),
        "unit": "maps/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per_step,
        "ms_per_map": per_step / B,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (bytes moved)",
        "data": "synthetic",
        "config": {"workload": f"nest2ring, {B} maps of nside {nside}", "nside": nside, "batch": B,
                   "l2": f"inputs larger than L2 ({byts / 2e9:.2f} GB each way per step)"},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                     "traffic": REMAP_TRAFFIC_PER_MAP * B if nside == 1024 else None, "kernel": "k_remap_async",
                     "peak_source": source, "algorithmic_bytes": byts},
        "other_pairs_gbs": {k: byts / (v / args.steps * 1e-3) / 1e9 for k, v in out.items()},
        "e2e": {"value": B * e2e_steps / (e2e_ms * 1e-3), "unit": "maps/s", "h2d_bytes_per_step": npix * 4 * B,
                "d2h_bytes_per_step": npix * 4 * B, "steps": e2e_steps},
        "gpu_launches": args.steps,
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_next(args):
    """The rows beside the headline path, timed on one GPU (maps/s, CUDA events,
    inputs resident, 3 warm-up steps):
      cfg5_loss   -- loss = sum_lm w_l |a_lm|^2, w_l = 1/(l+1), over the SHT of 16
                     maps at nside 512, L = M = 1023, forward and backward (FP32
                     SIMT and f16x3);
      cfg5_regrid -- Regridding HEALPix nside 256 -> equiangular 512 x 1024 at
                     L = M = 511, 16 maps, forward, and forward with backward;
      vector      -- spin-1 VectorSHTCUDA then VectoriSHTCUDA of 16 tangent
                     fields at nside 256, L = M = 511 (FP32), with the rel-L2 of
                     the analysis against the FP64 path on 2 fields;
      healpy      -- dense [64][2048][2048] complex64 a_lm -> healpy packing and
                     back: GB/s of each against the HBM peak."""
    import torch

    import cuhpx_b200 as hpx

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    steps, warm = args.steps, max(args.warmup, 3)
    g = torch.Generator(device=dev)
    g.manual_seed(7)
    hbm, _, source = load_peaks()
    rows = {}

    def rate(fn, maps):
        ms = time_steps(torch, fn, steps, warm, None, stream) / steps
        return {"ms_per_step": ms, "maps_per_s": maps / (ms * 1e-3)}

    # cfg5: power-spectrum loss through the SHT, with backward
    nside, L, B = 512, 1023, 16
    f = torch.randn((B, 12 * nside * nside), generator=g, device=dev)
    w = (1.0 / (torch.arange(L, device=dev, dtype=torch.float32) + 1.0))[:, None]
    rows["cfg5_loss"] = {"config": f"{B} maps, nside {nside}, L = M = {L}, loss + backward"}
    for prec in ("fp32", "f16x3"):
        sht = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision=prec)
        x = f.clone().requires_grad_(True)

        def loss_step():
            x.grad = None
            (w * sht(x).abs() ** 2).sum().backward()

        rows["cfg5_loss"][prec] = rate(loss_step, B)
        del sht
    # cfg5: regridding HEALPix 256 -> equiangular 512 x 1024, forward and with backward
    rg = hpx.Regridding(hpx.Grid("healpix", 256), hpx.Grid("equiangular", (512, 1024)), lmax=511, mmax=511)
    fr = torch.randn((B, 12 * 256 * 256), generator=g, device=dev)
    xr = fr.clone().requires_grad_(True)

    def regrid_fwd():
        with torch.no_grad():
            rg(fr)

    def regrid_bwd():
        xr.grad = None
        (rg(xr) ** 2).sum().backward()

    rows["cfg5_regrid"] = {"config": f"{B} maps, HEALPix 256 -> equiangular 512 x 1024, L = M = 511 (FP32)",
                           "forward": rate(regrid_fwd, B), "forward_backward": rate(regrid_bwd, B)}
    # spin-1 transforms
    nside, L = 256, 511
    vs = hpx.VectorSHTCUDA(nside, lmax=L, mmax=L)
    vi = hpx.VectoriSHTCUDA(nside, lmax=L, mmax=L)
    v = torch.randn((B, 2, 12 * nside * nside), generator=g, device=dev)

    def vec_step():
        with torch.no_grad():
            vi(vs(v))

    rows["vector"] = {"config": f"{B} tangent fields, nside {nside}, L = M = {L}, analysis then synthesis (FP32)"}
    rows["vector"].update(rate(vec_step, B))
    with torch.no_grad():
        a32 = vs(v[:2])
        a64 = vs(v[:2].double())
    rows["vector"]["analysis_rel_l2_vs_fp64"] = float((a32.to(a64.dtype) - a64).abs().pow(2).sum().sqrt()
                                                      / a64.abs().pow(2).sum().sqrt())
    del vs, vi, v
    # healpy packing
    Lh, Bh = 2048, 64
    dense = torch.randn((Bh, Lh, Lh), generator=g, device=dev, dtype=torch.complex64)
    dense = torch.tril(dense)
    packed = hpx.alm_to_healpy(dense)

    def pack():
        hpx.alm_to_healpy(dense)

    def unpack():
        hpx.healpy_to_alm(packed, Lh)

    bytes_pack = dense.numel() * 8 + packed.numel() * 8
    rp, ru = rate(pack, Bh), rate(unpack, Bh)
    rows["healpy"] = {"config": f"{Bh} x [{Lh}][{Lh}] complex64 <-> packed [{packed.shape[-1]}]",
                      "pack": dict(rp, gbs=bytes_pack / (rp["ms_per_step"] * 1e-3) / 1e9,
                                   frac=bytes_pack / (rp["ms_per_step"] * 1e-3) / 1e9 / hbm),
                      "unpack": dict(ru, gbs=bytes_pack / (ru["ms_per_step"] * 1e-3) / 1e9,
                                     frac=bytes_pack / (ru["ms_per_step"] * 1e-3) / 1e9 / hbm),
                      "peak_source": source}
    line = {
        "metric": "rows beside the headline path: cfg5 loss and regridding with backward, spin-1, healpy packing",
        "value": rows["cfg5_loss"]["f16x3"]["maps_per_s"],
        "unit": "maps/s (cfg5 loss + backward, f16x3)",
        "n_gpus": 1,
        "steps": steps,
        "warmup": warm,
        "higher_is_better": True,
        "data": "synthetic",
        "rows": rows,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ragged":
        return run_ragged(args)
    if args.workload == "remap":
        return run_remap(args)
    if args.workload == "next":
        return run_next(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
