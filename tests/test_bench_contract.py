"""The bench.py contract on the CPU: the reference arm's JSON line, and the
ring-kernel count its launch tally uses.

The reference arm (``--impl reference``) runs the C port of the reference's CPU
transform on the host, so it needs no GPU: at nside 32 (L = M = 65) one step
takes milliseconds.  Its one JSON line must carry the keys the driver reads.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


@pytest.fixture(scope="module")
def ref_line():
    from oracle import ref_cpu

    try:
        ref_cpu.load()
    except Exception as e:
        pytest.skip(f"CPU port not built: {e}")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nside", "32",
                          "--lmax", "65", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line(ref_line):
    d = ref_line
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC
    assert d["value"] > 0 and d["unit"] == "maps/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 3  # warm-up is raised to at least 3
    # steps x ms_per_step is the timed region, and value is its rate
    assert abs(d["value"] - 1000.0 / d["ms_per_step"]) <= 1e-6 * d["value"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def _kinds_by_rule(nside):
    """The ring lists a HEALPix plan builds, from the rule in hpx_plan.cu:
    power-of-two h, Bluestein 2^K, and Bluestein 3072 where 2h - 1 lies in
    (2048, 3072] (nside <= 1024)."""
    kinds = set()
    hs = [2 * i for i in range(1, nside)] + [2 * nside]
    for h in hs:
        if h & (h - 1) == 0:
            kinds.add("pow2")
        elif nside <= 1024 and 2048 < 2 * h - 1 <= 3072:
            kinds.add("3072")
        else:
            kinds.add("2^K")
    return kinds


@pytest.mark.parametrize("nside", [1, 2, 8, 64, 300, 512, 513, 600, 768, 1024, 2048])
def test_ring_kernel_count(nside):
    assert bench.ring_kernel_count(nside) == len(_kinds_by_rule(nside))


def test_ring_kernel_count_headline():
    # nside 1024: power-of-two equatorial rings, 2^K and 3072-point Bluestein rings
    assert bench.ring_kernel_count(1024) == 3
    assert bench.kernels_in_stage("ring_fft_forward", "f16x3", 1024) == 3
    assert bench.kernels_in_stage("alm_to_columns", "f16x3", 1024) == 2
    assert bench.kernels_in_stage("fold", "f16x3", 1024) == 1
