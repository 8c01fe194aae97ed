"""Launch schedules and their autotuner.

Every schedule (ring-FFT maps per CTA, analysis and synthesis tile deals,
CTA count) must give bit-identical transforms; the autotuner must pick one,
apply it, store it in its JSON cache and, in a later call, apply the cached
one without measuring.
"""

import json

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def hpx(cuda):
    import cuhpx_b200

    return cuhpx_b200


@pytest.mark.parametrize("prec", ["f16x3", "fp32"])
def test_every_schedule_is_bit_identical(hpx, cuda, prec):
    from cuhpx_b200 import autotune as AT

    nside, L = 32, 63
    plan = hpx.get_plan(nside, L, L, "ring", prec, 0)
    g = torch.Generator(device=cuda).manual_seed(3)
    x = torch.randn(70, 12 * nside * nside, generator=g, device=cuda)
    default = AT.get_schedule(plan)
    assert default == {"ring_maps_per_cta": 16, "fwd_deal": "order_snake", "inv_deal": "order_snake", "ctas": 0,
                       "ring_streams": 2}
    ref_a = plan.forward(x)
    ref_f = plan.inverse(ref_a)
    deals = AT.DEALS if prec == "f16x3" else ("order_snake",)
    try:
        for gsz in AT.RING_GROUPS:
            for d in deals:
                for ctas, rs in ((0, 2), (37, 1)):
                    s = {"ring_maps_per_cta": gsz, "fwd_deal": d, "inv_deal": d, "ctas": ctas, "ring_streams": rs}
                    AT.set_schedule(plan, s)
                    assert AT.get_schedule(plan) == s
                    a = plan.forward(x)
                    assert torch.equal(a, ref_a), s
                    assert torch.equal(plan.inverse(ref_a), ref_f), s
    finally:
        AT.set_schedule(plan, default)
    with pytest.raises(RuntimeError, match="ring_maps_per_cta"):
        AT.set_schedule(plan, dict(default, ring_maps_per_cta=12))


def test_autotune_caches_and_reapplies(hpx, cuda, tmp_path, monkeypatch):
    from cuhpx_b200 import autotune as AT

    monkeypatch.setenv("HPX_TUNE_CACHE", str(tmp_path / "schedules.json"))
    nside, L = 64, 127
    plan = hpx.get_plan(nside, L, L, "ring", "f16x3", 0)
    default = AT.get_schedule(plan)
    try:
        r = AT.tune(plan, 64, warmup=1, reps=2)
        assert not r["cached"]
        # every candidate was timed: 4 ring groupings, 2 ring-stream modes and 4 deals in each direction
        assert len(r["ms"]) == 14 and all(v > 0 for v in r["ms"].values())
        assert AT.get_schedule(plan) == r["schedule"]
        data = json.loads((tmp_path / "schedules.json").read_text())
        assert AT.key(plan, 64) in data
        AT.set_schedule(plan, default)
        r2 = AT.tune(plan, 64)
        assert r2["cached"] and r2["schedule"] == r["schedule"]
        assert AT.get_schedule(plan) == r["schedule"]
        # a module with autotune=True runs on the tuned schedule and gives the same results
        g = torch.Generator(device=cuda).manual_seed(5)
        x = torch.randn(8, 12 * nside * nside, generator=g, device=cuda)
        want = plan.forward(x)
        got = hpx.SHTCUDA(nside, lmax=L, mmax=L, precision="f16x3", autotune=True)(x)
        assert torch.equal(got, want)
    finally:
        AT.set_schedule(plan, default)
