"""The CPU oracle against golden vectors produced by the cuHPX reference itself.

``tests/golden/make_golden.py`` ran the reference's CPU ``SHT``/``iSHT``
(cuhpx/hpx_sht.py:173-283) on seeded inputs.  The reference's float64 path
evaluates the ring phase factor in complex64 (cuhpx/hpx_sht.py:50, 64); with
``phase_dtype=np.complex64`` the oracle reproduces that rounding and must agree
to ~1e-13, and with exact phases it must agree to the size of that rounding.
"""

import os

import numpy as np
import pytest

from oracle import hpx_oracle as O

G = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def load(name):
    return np.load(os.path.join(G, name))


def test_cfg1_forward_inverse_pinned():
    d = load("cfg1_n32.npz")
    a = O.sht(d["f"], 32, 65, 65, phase_dtype=np.complex64)
    assert rel(a, d["alm64"]) < 1e-13
    f = O.isht(d["alm64"], 32, phase_dtype=np.complex64)
    assert rel(f, d["map64"]) < 1e-13
    # exact phases: differs from the reference only by its complex64 phase rounding
    assert rel(O.sht(d["f"], 32, 65, 65), d["alm64"]) < 1e-7
    assert rel(O.isht(d["alm64"], 32), d["map64"]) < 1e-7
    # the reference's own float32 run is within 1e-6 of its float64 run
    assert rel(d["alm32"], d["alm64"]) < 1e-6


@pytest.mark.parametrize("nside", [2, 4, 8, 16])
@pytest.mark.parametrize("variant", ["default_", "equal_"])
def test_small_nside(nside, variant):
    d = load(f"small_n{nside}.npz")
    L, M = int(d[variant + "lmax"]), int(d[variant + "mmax"])
    a = O.sht(d[variant + "f"], nside, L, M, phase_dtype=np.complex64)
    assert a.shape == (L, M)
    assert rel(a, d[variant + "alm64"]) < 1e-13
    f = O.isht(d[variant + "alm64"], nside, phase_dtype=np.complex64)
    assert rel(f, d[variant + "map64"]) < 1e-13


def test_uniform_weights():
    d = load("none_n8.npz")
    a = O.sht(d["f"], 8, 17, 17, quad_weights="none", phase_dtype=np.complex64)
    assert rel(a, d["alm64"]) < 1e-13


@pytest.mark.parametrize("p", ["mgt_", "mlt_"])
def test_lmax_mmax_mismatch(p):
    d = load("lm_n8.npz")
    L, M = int(d[p + "lmax"]), int(d[p + "mmax"])
    a = O.sht(d[p + "f"], 8, L, M, phase_dtype=np.complex64)
    assert rel(a, d[p + "alm64"]) < 1e-13
    assert rel(O.isht(d[p + "alm64"], 8, phase_dtype=np.complex64), d[p + "map64"]) < 1e-13


def test_sparse_round_trip():
    d = load("sparse_n16.npz")
    m = O.isht(d["alm"], 16, phase_dtype=np.complex64)
    assert rel(m, d["map64"]) < 1e-13
    b = O.sht(d["map64"], 16, 33, 33, phase_dtype=np.complex64)
    assert rel(b, d["alm_back64"]) < 1e-13


def test_legendre_variants_agree():
    x = np.cos(O.ring_theta(16))
    T = O.legendre_table(20, 33, x)
    B = np.stack([p for _, p in O.legendre_by_l(20, 33, x)], 1)
    assert np.array_equal(T, B)
    for m in range(20):
        assert np.array_equal(O.legendre_column(m, 33, x), T[m])


def test_spot_oracle_matches_full():
    d = load("cfg1_n32.npz")
    ms = [0, 1, 7, 31, 64]
    s = O.sht_spot(d["f"], 32, 65, 65, ms)
    a = O.sht(d["f"], 32, 65, 65)
    assert rel(s, a[:, ms]) < 1e-14


def test_geometry_sums():
    for nside in (1, 2, 4, 32):
        tot = sum(O.nphi_ring(t, nside) for t in range(O.nrings(nside)))
        assert tot == O.npix(nside)
        for t in range(O.nrings(nside)):
            assert O.ring_start(t, nside) == sum(O.nphi_ring(u, nside) for u in range(t))
    z = O.ring_z(16)
    assert np.allclose(z, -z[::-1], atol=0, rtol=0) or np.abs(z + z[::-1]).max() < 1e-15


def test_weights_sum_to_sphere_area():
    for nside in (2, 8, 32, 1024):
        w = O.ring_weights(nside)
        nphi = np.array([O.nphi_ring(t, nside) for t in range(O.nrings(nside))])
        # pixel-weighted sum of the quadrature weights integrates 1 over the sphere
        assert abs((w * nphi).sum() / (4 * np.pi) - 1) < 5e-3


@pytest.mark.parametrize("name,L,M", [("cfg1_n32.npz", 65, 65), ("lm_n8.npz", 9, 17), ("lm_n8.npz", 17, 5)])
def test_per_order_oracle_matches_full(name, L, M):
    # the per-order transforms (used where the full ones would take minutes)
    # give the golden-pinned values
    d = load(name)
    nside = 32 if name.startswith("cfg1") else 8
    f = d["f"] if "f" in d.files else d["mgt_f"]
    a = O.sht(f, nside, L, M)
    assert rel(O.sht_by_m(f, nside, L, M), a) < 1e-14
    assert rel(O.isht_by_m(a, nside), O.isht(a, nside)) < 1e-14


@pytest.fixture(scope="module")
def ref_cpu():
    from oracle import ref_cpu as RC

    try:
        RC.load()
    except Exception as e:  # no C compiler with OpenMP on this machine
        pytest.skip(f"ref_cpu not built: {e}")
    return RC


@pytest.mark.parametrize("nside,L,M", [(8, 17, 17), (8, 9, 17), (8, 17, 5), (16, 33, 33), (32, 65, 65)])
def test_cpu_baseline_port_matches_oracle(ref_cpu, nside, L, M):
    # the multi-threaded C port that bench.py times as the reference's CPU
    # implementation computes the oracle's transforms
    rng = np.random.default_rng(nside + L + M)
    f = rng.standard_normal(12 * nside * nside)
    a = O.sht(f, nside, L, M)
    assert rel(ref_cpu.sht(f, nside, L, M), a) < 1e-13
    assert rel(ref_cpu.isht(a, nside), O.isht(a, nside)) < 1e-13


def test_cpu_baseline_port_matches_reference_goldens(ref_cpu):
    d = load("cfg1_n32.npz")
    assert rel(ref_cpu.sht(d["f"], 32, 65, 65), d["alm64"]) < 1e-7
    assert rel(ref_cpu.isht(d["alm64"], 32), d["map64"]) < 1e-7


def test_spot_oracle_exact_nodes_close_to_reference_nodes():
    # the exact nodes differ from the reference's cos(arccos z) by roundings only
    d = load("cfg1_n32.npz")
    ms = [0, 1, 7, 31, 64]
    a = O.sht_spot(d["f"], 32, 65, 65, ms)
    b = O.sht_spot(d["f"], 32, 65, 65, ms, nodes="exact")
    assert 0 < rel(b, a) < 1e-12
    s2 = O.ring_sin2(32)
    z = O.ring_z(32)
    assert np.abs(s2 - (1 - z) * (1 + z)).max() < 1e-15


def test_extended_legendre_against_50_digit_recurrence():
    # Near the poles the reference's FP64 diagonal Pbar_m^m goes subnormal for
    # high orders, and the recurrence carries the lost bits up to degrees where
    # the values matter.  At nside 1024, m = 1023, ring 624 (sin theta = 0.483)
    # the FP64 diagonal is the smallest subnormal and Pbar_2046^1023 comes out
    # 0 instead of 3.3e-4; at ring 625 it is 13% off.  The extended-precision
    # column of the exact-node spot oracle matches the same recurrence run with
    # 50 digits.
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 50
    N, L, m = 1024, 2047, 1023
    rings = np.array([600, 624, 625, 660, 700])
    z = O.ring_z(N)[rings]
    s2 = O.ring_sin2(N)[rings]
    ext = O.legendre_column_extended(m, L, z, s2)
    ref = O.legendre_column(m, L, z, s2)
    for k in range(len(rings)):
        x, sq = mpmath.mpf(z[k]), mpmath.mpf(s2[k])
        d = 1 / mpmath.sqrt(4 * mpmath.pi)
        for l in range(1, m + 1):
            d = mpmath.sqrt((2 * l + 1) * sq / (2 * l)) * d
        p2, p1 = d, mpmath.sqrt(2 * m + 3) * x * d
        for l in range(m + 2, L):
            f1 = mpmath.sqrt(mpmath.mpf(2 * l - 1) / (l - m) * (2 * l + 1) / (l + m))
            f2 = mpmath.sqrt(mpmath.mpf(l + m - 1) / (l - m) * (2 * l + 1) / (2 * l - 3) * (l - m - 1) / (l + m))
            p2, p1 = p1, x * f1 * p1 - f2 * p2
        want = float(p1)  # degree L - 1
        assert abs(ext[L - 1, k] - want) <= 1e-14 * abs(want), rings[k]
    assert ref[L - 1, 1] == 0.0 and abs(ext[L - 1, 1] - 3.26e-4) < 1e-6
    assert abs(ref[L - 1, 2] / ext[L - 1, 2] - 1) > 0.1


def test_reference_fp64_recurrence_diverges_at_nside1024():
    # The reference's own table at nside 1024, L = 2047: for m = 1198 on the
    # south ring 3445 (sin theta = 0.5006) its FP64 diagonal is subnormal, the
    # start pair is inconsistent and the three-term recurrence picks up the
    # wrong solution: Pbar_2046^1198 comes out ~40 where the true value is
    # ~1e-35.  The extended-precision column does not.
    N, L, m, t = 1024, 2047, 1198, 3445
    z, s2 = O.ring_z(N)[[t]], O.ring_sin2(N)[[t]]
    ref = O.legendre_column(m, L, np.cos(O.ring_theta(N))[[t]])
    ext = O.legendre_column_extended(m, L, z, s2)
    assert abs(ref[L - 1, 0]) > 1.0
    assert abs(ext[L - 1, 0]) < 1e-30


@pytest.mark.parametrize("nside,L,M", [(8, 17, 17), (16, 33, 33), (32, 65, 65)])
def test_cpu_port_extended_matches_oracle(ref_cpu, nside, L, M):
    # where nothing underflows, the extended-precision port agrees with the oracle
    rng = np.random.default_rng(nside)
    f = rng.standard_normal(12 * nside * nside)
    a = O.sht(f, nside, L, M)
    assert rel(ref_cpu.sht_extended(f, nside, L, M), a) < 1e-12
    assert rel(ref_cpu.isht_extended(a, nside), O.isht(a, nside)) < 1e-12
