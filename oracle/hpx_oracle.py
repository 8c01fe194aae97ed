"""CPU oracle for the HEALPix real SHT / inverse SHT -- TEST INFRASTRUCTURE ONLY.

This module restates, in float64 numpy, the algorithm of the cuHPX reference's
CPU transforms so that the CUDA path can be checked against it.  It is the
checker, never the product: only the test suite, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` may import it.

Parity is pinned: ``tests/test_oracle_golden.py`` compares every function
here against golden vectors written by ``tests/golden/make_golden.py``, which
runs the reference's own ``cuhpx.SHT`` / ``cuhpx.iSHT`` (CPU torch path).

Reference functions restated (paths relative to the cuHPX repository):
  ring_z / ring_theta       cuhpx/sht_tools.py:114-140  (healpix_weights, z formula)
  ring_weights              cuhpx/sht_tools.py:34-59, 131-134 (apply_ring_weight)
  nphi_ring                 cuhpx/sht_tools.py:179-189
  ring_start                cuhpx/sht_tools.py:319-332  (cumulative_nphi_ring)
  ring_phi0                 cuhpx/sht_tools.py:161-176  (p2phi_ring with p=0)
  legendre_table / _by_l    cuhpx/sht_tools.py:192-229  (legpoly, norm='ortho')
  ring_rfft                 cuhpx/hpx_sht.py:37-55      (healpix_rfft_torch)
  ring_irfft                cuhpx/hpx_sht.py:58-76      (healpix_irfft_torch)
  sht / isht                cuhpx/hpx_sht.py:214-236, 268-283 (SHT.forward, iSHT.forward)
"""

import os

import numpy as np

_WEIGHTS_NPZ = os.path.join(
    os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cuhpx_b200", "data", "ring_weights.npz"
)


# --------------------------------------------------------------------------- geometry
def nrings(nside):
    return 4 * nside - 1


def npix(nside):
    return 12 * nside * nside


def nphi_ring(t, nside):
    """Pixels on ring t (0 = northernmost).  cuhpx/sht_tools.py:179-189."""
    if 0 <= t < nside - 1:
        return 4 * (t + 1)
    if nside - 1 <= t <= 3 * nside - 1:
        return 4 * nside
    if 3 * nside - 1 < t <= 4 * nside - 2:
        return 4 * (4 * nside - t - 1)
    raise ValueError(f"ring {t} outside nside={nside}")


def ring_start(t, nside):
    """First pixel index of ring t in RING order.  cuhpx/sht_tools.py:319-332."""
    if 0 <= t < nside:
        return 2 * t * (t + 1)
    if t < 3 * nside:
        return 2 * nside * (nside + 1) + (t - nside) * 4 * nside
    if t < 4 * nside:
        r = 4 * nside - t - 1
        return 12 * nside * nside - 2 * r * (r + 1)
    raise ValueError(f"ring {t} outside nside={nside}")


def ring_phi0(t, nside):
    """Longitude of the first pixel of ring t.  cuhpx/sht_tools.py:161-176 (p=0)."""
    shift = 0.5
    if nside <= t + 1 <= 3 * nside:
        shift *= (t - nside + 2) % 2
        return np.pi / (2 * nside) * shift
    if t + 1 > 3 * nside:
        return np.pi / (2 * (4 * nside - t - 1)) * shift
    return np.pi / (2 * (t + 1)) * shift


def ring_z(nside):
    """z = cos(theta) of every ring, north to south.  cuhpx/sht_tools.py:114-140.

    The reference flips z to south->north and then flips theta back
    (cuhpx/hpx_sht.py:192, 665), so ring t is at the z given here.
    """
    t = np.arange(4 * nside - 1)
    z = np.zeros(t.shape, dtype=np.float64)
    m1 = t < nside - 1
    m2 = (t >= nside - 1) & (t <= 3 * nside - 1)
    m3 = (t > 3 * nside - 1) & (t <= 4 * nside - 2)
    z[m1] = 1 - ((t[m1] + 1) ** 2) / (3 * nside**2)
    z[m2] = 4 / 3 - 2 * (t[m2] + 1) / (3 * nside)
    z[m3] = ((4 * nside - 1 - t[m3]) ** 2) / (3 * nside**2) - 1
    return z


def ring_sin2(nside):
    """sin^2(theta) of every ring from the z formula without cancellation near
    the poles: a (2 - a) with a = 1 - |z| = (t+1)^2 / (3 nside^2) on the polar
    rings, (1 - z)(1 + z) elsewhere (the "exact" nodes of ``sht_spot``)."""
    t = np.arange(4 * nside - 1)
    tn = np.where(t < 2 * nside, t, 4 * nside - 2 - t)
    a = (tn + 1.0) ** 2 / (3.0 * nside**2)
    z = ring_z(nside)
    return np.where(tn < nside - 1, a * (2.0 - a), (1.0 - z) * (1.0 + z))


def ring_theta(nside):
    """theta of every ring, north to south, as the reference derives it (arccos of z)."""
    return np.arccos(ring_z(nside))


def fits_ring_weights(nside):
    """The 2*nside HEALPix ring-weight corrections (FITS column 0)."""
    with np.load(_WEIGHTS_NPZ) as d:
        key = f"n{nside}"
        if key not in d:
            raise ValueError(f"no ring weights for nside={nside}")
        return np.array(d[key], dtype=np.float64)


def ring_weights(nside, quad_weights="ring"):
    """Quadrature weight of each ring.  cuhpx/sht_tools.py:47-59 and 131-134."""
    R = 4 * nside - 1
    if quad_weights != "ring":
        return np.full(R, 4.0 * np.pi / npix(nside))
    w = fits_ring_weights(nside)
    out = np.zeros(R)
    for t in range(R):
        ring = t + 1
        north = 4 * nside - ring if ring > 2 * nside else ring
        out[t] = 4.0 * np.pi / npix(nside) * (1.0 + w[north - 1])
    return out


# --------------------------------------------------------------------------- Legendre
def _rec_coeffs(l, m):
    """Three-term coefficients of cuhpx/sht_tools.py:215-218, same operation order."""
    f1 = np.sqrt((2 * l - 1) / (l - m) * (2 * l + 1) / (l + m))
    f2 = np.sqrt((l + m - 1) / (l - m) * (2 * l + 1) / (2 * l - 3) * (l - m - 1) / (l + m))
    return f1, f2


def legendre_table(mmax, lmax, x):
    """Orthonormal P[m, l, k] = Pbar_l^m(x_k), no Condon-Shortley phase, zero for l<m.

    Restates ``legpoly`` (cuhpx/sht_tools.py:192-229) with norm='ortho'.  Memory
    is O(max(M,L)^2 * len(x)); use ``legendre_by_l`` for large cases.
    """
    x = np.asarray(x, dtype=np.float64)
    nmax = max(mmax, lmax)
    vdm = np.zeros((nmax, nmax, x.size))
    vdm[0, 0] = 1.0 / np.sqrt(4 * np.pi)
    for l in range(1, nmax):
        vdm[l - 1, l] = np.sqrt(2 * l + 1) * x * vdm[l - 1, l - 1]
        vdm[l, l] = np.sqrt((2 * l + 1) * (1 + x) * (1 - x) / 2 / l) * vdm[l - 1, l - 1]
    for l in range(2, nmax):
        for m in range(0, l - 1):
            f1, f2 = _rec_coeffs(l, m)
            vdm[m, l] = x * f1 * vdm[m, l - 1] - f2 * vdm[m, l - 2]
    return vdm[:mmax, :lmax]


def legendre_by_l(mmax, lmax, x):
    """Yield (l, P_l[m, k]) for l = 0..lmax-1 with O(M * len(x)) memory.

    Same recurrence and operation order as ``legendre_table``; the rows for
    m > l are zero.
    """
    x = np.asarray(x, dtype=np.float64)
    nmax = max(mmax, lmax)
    K = x.size
    # diagonal Pbar_m^m for all m < nmax, built as the reference builds it
    diag = np.zeros((nmax, K))
    diag[0] = 1.0 / np.sqrt(4 * np.pi)
    for l in range(1, nmax):
        diag[l] = np.sqrt((2 * l + 1) * (1 + x) * (1 - x) / 2 / l) * diag[l - 1]
    ms = np.arange(nmax)
    p2 = np.zeros((nmax, K))  # P_{l-2}
    p1 = np.zeros((nmax, K))  # P_{l-1}
    for l in range(0, lmax):
        pl = np.zeros((nmax, K))
        if l >= 2:
            mm = ms[: l - 1]
            f1 = np.sqrt((2 * l - 1) / (l - mm) * (2 * l + 1) / (l + mm))
            f2 = np.sqrt((l + mm - 1) / (l - mm) * (2 * l + 1) / (2 * l - 3) * (l - mm - 1) / (l + mm))
            pl[: l - 1] = x * f1[:, None] * p1[: l - 1] - f2[:, None] * p2[: l - 1]
        if l >= 1:
            pl[l - 1] = np.sqrt(2 * l + 1) * x * diag[l - 1]
        if l < nmax:
            pl[l] = diag[l]
        yield l, pl[:mmax]
        p2, p1 = p1, pl


def legendre_column(m, lmax, x, s2=None):
    """Pbar_l^m(x) for one m and l < lmax (spot oracle; O(lmax * len(x)) memory).

    The diagonal uses sin^2 = (1 + x)(1 - x) as the reference does, or ``s2``
    when given."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((lmax, x.size))
    d = np.full(x.shape, 1.0 / np.sqrt(4 * np.pi))
    for l in range(1, m + 1):
        if s2 is None:  # the reference's operation order (cuhpx/sht_tools.py:208)
            d = np.sqrt((2 * l + 1) * (1 + x) * (1 - x) / 2 / l) * d
        else:
            d = np.sqrt((2 * l + 1) * s2 / 2 / l) * d
    if m < lmax:
        out[m] = d
    if m + 1 < lmax:
        out[m + 1] = np.sqrt(2 * (m + 1) + 1) * x * d
    for l in range(m + 2, lmax):
        f1, f2 = _rec_coeffs(l, m)
        out[l] = x * f1 * out[l - 1] - f2 * out[l - 2]
    return out


def legendre_column_extended(m, lmax, x, s2):
    """``legendre_column`` carried in 80-bit extended precision (np.longdouble,
    exponent range to 1e-4951) and returned as float64.

    The reference's FP64 diagonal Pbar_m^m ~ sin^m(theta) goes subnormal below
    1e-308 for high m near the poles (at nside 1024, orders above ~500); where
    the recurrence then grows those values back to O(1e-2) within l < L they
    carry the subnormal's lost bits (relative errors up to ~1e-6 in orders near
    1023).  Here nothing underflows that matters, so this is the accurate
    column at the given nodes."""
    ld = np.longdouble
    x = np.asarray(x, dtype=np.float64).astype(ld)
    sq = np.asarray(s2, dtype=np.float64).astype(ld)
    out = np.zeros((lmax, x.size), dtype=ld)
    d = np.full(x.shape, ld(1) / np.sqrt(ld(4) * ld(np.pi)), dtype=ld)
    for l in range(1, m + 1):
        d = np.sqrt(ld(2 * l + 1) * sq / ld(2 * l)) * d
    if m < lmax:
        out[m] = d
    if m + 1 < lmax:
        out[m + 1] = np.sqrt(ld(2 * (m + 1) + 1)) * x * d
    for l in range(m + 2, lmax):
        f1 = np.sqrt(ld(2 * l - 1) / ld(l - m) * ld(2 * l + 1) / ld(l + m))
        f2 = np.sqrt(ld(l + m - 1) / ld(l - m) * ld(2 * l + 1) / ld(2 * l - 3) * ld(l - m - 1) / ld(l + m))
        out[l] = x * f1 * out[l - 1] - f2 * out[l - 2]
    return out.astype(np.float64)


# --------------------------------------------------------------------------- ring FFTs
def _phase(ms, phi0, sign, phase_dtype):
    """e^{sign i m phi0}.

    The reference builds this factor as ``torch.exp(-1j * torch.arange(L) * phi0)``
    (cuhpx/hpx_sht.py:50, 64), which torch evaluates in complex64 even when the
    data are float64.  ``phase_dtype=np.complex64`` reproduces that rounding
    (used to pin this oracle to the reference's float64 outputs); the default
    complex128 gives the exact transform.
    """
    if phase_dtype == np.complex64:
        return np.exp(np.complex64(sign * 1j) * (ms.astype(np.float32) * np.float32(phi0)))
    return np.exp(sign * 1j * ms * phi0)


def ring_rfft(f, mmax, nside, phase_dtype=np.complex128):
    """ftm[..., t, m] = e^{-i m phi0_t} rfft(ring t)[m] for m < min(M, nphi/2+1), else 0.

    cuhpx/hpx_sht.py:37-55.  Leading dimensions of ``f`` are batch dimensions.
    """
    f = np.asarray(f, dtype=np.float64)
    R = nrings(nside)
    out = np.zeros(f.shape[:-1] + (R, mmax), dtype=np.complex128)
    ms = np.arange(mmax)
    for t in range(R):
        n = nphi_ring(t, nside)
        s = ring_start(t, nside)
        k = min(n // 2 + 1, mmax)
        fm = np.fft.rfft(f[..., s : s + n], axis=-1)
        out[..., t, :k] = fm[..., :k]
        out[..., t, :] *= _phase(ms, ring_phi0(t, nside), -1, phase_dtype)
    return out


def ring_irfft(ftm, mmax, nside, phase_dtype=np.complex128):
    """f[ring t] = irfft(ftm[t] e^{+i m phi0_t}, n=nphi, norm='forward').  cuhpx/hpx_sht.py:58-76.

    As torch.fft.irfft does, only m <= nphi/2 is used, the imaginary parts of
    the m=0 and Nyquist terms are dropped, and there is no 1/n factor.
    """
    ftm = np.asarray(ftm, dtype=np.complex128)
    R = nrings(nside)
    out = np.zeros(ftm.shape[:-2] + (npix(nside),), dtype=np.float64)
    ms = np.arange(ftm.shape[-1])
    for t in range(R):
        n = nphi_ring(t, nside)
        s = ring_start(t, nside)
        row = ftm[..., t, :] * _phase(ms, ring_phi0(t, nside), 1, phase_dtype)
        k = min(n // 2 + 1, row.shape[-1])
        spec = np.zeros(ftm.shape[:-2] + (n // 2 + 1,), dtype=np.complex128)
        spec[..., :k] = row[..., :k]
        out[..., s : s + n] = np.fft.irfft(spec, n=n, axis=-1) * n
    return out


# --------------------------------------------------------------------------- transforms
def default_lm(nside, lmax=None, mmax=None):
    """cuhpx/hpx_sht.py:654-655: lmax defaults to 4*nside-1, mmax to 2*nside+1."""
    return (lmax or 4 * nside - 1), (mmax or (4 * nside) // 2 + 1)


def sht(f, nside, lmax=None, mmax=None, quad_weights="ring", phase_dtype=np.complex128):
    """Forward real SHT: a[..., l, m] = sum_t w_t Pbar_l^m(theta_t) ftm[..., t, m].

    cuhpx/hpx_sht.py:214-236 in float64.  Output is dense [..., L, M] complex
    with zeros for m > l.
    """
    L, M = default_lm(nside, lmax, mmax)
    ftm = ring_rfft(f, M, nside, phase_dtype)
    w = ring_weights(nside, quad_weights)
    x = np.cos(ring_theta(nside))
    wf = ftm * w[:, None]  # [..., R, M]
    out = np.zeros(ftm.shape[:-2] + (L, M), dtype=np.complex128)
    for l, pl in legendre_by_l(M, L, x):  # pl [M, R]
        out[..., l, :] = np.einsum("...tm,mt->...m", wf, pl)
    return out


def isht(alm, nside, lmax=None, mmax=None, phase_dtype=np.complex128):
    """Inverse real SHT: f = irfft_rings( sum_l Pbar_l^m(theta_t) a[..., l, m] ).

    cuhpx/hpx_sht.py:268-283 in float64; ``alm`` is dense [..., L, M] complex.
    """
    alm = np.asarray(alm, dtype=np.complex128)
    L, M = alm.shape[-2], alm.shape[-1]
    x = np.cos(ring_theta(nside))
    ftm = np.zeros(alm.shape[:-2] + (x.size, M), dtype=np.complex128)
    for l, pl in legendre_by_l(M, L, x):
        ftm += np.einsum("...m,mt->...tm", alm[..., l, :], pl)
    return ring_irfft(ftm, M, nside, phase_dtype)


def sht_spot(f, nside, lmax, mmax, ms, quad_weights="ring", nodes="reference"):
    """Forward SHT restricted to the columns ``ms`` (returns [..., L, len(ms)]).

    Same algorithm as ``sht`` with one Legendre column at a time, so memory is
    O(lmax * rings) and it runs at nside 1024 on a few maps.

    ``nodes="reference"`` follows the reference exactly: Pbar at
    cos(arccos z_t), sin^2 = (1 + x)(1 - x), FP64 recurrence from the FP64
    diagonal (cuhpx/hpx_sht.py:192; cuhpx/sht_tools.py:204-214), including the
    subnormal diagonal of high orders near the poles that costs the
    reference up to ~1e-6 relative accuracy in orders near M/2 at nside 1024
    (see ``legendre_column_extended``).  ``nodes="exact"`` evaluates Pbar at
    the ring's z_t with sin^2 from ``ring_sin2`` by the same recurrence in
    extended precision: the accurate transform at the nodes the CUDA plan uses.
    """
    L, M = lmax, mmax
    ftm = ring_rfft(f, M, nside)
    w = ring_weights(nside, quad_weights)
    if nodes == "exact":
        x, s2 = ring_z(nside), ring_sin2(nside)
    else:
        x, s2 = np.cos(ring_theta(nside)), None
    out = np.zeros(ftm.shape[:-2] + (L, len(ms)), dtype=np.complex128)
    for j, m in enumerate(ms):
        P = legendre_column(m, L, x) if s2 is None else legendre_column_extended(m, L, x, s2)  # [L, R]
        out[..., :, j] = np.einsum("...t,lt->...l", ftm[..., :, m] * w, P)
    return out


def sht_by_m(f, nside, lmax, mmax, quad_weights="ring"):
    """``sht`` computed one order at a time (all columns of ``sht_spot``).

    Same values as ``sht`` (the Legendre columns come from the same
    recurrence); O(lmax * rings) Legendre memory and matrix products per
    order, so it finishes in seconds at nside 256, L = M = 511.
    """
    return sht_spot(f, nside, lmax, mmax, list(range(mmax)), quad_weights)


def isht_by_m(alm, nside):
    """``isht`` computed one order at a time (cuhpx/hpx_sht.py:268-283): the
    ring spectra of order m are the Legendre column of m applied to a[..., :, m]."""
    alm = np.asarray(alm, dtype=np.complex128)
    L, M = alm.shape[-2], alm.shape[-1]
    x = np.cos(ring_theta(nside))
    ftm = np.zeros(alm.shape[:-2] + (x.size, M), dtype=np.complex128)
    for m in range(min(M, L)):
        P = legendre_column(m, L, x)  # [L, R]
        ftm[..., :, m] = np.einsum("...l,lt->...t", alm[..., :, m], P)
    return ring_irfft(ftm, M, nside)


# --------------------------------------------------------------------------- CPU baseline timing
def time_reference_sample(nside, lmax, mmax, n_m=8, seed=0, threads=None):
    """Time the reference CPU algorithm on one map, sampling the Legendre stage.

    The reference's CPU SHT/iSHT (cuhpx/hpx_sht.py:214-236, 268-283) do, per
    call: per-ring rfft/irfft over all rings, and a dense einsum against the
    precomputed [M, L, rings] table (built at construction, not per call).  At
    nside=1024 that table is 68.6 GB, so this times the ring FFTs in full and
    the dense per-m contraction (table slice [L, rings] precomputed outside the
    timer, as the reference does) for ``n_m`` sampled orders, then scales the
    contraction time by M / n_m.  Returns dict(seconds_per_map, detail...).
    """
    import time

    if threads:
        try:
            import threadpoolctl

            threadpoolctl.threadpool_limits(threads)
        except Exception:
            pass
    L, M = lmax, mmax
    rng = np.random.default_rng(seed)
    f = rng.standard_normal(npix(nside))
    w = ring_weights(nside)
    x = np.cos(ring_theta(nside))
    t0 = time.perf_counter()
    ftm = ring_rfft(f, M, nside)
    t_rfft = time.perf_counter() - t0
    ms = np.unique(np.linspace(0, M - 1, n_m).astype(int))
    t_fwd = 0.0
    t_inv = 0.0
    for m in ms:
        P = legendre_column(int(m), L, x) * w[None, :]  # [L, R] slice of the weighted table
        Pi = legendre_column(int(m), L, x)
        fm = np.ascontiguousarray(ftm[:, m])
        t0 = time.perf_counter()
        a_re = P @ fm.real
        a_im = P @ fm.imag
        t_fwd += time.perf_counter() - t0
        av = a_re + 1j * a_im
        t0 = time.perf_counter()
        _ = Pi.T @ av.real
        _ = Pi.T @ av.imag
        t_inv += time.perf_counter() - t0
    scale = M / len(ms)
    t0 = time.perf_counter()
    ring_irfft(ftm, M, nside)
    t_irfft = time.perf_counter() - t0
    total = t_rfft + t_irfft + (t_fwd + t_inv) * scale
    return dict(
        seconds_per_map=total,
        t_rfft=t_rfft,
        t_irfft=t_irfft,
        t_contract_sampled=t_fwd + t_inv,
        n_m=len(ms),
        scale=scale,
    )
