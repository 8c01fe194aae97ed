"""CPU oracle for HEALPix pixel-order remapping -- TEST INFRASTRUCTURE ONLY.

Restates, in int64 numpy, the cuHPX reference's ``cuhpx_remap`` module: for
every source pixel it derives the HEALPix face coordinates (face, ix, iy), then
the destination pixel, and scatters ``out[..., dst] = in[..., src]``
(src/data_remapping/hpx_remapping_cuda.cu:137-146).  It is the checker, never
the product: only the test suite, ``__graft_entry__.smoke()`` and the CPU legs
of ``bench.py`` may import it.

Reference functions restated (paths relative to the cuHPX repository):
  ring2xyf          src/data_remapping/hpx_remapping_cuda.cu:161-223
  xyf2ring          src/data_remapping/hpx_remapping_cuda.cu:228-283
  nest2xyf          src/data_remapping/hpx_remapping_cuda.cu:285-305
  xyf2nest          src/data_remapping/hpx_remapping_cuda.cu:307-321
  _orient           correct_xy_orient, :100-134
  xyf2flat          :55-73;  flat2xyf :76-97;  flat2flat_pix :33-52
  _flip_k           the (flip, k) of every wrapper, :413-417 (and :448-450, ...)
  isqrt             d_isqrt, :376-388
  ring2nest ... flat2flat   the wrappers of hpx_remapping.cpp:21-239 and
                    cuhpx/hpx_remap.py:24-102 (origin letters S, E, N, W = 0..3)

Parity pin: the reference checks these functions only against healpy
(tests/test_data_remapping.py), which is not installed here.  The pin is
(a) the known answers of the HEALPix definition at nside 1 and 2, (b) the
NEST hierarchy measured against the ring geometry of ``oracle.hpx_oracle``
(itself pinned to the reference's golden vectors): every NEST pixel at
nside 2N lies nearest to the centre of its parent pixel at nside N, and
(c) consistency of the reference's direct flat->flat formula with the
composition of its flat->nest and nest->flat formulas
(tests/test_oracle_remap.py).  On a GPU, tests/test_remap_gpu.py also runs the
reference's own kernels (``oracle/build_ref_remap.py``) beside the library.
"""

import numpy as np

ORIGINS = {"S": 0, "E": 1, "N": 2, "W": 3}


def is_power_of_two(n):
    return n > 0 and (n & (n - 1)) == 0


def compute_order(nside):
    return int(nside).bit_length() - 1


def isqrt(v):
    """d_isqrt (:376-388): floor(sqrt(v)) with an integer correction."""
    v = np.asarray(v, dtype=np.int64)
    r = np.floor(np.sqrt(v.astype(np.float64) + 0.5)).astype(np.int64)
    r = np.where(r * r > v, r - 1, r)
    r = np.where((r + 1) * (r + 1) <= v, r + 1, r)
    return r


def _spread(v):
    v = np.asarray(v, dtype=np.int64)
    out = np.zeros_like(v)
    for b in range(16):
        out |= ((v >> b) & 1) << (2 * b)
    return out


def _compress(v):
    v = np.asarray(v, dtype=np.int64)
    out = np.zeros_like(v)
    for b in range(16):
        out |= ((v >> (2 * b)) & 1) << b
    return out


# ------------------------------------------------------------------ pixel <-> (x, y, face)
def ring2xyf(pix, nside):
    pix = np.asarray(pix, dtype=np.int64)
    n = np.int64(nside)
    order = compute_order(nside)
    npface = n * n
    ncap = (npface - n) << 1
    npx = 12 * npface
    north = pix < ncap
    equ = (~north) & (pix < npx - ncap)
    south = ~(north | equ)

    iring = np.zeros_like(pix)
    iphi = np.zeros_like(pix)
    kshift = np.zeros_like(pix)
    nr = np.zeros_like(pix)
    face = np.zeros_like(pix)

    p = pix[north]
    ir = (1 + isqrt(1 + 2 * p)) >> 1
    ip = (p + 1) - 2 * ir * (ir - 1)
    iring[north], iphi[north], nr[north] = ir, ip, ir
    face[north] = (ip - 1) // ir

    p = pix[equ] - ncap
    tmp = p >> (order + 2)
    ir = tmp + n
    ip = p - tmp * 4 * n + 1
    iring[equ], iphi[equ] = ir, ip
    kshift[equ] = (ir + n) & 1
    nr[equ] = n
    ire = tmp + 1
    irm = 2 * n + 1 - tmp
    ifm = (ip - (ire >> 1) + n - 1) >> order
    ifp = (ip - (irm >> 1) + n - 1) >> order
    face[equ] = np.where(ifp == ifm, ifp | 4, np.where(ifp < ifm, ifp, ifm + 8))

    p = npx - pix[south]
    ir = (1 + isqrt(2 * p - 1)) >> 1
    ip = 4 * ir + 1 - (p - 2 * ir * (ir - 1))
    nr[south] = ir
    iring[south] = 4 * n - ir
    iphi[south] = ip
    face[south] = (ip - 1) // ir + 8

    irt = iring - ((2 + (face >> 2)) * n) + 1
    ipt = ((face & 3) << 1) - ((face >> 2) & 1) + 1
    ipt = 2 * iphi - ipt * nr - kshift - 1
    ipt = np.where(ipt >= 2 * n, ipt - 8 * n, ipt)
    ix = (ipt - irt) >> 1
    iy = (-ipt - irt) >> 1
    return ix, iy, face


def xyf2ring(ix, iy, face, nside):
    ix = np.asarray(ix, dtype=np.int64)
    iy = np.asarray(iy, dtype=np.int64)
    face = np.asarray(face, dtype=np.int64)
    n = np.int64(nside)
    nl4 = 4 * n
    jr = ((face >> 2) + 2) * n - ix - iy - 1
    npface = n * n
    ncap = (npface - n) << 1
    npx = 12 * npface
    north = jr < n
    equ = (~north) & (jr < 3 * n)
    ring_nr = 4 * n - jr
    nr = np.where(north, 4 * jr, np.where(equ, 4 * n, 4 * ring_nr))
    n_before = np.where(north, 2 * jr * (jr - 1),
                        np.where(equ, ncap + (jr - n) * 4 * n, npx - 2 * ring_nr * (ring_nr + 1)))
    shifted = np.where(equ, ((jr - n) & 1) == 0, True)
    nr = nr >> 2
    kshift = 1 - shifted.astype(np.int64)
    jp = ((face & 3) << 1) - ((face >> 2) & 1) + 1
    num = jp * nr + ix - iy + 1 + kshift
    jp = np.sign(num) * (np.abs(num) // 2)  # C division of signed integers
    jp = np.where(jp < 1, jp + nl4, jp)
    return n_before + jp - 1


def nest2xyf(pix, nside):
    pix = np.asarray(pix, dtype=np.int64)
    order = compute_order(nside)
    face = pix >> (2 * order)
    p = pix & (nside * nside - 1)
    return _compress(p), _compress(p >> 1), face


def xyf2nest(ix, iy, face, nside):
    order = compute_order(nside)
    return (np.asarray(face, dtype=np.int64) << (2 * order)) + _spread(ix) + (_spread(iy) << 1)


def _orient(ix, iy, nside, flip, k):
    """correct_xy_orient (:100-134)."""
    ix = np.asarray(ix, dtype=np.int64)
    iy = np.asarray(iy, dtype=np.int64)
    if flip:
        ix, iy = iy, ix
    if k == 1:
        nx, ny = -iy - 1, ix
    elif k == 2:
        nx, ny = -ix - 1, -iy - 1
    elif k == 3:
        nx, ny = iy, -ix - 1
    else:
        nx, ny = ix, iy
    return nx & (nside - 1), ny & (nside - 1)


def _flip_k(src_origin, src_clockwise, dest_origin, dest_clockwise):
    flip = bool(src_clockwise) != bool(dest_clockwise)
    rotations = dest_origin - src_origin
    k = (-rotations if dest_clockwise else rotations) & 3
    return flip, k


def xyf2flat(ix, iy, face, nside, flip, k):
    order = compute_order(nside)
    ix, iy = _orient(ix, iy, nside, flip, k)
    return (np.asarray(face, dtype=np.int64) << (2 * order)) + (iy << order) + ix


def flat2xyf(pix, nside, flip, k):
    pix = np.asarray(pix, dtype=np.int64)
    order = compute_order(nside)
    face = pix >> (2 * order)
    iy = (pix >> order) & (nside - 1)
    ix = pix & (nside - 1)
    ix, iy = _orient(ix, iy, nside, flip, k)
    return ix, iy, face


def flat2flat_pix(pix, nside, flip, k):
    ix, iy, face = flat2xyf(pix, nside, flip, k)
    order = compute_order(nside)
    return (face << (2 * order)) + (iy << order) + ix


# ------------------------------------------------------------------ data movement
def _origin(o, what="The origin"):
    if o not in ORIGINS:
        raise RuntimeError(f"{what} must be one from S, E, N, W. Stop")
    return ORIGINS[o]


def _check(data, nside):
    if not is_power_of_two(nside):
        raise ValueError("nside must be a power of two")
    if data.shape[-1] != 12 * nside * nside:
        raise RuntimeError("The number of elements in the input array is not equal to the number of HEALPix grid "
                           "at current nside. Stop.")


def _scatter(data, dst):
    out = np.empty_like(data)
    out[..., dst] = data
    return out


def destination(kind, nside, *args):
    """Destination index of every source pixel for remap ``kind``."""
    pix = np.arange(12 * nside * nside, dtype=np.int64)
    if kind == "ring2nest":
        return xyf2nest(*ring2xyf(pix, nside), nside)
    if kind == "nest2ring":
        return xyf2ring(*nest2xyf(pix, nside), nside)
    if kind in ("nest2flat", "ring2flat"):
        o, cw = args
        flip, k = _flip_k(0, False, o, cw)
        xyf = nest2xyf(pix, nside) if kind == "nest2flat" else ring2xyf(pix, nside)
        return xyf2flat(*xyf, nside, flip, k)
    if kind in ("flat2nest", "flat2ring"):
        o, cw = args
        flip, k = _flip_k(o, cw, 0, False)
        xyf = flat2xyf(pix, nside, flip, k)
        return xyf2nest(*xyf, nside) if kind == "flat2nest" else xyf2ring(*xyf, nside)
    if kind == "flat2flat":
        so, scw, do, dcw = args
        flip, k = _flip_k(so, scw, do, dcw)
        return flat2flat_pix(pix, nside, flip, k)
    raise ValueError(kind)


def ring2nest(data, nside):
    _check(data, nside)
    return _scatter(data, destination("ring2nest", nside))


def nest2ring(data, nside):
    _check(data, nside)
    return _scatter(data, destination("nest2ring", nside))


def nest2flat(data, origin, clockwise, nside):
    _check(data, nside)
    return _scatter(data, destination("nest2flat", nside, _origin(origin), clockwise))


def flat2nest(data, origin, clockwise, nside):
    _check(data, nside)
    return _scatter(data, destination("flat2nest", nside, _origin(origin), clockwise))


def ring2flat(data, origin, clockwise, nside):
    _check(data, nside)
    return _scatter(data, destination("ring2flat", nside, _origin(origin), clockwise))


def flat2ring(data, origin, clockwise, nside):
    _check(data, nside)
    return _scatter(data, destination("flat2ring", nside, _origin(origin), clockwise))


def flat2flat(data, src_origin, src_clockwise, dest_origin, dest_clockwise, nside):
    _check(data, nside)
    so = _origin(src_origin, "The src origin")
    do = _origin(dest_origin, "The dest origin")
    return _scatter(data, destination("flat2flat", nside, so, src_clockwise, do, dest_clockwise))
