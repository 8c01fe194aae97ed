// Per-ring real DFT stages of the HEALPix SHT (sm_100a, SIMT + shared memory).
//
// Forward (replaces healpix_rfft_batch, src/harmonic_transform/hpx_fft.cpp:21-84,
// and healpix_rfft_torch, cuhpx/hpx_sht.py:37-55):
//   F_t[m] = e^{-i m phi0_t} sum_p f_p e^{-2 pi i m p / nphi_t},  m < min(M, nphi_t/2+1)
// Inverse (replaces healpix_irfft_batch, hpx_fft.cpp:86-149, and
// healpix_irfft_torch, hpx_sht.py:58-76):
//   f_p = Re X_0 + 2 sum_{0<m<nphi/2} Re(X_m e^{2 pi i m p/nphi}) + Re X_{nphi/2} (-1)^p,
//   X_m = e^{+i m phi0_t} F_t[m] for m < min(M, nphi/2+1), 0 above.
//
// Design (not the reference's): a real ring of length n = nphi is packed into
// a complex sequence of length h = n/2.  If h is a power of two it goes
// through a Stockham FFT in shared memory (one radix-2/4/8 pass, then radix-16
// passes, specialised per length), otherwise through Bluestein's chirp-z
// convolution with a per-ring size P >= 2h-1, a power of two or, where that is
// smaller (P = 3072), three times one: a twiddle-free radix-12 pass before the
// radix-16 passes (the reference pads every ring to 8*nside).  Small rings are transformed by sub-groups of a CTA
// (one warp, two, four or all eight) so that every thread handles ~16 points
// whatever the ring length.
//
// Phases are exact: the chirp e^{-i pi j^2/h} is tabulated per ring in the plan
// from the integer j^2 mod 2h in FP64, and the real-FFT split and phase-shift
// factors e^{-i pi q/n} (q <= 2n) and the FFT twiddles come from two-level
// tables built in FP64 once per plan and ring pair -- never from a float
// "pi*j*j/n" as in hpx_fft_cuda.cu:1090.
//
// Spectra are stored ring-major, F[map][foff_t + m] (m < mt_t), so every ring
// reads and writes contiguous memory; separate fold/unfold kernels (in
// hpx_kernels.cuh) transpose to and from the m-major layout of the Legendre
// stage.
#pragma once

#include "hpx_common.cuh"

namespace hpx {

struct RingPair {
    int nphi;       // pixels on both rings of the pair
    int h;          // nphi / 2
    int mt;         // min(M, nphi/2 + 1): orders kept on this ring
    int shift_n;    // phi0 = shift * pi / nphi for the north ring
    int shift_s;    // ... and for the south ring
    int logh;       // log2(h) when h is a power of two, else -1
    int logP;       // log2 of the FFT length actually run (h or the Bluestein size)
    int tpf;        // threads per FFT (32 .. 256)
    int has_south;  // 0 for the equator
    int rad3;       // Bluestein length 3 * 2^logP instead of 2^logP
    int64_t start_n;   // first pixel of the north ring
    int64_t start_s;   // first pixel of the south ring
    int64_t foff_n;    // spectrum offset of the north ring in F[map][.]
    int64_t foff_s;    // ... of the south ring
    int64_t gtab_off;  // offset of the chirp spectrum / chirp (complex elements), -1 if direct
    double z;          // cos(theta) of the north ring
    double w;          // quadrature weight of the ring
    double s2;         // sin^2(theta) of the north ring (no cancellation near the poles)
};

// Length of the FFT a ring runs: h (power-of-two rings), 2^logP or 3 * 2^logP (Bluestein)
__host__ __device__ __forceinline__ int ring_fft_len(const RingPair& rp) { return (rp.rad3 ? 3 : 1) << rp.logP; }
// ... for the ring kernels' kinds: 0 power-of-two rings, 1 Bluestein 2^logP, 2 Bluestein 3 * 2^logP
template <int KIND>
__device__ __forceinline__ int ring_fft_len_k(const RingPair& rp) { return (KIND == 2 ? 3 : 1) << rp.logP; }

// FFT work buffers are padded by one element every 16 so that the strided
// Stockham stores of the first pass (stride 16 complex) spread over all banks;
// their length is even, so that consecutive buffers stay 16-byte aligned.
__device__ __forceinline__ int padi(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int P) { return (P + (P >> 4) + 2) & ~1; }

// ----------------------------------------------------------------- sync helpers
// Threads [g*tpf, (g+1)*tpf) of the CTA form FFT group g.
__device__ __forceinline__ void group_sync(int tpf, int g) {
    if (tpf >= (int)blockDim.x) {
        __syncthreads();
    } else if (tpf == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;\n" ::"r"(1 + g), "r"(tpf) : "memory");
    }
}

// 4-point DFT in registers (forward: e^-, inverse: e^+)
template <typename T, bool INV>
__device__ __forceinline__ void dft4(cplx<T>& v0, cplx<T>& v1, cplx<T>& v2, cplx<T>& v3) {
    const cplx<T> t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3);
    const cplx<T> d = csub(v1, v3);
    const cplx<T> t3 = INV ? cplx<T>{-d.im, d.re} : cplx<T>{d.im, -d.re};  // +/- i d
    v0 = cadd(t0, t2);
    v1 = cadd(t1, t3);
    v2 = csub(t0, t2);
    v3 = csub(t1, t3);
}

// 16-point DFT in registers as 4 x 4 with the internal factors W16^(b c).
template <typename T, bool INV>
__device__ __forceinline__ void dft16(cplx<T>* v) {
    // columns: v[b + 4a], a = 0..3
#pragma unroll
    for (int b = 0; b < 4; ++b) dft4<T, INV>(v[b], v[b + 4], v[b + 8], v[b + 12]);
    // now v[b + 4c] = Y[b][c]; multiply by W16^(b c)
    const T r = (T)0.70710678118654752440;  // cos(pi/4)
    const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173;  // cos/sin(pi/8)
    const T sg = INV ? (T)1 : (T)-1;
    // W16^k = cos(2 pi k/16) + sg*i sin(2 pi k/16)
    const cplx<T> w1 = {c1, sg * s1}, w2 = {r, sg * r}, w3 = {s1, sg * c1}, w4 = {(T)0, sg},
                  w6 = {-r, sg * r}, w9 = {-c1, -sg * s1};
    v[1 + 4 * 1] = cmul(v[5], w1);
    v[1 + 4 * 2] = cmul(v[9], w2);
    v[1 + 4 * 3] = cmul(v[13], w3);
    v[2 + 4 * 1] = cmul(v[6], w2);
    v[2 + 4 * 2] = cmul(v[10], w4);
    v[2 + 4 * 3] = cmul(v[14], w6);
    v[3 + 4 * 1] = cmul(v[7], w3);
    v[3 + 4 * 2] = cmul(v[11], w6);
    v[3 + 4 * 3] = cmul(v[15], w9);
    // rows: for each c, DFT over b -> X[c + 4d]
#pragma unroll
    for (int c = 0; c < 4; ++c) dft4<T, INV>(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
    // v[4c + d] = X[c + 4d]; reorder to natural order
    cplx<T> o[16];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 4; ++d) o[c + 4 * d] = v[4 * c + d];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = o[i];
}

// 8-point DFT in registers: two 4-point DFTs of the even and odd samples and
// the factors W8^k.
template <typename T, bool INV>
__device__ __forceinline__ void dft8(cplx<T>* v) {
    cplx<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cplx<T> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<T, INV>(e0, e1, e2, e3);
    dft4<T, INV>(o0, o1, o2, o3);
    const T r = (T)0.70710678118654752440;
    const T sg = INV ? (T)1 : (T)-1;
    o1 = cmul(o1, cplx<T>{r, sg * r});
    o2 = cplx<T>{-sg * o2.im, sg * o2.re};  // times (0, sg)
    o3 = cmul(o3, cplx<T>{-r, sg * r});
    v[0] = cadd(e0, o0);
    v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1);
    v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2);
    v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3);
    v[7] = csub(e3, o3);
}

// 3-point DFT in registers: X0 = a + (b + c), X1,2 = a - (b + c)/2 -/+ i s (b - c)
// (forward, s = sin(2 pi/3); the inverse swaps X1 and X2)
template <typename T, bool INV>
__device__ __forceinline__ void dft3(cplx<T>* v) {
    const T s = (T)0.86602540378443864676;
    const cplx<T> t1 = cadd(v[1], v[2]);
    const cplx<T> d = cscale(csub(v[1], v[2]), s);
    const cplx<T> m = {v[0].re - (T)0.5 * t1.re, v[0].im - (T)0.5 * t1.im};
    v[0] = cadd(v[0], t1);
    const cplx<T> mi = {m.re + d.im, m.im - d.re};  // m - i d
    const cplx<T> pi = {m.re - d.im, m.im + d.re};  // m + i d
    v[1] = INV ? pi : mi;
    v[2] = INV ? mi : pi;
}

// 6- and 12-point DFTs in registers as 3 x N2 (N2 = 2, 4) by the prime-factor
// (Good-Thomas) mapping, which needs no twiddles between the two stages: with
// n = (N2 n1 + 3 n2) mod N, X[k] = sum_n1 W3^{n1 k} sum_n2 W_N2^{n2 k} x[n], and
// W3^{n1 k}, W_N2^{n2 k} depend on k only through k mod 3 and k mod N2.
template <typename T, bool INV, int N2>
__device__ __forceinline__ void dft3xN2(cplx<T>* v) {
    constexpr int N = 3 * N2;
    cplx<T> y[3][N2];
#pragma unroll
    for (int n1 = 0; n1 < 3; ++n1) {
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) y[n1][n2] = v[(N2 * n1 + 3 * n2) % N];
        if constexpr (N2 == 2) {
            const cplx<T> a = y[n1][0], b = y[n1][1];
            y[n1][0] = cadd(a, b);
            y[n1][1] = csub(a, b);
        } else {
            dft4<T, INV>(y[n1][0], y[n1][1], y[n1][2], y[n1][3]);
        }
    }
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) {
        cplx<T> t[3] = {y[0][k2], y[1][k2], y[2][k2]};
        dft3<T, INV>(t);
        y[0][k2] = t[0];
        y[1][k2] = t[1];
        y[2][k2] = t[2];
    }
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = y[k % 3][k % N2];
}

template <typename T, bool INV, int R>
__device__ __forceinline__ void dftR(cplx<T>* v) {
    if constexpr (R == 3) {
        dft3<T, INV>(v);
    } else if constexpr (R == 6) {
        dft3xN2<T, INV, 2>(v);
    } else if constexpr (R == 12) {
        dft3xN2<T, INV, 4>(v);
    } else if constexpr (R == 2) {
        const cplx<T> a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        dft4<T, INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        dft8<T, INV>(v);
    } else {
        dft16<T, INV>(v);
    }
}

// W^r for r = 1 .. R-1 from W (one table load per butterfly): W^2, W^4, W^8 by
// squaring, every other power as the product of two of these or of W, so each
// carries at most a few roundings.
template <typename T, int R>
__device__ __forceinline__ void twiddle_powers(cplx<T> w1, cplx<T>* w) {
    w[1] = w1;
    if constexpr (R > 2) w[2] = cmul(w1, w1);
    if constexpr (R > 3) w[3] = cmul(w[2], w1);
    if constexpr (R > 4) {
        w[4] = cmul(w[2], w[2]);
        w[5] = cmul(w[4], w1);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
    }
    if constexpr (R > 8) {
        w[8] = cmul(w[4], w[4]);
#pragma unroll
        for (int r = 9; r < 16; ++r) w[r] = cmul(w[8], w[r - 8]);
    }
}

// e^{-i pi q / n} for 0 <= q < 2n from small tables, q = 64 a + b:
// e^{-i pi 64 a/n} = hi[a] + hc[a] (float + float: hc is the rounding error of
// hi) and lo[b] = e^{-i pi b/n} - 1 (|lo| < 0.1 for n >= 2048), so that
// hi + (hc + hi lo) rounds once, at the end, like a correctly rounded table
// entry.  That matters for FFT twiddles, whose powers W^r multiply the error of
// W by r.  The ring kernels keep two: the phases of the real-FFT split and
// ring shift (n = nphi) and the FFT twiddles e^{-2 pi i q/P} (n = P/2), about
// 1.5 KB instead of a P/2-entry twiddle table.
template <typename T>
struct PhaseTab {
    const cplx<T>* lo;  // 64 entries
    const cplx<T>* hi;  // phase_tab_nhi(n) entries, followed by as many hc entries
    int nhi;
    __device__ __forceinline__ cplx<T> operator()(int q) const {
        const cplx<T> a = hi[q >> 6], c = hi[nhi + (q >> 6)], d = lo[q & 63];
        return {a.re + fma(a.re, d.re, fma(-a.im, d.im, c.re)), a.im + fma(a.re, d.im, fma(a.im, d.re, c.im))};
    }
};

HPX_HD constexpr int phase_tab_nhi(int n) { return (2 * n + 63) / 64; }
// complex entries of the tables for n
HPX_HD constexpr int phase_tab_elems(int n) { return 64 + 2 * phase_tab_nhi(n); }

template <typename T>
__device__ PhaseTab<T> build_phase_tab(cplx<T>* lo, int n) {
    const int nhi = phase_tab_nhi(n);
    cplx<T>* hi = lo + 64;
    for (int i = threadIdx.x; i < 64 + nhi; i += blockDim.x) {
        const int q = i < 64 ? i : 64 * (i - 64);
        double s, c;
        sincospi(-(double)q / (double)n, &s, &c);
        if (i < 64) {
            const double sh = sinpi((double)q / (double)(2 * n));
            lo[i] = {(T)(-2.0 * sh * sh), (T)s};  // cos - 1 = -2 sin^2(theta/2)
        } else {
            const cplx<T> v = {(T)c, (T)s};
            hi[i - 64] = v;
            hi[nhi + i - 64] = {(T)(c - (double)v.re), (T)(s - (double)v.im)};
        }
    }
    return PhaseTab<T>{lo, hi, nhi};
}

// twiddles e^{-2 pi i q/P} read from a full padded table tw[padi(q)], q < P/2
template <typename T>
struct FullTw {
    const cplx<T>* p;
    __device__ __forceinline__ cplx<T> operator()(int q) const { return p[padi(q)]; }
};

// One Stockham pass of radix R over a length-P sequence whose first Ns-point
// sub-transforms are done: inputs src[j + rQ] (Q = P/R), outputs dst[o + r Ns]
// with o = (j mod Ns) + R (j - j mod Ns).  Twiddles e^{-/+2 pi i r k/(Ns R)}:
// one lookup tw(k step) = e^{-2 pi i k step/P} (step = P/(Ns R)) and its powers
// by twiddle_powers.  The first pass maps its inputs through pre(i, v)
// (natural index i), the last pass its outputs through post(i, v).
template <typename T, bool INV, int R, bool FIRST, bool LAST, typename TW, typename Pre, typename Post>
__device__ __forceinline__ void fft_pass(const cplx<T>* src, cplx<T>* dst, int P, int Ns, const TW& tw, int lt,
                                         int tpf, Pre& pre, Post& post) {
    const int Q = P / R;
    const int step = P / (Ns * R);
    for (int j = lt; j < Q; j += tpf) {
        const int k = j & (Ns - 1);
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            v[r] = src[padi(j + r * Q)];
            if constexpr (FIRST) v[r] = pre(j + r * Q, v[r]);
        }
        if (Ns > 1) {
            cplx<T> w1 = tw(k * step);
            if (INV) w1.im = -w1.im;
            cplx<T> w[R];
            twiddle_powers<T, R>(w1, w);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
        }
        dftR<T, INV, R>(v);
        const int o = ((j - k) * R) + k;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            cplx<T> x = v[r];
            if constexpr (LAST) x = post(o + r * Ns, x);
            dst[padi(o + r * Ns)] = x;
        }
    }
}

struct IdentityMap {
    template <typename V>
    __device__ __forceinline__ V operator()(int, V v) const { return v; }
};

// Stockham autosort FFT of length P = 2^logP (logP >= 1) on src (natural
// order, padded indexing); returns the buffer (src or dst) holding the
// natural-order result.  One radix-2/4/8 pass for logP mod 4, then radix-16
// passes: 3 passes for P = 4096.  tw(q) = e^{-2 pi i q/P}, q < P/2.
// INV: e^{+2 pi i jk/P} (unnormalised).  pre/post as in fft_pass.
template <typename T, bool INV, typename TW, typename Pre, typename Post>
__device__ cplx<T>* fft_pow2(cplx<T>* src, cplx<T>* dst, int logP, const TW& tw, int lt, int tpf, int g, Pre pre,
                             Post post) {
    const int P = 1 << logP;
    const int n16 = logP >> 2, r0 = logP & 3;
    const int npass = n16 + (r0 ? 1 : 0);
    int Ns = 1, pass = 0;
    auto next = [&]() {
        group_sync(tpf, g);
        cplx<T>* t = src;
        src = dst;
        dst = t;
        ++pass;
    };
    if (r0) {
        const bool last = npass == 1;
        if (r0 == 1) {
            if (last) fft_pass<T, INV, 2, true, true>(src, dst, P, Ns, tw, lt, tpf, pre, post);
            else fft_pass<T, INV, 2, true, false>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        } else if (r0 == 2) {
            if (last) fft_pass<T, INV, 4, true, true>(src, dst, P, Ns, tw, lt, tpf, pre, post);
            else fft_pass<T, INV, 4, true, false>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        } else {
            if (last) fft_pass<T, INV, 8, true, true>(src, dst, P, Ns, tw, lt, tpf, pre, post);
            else fft_pass<T, INV, 8, true, false>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        }
        Ns <<= r0;
        next();
    }
    for (int i = 0; i < n16; ++i) {
        const bool first = pass == 0, last = pass == npass - 1;
        if (first && last) fft_pass<T, INV, 16, true, true>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        else if (first) fft_pass<T, INV, 16, true, false>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        else if (last) fft_pass<T, INV, 16, false, true>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        else fft_pass<T, INV, 16, false, false>(src, dst, P, Ns, tw, lt, tpf, pre, post);
        Ns <<= 4;
        next();
    }
    return src;
}

// ---------------------------------------------------------------- size-specialised FFT
// The ring kernels run one group of fft_tpf(P) threads per transform, so for
// every length the whole pass sequence can be instantiated with P, the pass
// strides and the group size as compile-time constants: the padded indices
// and twiddle indices then fold into immediate offsets and shifts instead of
// the integer arithmetic of the generic passes.
HPX_HD constexpr int fft_tpf(int P) { return P / 16 < 32 ? 32 : (P / 16 > 256 ? 256 : P / 16); }
HPX_HD constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

// Padding by one element every D: padi is D = 16.  (The pass after the first
// radix-6/12 pass of the lengths 3 * 2^K reads a buffer padded every 48, which
// keeps that first pass's stride-R stores and the next pass's loads free of
// bank conflicts; padded_len(P) covers it.)
template <int D>
__device__ __forceinline__ int padd(int i) { return i + i / D; }
// padded index of i + r * S when the stride S is a multiple of D (then the
// padding of i + rS is the padding of i plus r S/D)
template <int S, int D = 16>
__device__ __forceinline__ int padi_step(int pi, int i, int r) {
    if constexpr (S % D == 0) return pi + r * (S + S / D);
    else return padd<D>(i + r * S);
}

// ZIN: the input is zero from P/2 on (the first pass then skips the inputs
// r >= R/2 of its R, which lie at or above P/2); HOUT: only outputs below P/2
// are wanted (the last pass forms and stores only those).  Bluestein's convolution has both.
// UNPAD: the last pass stores in natural, unpadded order (its stores are
// consecutive across a warp, so the padding buys nothing there) -- the inverse
// ring transform then copies its result out with 16-byte accesses.  UNPIN:
// likewise the first pass reads an unpadded input (the ring loads then move 16
// bytes per copy).  DI, DO: the padding of the input and output buffers.
template <typename T, bool INV, int R, int NS, int P, int TPF, bool FIRST, bool LAST, bool ZIN, bool HOUT, bool UNPAD,
          bool UNPIN, int DI = 16, int DO = 16, typename TW, typename Pre, typename Post>
__device__ __forceinline__ void fft_pass_ct(const cplx<T>* src, cplx<T>* dst, const TW& tw, int lt, Pre& pre,
                                            Post& post) {
    constexpr int Q = P / R;
    constexpr int LSTEP = ilog2c(P / (NS * R));
    // the twiddle step P / (NS R) is a power of two (lengths 2^K and 3 * 2^K, radix 3 first)
    static_assert(NS == 1 || (NS * R) << LSTEP == P, "twiddle step must be a power of two");
#pragma unroll
    for (int j0 = 0; j0 < Q; j0 += TPF) {
        const int j = j0 + lt;
        if (Q % TPF != 0 && j >= Q) break;
        const int k = (NS & (NS - 1)) == 0 ? (j & (NS - 1)) : (j % NS);
        const int pj = padd<DI>(j);
        cplx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (FIRST && ZIN && 2 * r >= R) {
                v[r] = {(T)0, (T)0};  // j + r Q >= P/2
                continue;
            }
            if constexpr (FIRST && UNPIN)
                v[r] = src[j + r * Q];
            else
                v[r] = src[padi_step<Q, DI>(pj, j, r)];
            if constexpr (FIRST) v[r] = pre(j + r * Q, v[r]);
        }
        if constexpr (NS > 1) {
            cplx<T> w1 = tw(k << LSTEP);
            if (INV) w1.im = -w1.im;
            cplx<T> w[R];
            twiddle_powers<T, R>(w1, w);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
        }
        dftR<T, INV, R>(v);
        const int o = ((j - k) * R) + k;
        const int po = padd<DO>(o);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (LAST && HOUT && 2 * r >= R) continue;  // o + r NS >= P/2
            cplx<T> x = v[r];
            if constexpr (LAST) x = post(o + r * NS, x);
            if constexpr (LAST && UNPAD)
                dst[o + r * NS] = x;
            else
                dst[padi_step<NS, DO>(po, o, r)] = x;
        }
    }
}

// radix-16 passes NS, 16 NS, ... until the length is P
template <typename T, bool INV, int P, int TPF, int NS, bool FIRST, bool ZIN, bool HOUT, bool UNPAD, bool UNPIN,
          int DI = 16, typename TW, typename Pre, typename Post>
__device__ __forceinline__ cplx<T>* fft_r16_ct(cplx<T>* src, cplx<T>* dst, const TW& tw, int lt, int g, Pre& pre,
                                               Post& post) {
    if constexpr (NS >= P) {
        return src;
    } else {
        constexpr bool LAST = NS * 16 == P;
        fft_pass_ct<T, INV, 16, NS, P, TPF, FIRST, LAST, ZIN, HOUT, UNPAD, UNPIN, DI>(src, dst, tw, lt, pre, post);
        group_sync(TPF, g);
        return fft_r16_ct<T, INV, P, TPF, NS * 16, false, ZIN, HOUT, UNPAD, UNPIN>(dst, src, tw, lt, g, pre, post);
    }
}

template <typename T, bool INV, int LOGP, bool ZIN, bool HOUT, bool UNPAD, bool UNPIN, typename TW, typename Pre,
          typename Post>
__device__ __forceinline__ cplx<T>* fft_ct(cplx<T>* src, cplx<T>* dst, const TW& tw, int lt, int g, Pre& pre,
                                           Post& post) {
    constexpr int P = 1 << LOGP, TPF = fft_tpf(P), R0 = 1 << (LOGP & 3);
    if constexpr (R0 > 1) {
        constexpr bool LAST = R0 == P;
        fft_pass_ct<T, INV, R0, 1, P, TPF, true, LAST, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, pre, post);
        group_sync(TPF, g);
        return fft_r16_ct<T, INV, P, TPF, R0, false, ZIN, HOUT, UNPAD, UNPIN>(dst, src, tw, lt, g, pre, post);
    } else {
        return fft_r16_ct<T, INV, P, TPF, 1, true, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
    }
}

// Length P = 3 * 2^K: one twiddle-free pass of radix 3 * 2^(K mod 4), then
// radix-16 passes (6, 16, 16 for P = 1536; 12, 16, 16 for P = 3072): as many
// passes through shared memory as 2048 and 4096 take, over 25% fewer points.
// The group is fft_tpf(P) = P / 16 threads, which named barriers need to be
// whole warps.
template <typename T, bool INV, int K, bool ZIN, bool HOUT, bool UNPAD, bool UNPIN, typename TW, typename Pre,
          typename Post>
__device__ __forceinline__ cplx<T>* fft_ct3(cplx<T>* src, cplx<T>* dst, const TW& tw, int lt, int g, Pre& pre,
                                            Post& post) {
    constexpr int P = 3 << K, TPF = fft_tpf(P), R3 = 3 << (K & 3);
    static_assert(TPF % 32 == 0, "an FFT group must be whole warps");
    static_assert(R3 == 6 || R3 == 12, "first-pass radix");
    constexpr int D3 = 48;
    static_assert((P / 16) % D3 == 0, "the second pass's input stride is a multiple of D3");
    static_assert(P + P / D3 < padded_len(P), "the buffers hold the padding every D3");
    fft_pass_ct<T, INV, R3, 1, P, TPF, true, false, ZIN, HOUT, UNPAD, UNPIN, 16, D3>(src, dst, tw, lt, pre, post);
    group_sync(TPF, g);
    return fft_r16_ct<T, INV, P, TPF, R3, false, ZIN, HOUT, UNPAD, UNPIN, D3>(dst, src, tw, lt, g, pre, post);
}
// passes of fft_ct3 (the result is in src when even)
HPX_HD constexpr int fft3_passes(int K) { return 1 + K / 4; }
// the length 3 * 2^K the ring kernels run: 3072 (group size 192 threads); a
// second length would double the kernel's FFT code and its registers
constexpr int kRad3MinK = 10, kRad3MaxK = 10;

// The ring kernels' FFT: the specialised pass sequence for the group size
// fft_tpf(P) these kernels use (the generic fft_pow2 otherwise).  ZIN / HOUT
// as for fft_pass_ct (the generic passes ignore them: they transform and store
// everything, which is also correct).
// (tw, pre and post by value: this function may not be inlined, and a
// reference would make every twiddle lookup reload the table's pointers from
// the stack)
template <typename T, bool INV, bool ZIN = false, bool HOUT = false, bool UNPAD = false, bool UNPIN = false, typename TW,
          typename Pre, typename Post>
__device__ __forceinline__ cplx<T>* fft_ring(cplx<T>* src, cplx<T>* dst, int logP, const TW tw, int lt, int tpf, int g,
                                             Pre pre, Post post) {
    if (tpf == fft_tpf(1 << logP)) {
        switch (logP) {
            case 1: return fft_ct<T, INV, 1, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 2: return fft_ct<T, INV, 2, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 3: return fft_ct<T, INV, 3, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 4: return fft_ct<T, INV, 4, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 5: return fft_ct<T, INV, 5, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 6: return fft_ct<T, INV, 6, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 7: return fft_ct<T, INV, 7, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 8: return fft_ct<T, INV, 8, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 9: return fft_ct<T, INV, 9, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 10: return fft_ct<T, INV, 10, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 11: return fft_ct<T, INV, 11, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 12: return fft_ct<T, INV, 12, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            case 13: return fft_ct<T, INV, 13, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
            default: break;
        }
    }
    // generic passes (padded input and output); UNPIN: the input is first
    // copied into the other buffer padded; UNPAD: the result is copied into the
    // other buffer unpadded
    if constexpr (UNPIN) {
        for (int j = lt; j < (1 << logP); j += tpf) dst[padi(j)] = src[j];
        group_sync(tpf, g);
        cplx<T>* t = src;
        src = dst;
        dst = t;
    }
    cplx<T>* r = fft_pow2<T, INV>(src, dst, logP, tw, lt, tpf, g, pre, post);
    if constexpr (UNPAD) {
        cplx<T>* o = (r == src) ? dst : src;
        for (int j = lt; j < (1 << logP); j += tpf) o[j] = r[padi(j)];
        group_sync(tpf, g);
        return o;
    }
    return r;
}

// fft_ring for the length 3 * 2^K, K = kRad3MinK = kRad3MaxK, with the group
// size fft_tpf(3 << K)
template <typename T, bool INV, bool ZIN = false, bool HOUT = false, bool UNPAD = false, bool UNPIN = false,
          typename TW, typename Pre, typename Post>
__device__ __forceinline__ cplx<T>* fft_ring3(cplx<T>* src, cplx<T>* dst, int K, const TW tw, int lt, int g, Pre pre,
                                              Post post) {
    static_assert(kRad3MinK == kRad3MaxK, "one instantiated length");
    (void)K;
    return fft_ct3<T, INV, kRad3MinK, ZIN, HOUT, UNPAD, UNPIN>(src, dst, tw, lt, g, pre, post);
}

// twP[padi(q)] = e^{-2 pi i q / P}, q < P/2, from the plan's table for Pmax
// (all threads of the CTA); the table takes padded_len(P/2) entries
template <typename T>
__device__ void load_twiddles(cplx<T>* twP, int logP, const cplx<T>* __restrict__ tw, int logPmax) {
    const int half = 1 << (logP - 1);
    const int stride = 1 << (logPmax - logP);
    for (int q = threadIdx.x; q < half; q += blockDim.x) twP[padi(q)] = tw[q * stride];
}

// Complex DFT of length h of buf (natural order, h entries written by this
// group), forward (e^-) or inverse (e^+); returns the buffer with Z in natural order.
// KIND: 0 power-of-two ring, 1 Bluestein of length 2^logP, 2 of length 3 * 2^logP.
template <int KIND, typename T, typename TW>
__device__ cplx<T>* ring_dft(cplx<T>* buf, cplx<T>* buf2, const RingPair& rp, const TW tw, const cplx<T>* __restrict__ G,
                             const cplx<T>* __restrict__ chirp, bool inv, int lt, int tpf, int g) {
    group_sync(tpf, g);
    IdentityMap id;
    if constexpr (KIND == 0) {
        // power-of-two ring
        // (the inverse transform's result in natural unpadded order)
        if (rp.logh == 0) return buf;
        return inv ? fft_ring<T, true, false, false, true, true>(buf, buf2, rp.logh, tw, lt, tpf, g, id, id)
                   : fft_ring<T, false, false, false, false, true>(buf, buf2, rp.logh, tw, lt, tpf, g, id, id);
    } else {
        // Bluestein, c_j = e^{-i pi j^2/h}: Z_k = c_k sum_j (z_j c_j) conj(c_{k-j}), the
        // convolution done as IFFT(FFT(z c) G) with G the plan's FFT of conj(c)
        // (scaled by 1/P); the inverse transform is conj(DFT(conj z)).  The chirp
        // products ride on the first loads and the last stores of the two FFTs.
        // chirp[0..h) and G[0..P/2] are the ring's tables in shared memory (G is
        // symmetric, G_k = G_{P-k}).
        const int h = rp.h, P = ring_fft_len_k<KIND>(rp);
        // captures by value: the passes may run in a called (not inlined) function,
        // where a captured reference would be a load from the stack per element
        auto pre = [h, inv, chirp](int j, cplx<T> a) {
            if (j >= h) return cplx<T>{(T)0, (T)0};
            if (inv) a.im = -a.im;
            return cmul(a, chirp[j]);
        };
        auto mulG = [G, P](int k, cplx<T> a) { return cmul(a, G[2 * k <= P ? k : P - k]); };
        auto postc = [h, inv, chirp](int k, cplx<T> a) {
            if (k >= h) return a;
            cplx<T> v = cmul(a, chirp[k]);
            if (inv) v.im = -v.im;
            return v;
        };
        // a_j = z_j c_j is zero from j = h <= P/2 on, and only Z_k, k < h, is wanted
        if constexpr (KIND == 2) {
            cplx<T>* r = fft_ring3<T, false, true, false, false, true>(buf, buf2, rp.logP, tw, lt, g, pre, mulG);
            cplx<T>* o = (r == buf) ? buf2 : buf;
            return inv ? fft_ring3<T, true, false, true, true>(r, o, rp.logP, tw, lt, g, id, postc)
                       : fft_ring3<T, true, false, true, false>(r, o, rp.logP, tw, lt, g, id, postc);
        } else {
            cplx<T>* r = fft_ring<T, false, true, false, false, true>(buf, buf2, rp.logP, tw, lt, tpf, g, pre, mulG);
            cplx<T>* o = (r == buf) ? buf2 : buf;
            // (the inverse transform's result in natural unpadded order)
            return inv ? fft_ring<T, true, false, true, true>(r, o, rp.logP, tw, lt, tpf, g, id, postc)
                       : fft_ring<T, true, false, true, false>(r, o, rp.logP, tw, lt, tpf, g, id, postc);
        }
    }
}

// One complex element (8 or 16 bytes) global -> shared, asynchronously.
template <typename T>
__device__ __forceinline__ void cp_async_cplx(cplx<T>* dst, const cplx<T>* src) {
    if constexpr (sizeof(T) == 4) cp_async8(dst, src);
    else cp_async16(dst, src);
}

// The group starts copying ring x[0..n) (h complex) into dst[0..h) (unpadded:
// the first FFT pass reads it with consecutive addresses), two complex values
// per 16-byte copy when both ends allow; the copy is one cp.async commit group
// of the calling threads.
template <typename T>
__device__ __forceinline__ void ring_load_async(cplx<T>* dst, const T* x, int h, int lt, int tpf) {
    bool vec = false;
    if constexpr (sizeof(T) == 4) vec = (h & 1) == 0 && ((((uintptr_t)x) | ((uintptr_t)dst)) & 15) == 0;
    if (vec) {
        for (int j = lt; 2 * j < h; j += tpf) cp_async16(dst + 2 * j, x + 4 * j);
    } else {
        for (int j = lt; j < h; j += tpf) cp_async_cplx(dst + j, (const cplx<T>*)x + j);
    }
    cp_async_commit();
}

// ... and the spectrum Fg[0..mt) into dst[0..mt) (contiguous).
template <typename T>
__device__ __forceinline__ void spec_load_async(cplx<T>* dst, const cplx<T>* Fg, int mt, int lt, int tpf) {
    bool vec = false;
    if constexpr (sizeof(T) == 4) vec = ((((uintptr_t)Fg) | ((uintptr_t)dst)) & 15) == 0;
    if (vec) {
        // two complex values per 16-byte copy (spectra start at even offsets)
        for (int k = lt; 2 * k + 1 < mt; k += tpf) cp_async16(dst + 2 * k, Fg + 2 * k);
        if ((mt & 1) && lt == 0) cp_async_cplx(dst + mt - 1, Fg + mt - 1);
    } else {
        for (int k = lt; k < mt; k += tpf) cp_async_cplx(dst + k, Fg + k);
    }
    cp_async_commit();
}

// Forward transform of one real ring into F[0..mt) (global, contiguous).  The
// ring was loaded into cur[j] by ring_load_async; the two FFT buffers
// alternate roles from map to map: once the DFT is done, the buffer it left
// free receives the next map's ring (load_next, asynchronous) while this map's
// spectrum is formed and stored.  On return cur holds the next input.
// Returns the largest |re|, |im| this thread wrote.
template <int KIND, typename T, typename Next>
__device__ T ring_forward(cplx<T>*& cur, cplx<T>*& other, int shift, T* __restrict__ F, const RingPair& rp,
                          const PhaseTab<T>& tw, const cplx<T>* __restrict__ gtab,
                          const cplx<T>* __restrict__ chirp, const PhaseTab<T>& E, int lt, int tpf, int g,
                          Next load_next) {
    const int h = rp.h;
    cp_async_wait<0>();
    cplx<T>* Z = ring_dft<KIND>(cur, other, rp, tw, gtab, chirp, false, lt, tpf, g);  // starts with a group sync
    cplx<T>* freeb = (Z == cur) ? other : cur;
    load_next(freeb);
    T mx = (T)0;
    // Outputs k and h-k share Z_k, Z_{h-k} and the twiddle W = e^{-2 pi i k/n}:
    // X_k = E_k + W O_k and X_{h-k} = conj(E_k - W O_k); the ring phase of h-k
    // is e^{-i pi (h-k)/n} = -i conj(e^{-i pi k/n}).
    const int mt = rp.mt;
    for (int k = lt; 2 * k <= h; k += tpf) {
        const int kb = h - k;
        const cplx<T> Zk = Z[padi(k)];
        const cplx<T> Zc = cconj(Z[padi(k == 0 ? 0 : kb)]);
        const cplx<T> Ek = cscale(cadd(Zk, Zc), (T)0.5);
        const cplx<T> d = cscale(csub(Zk, Zc), (T)0.5);
        const cplx<T> WO = cmul(E(2 * k), cplx<T>{d.im, -d.re});  // W (-i d)
        cplx<T> Xa = cadd(Ek, WO);
        cplx<T> Xb = cconj(csub(Ek, WO));
        if (shift) {
            const cplx<T> e = E(k);
            Xa = cmul(e, Xa);
            Xb = cmul(cplx<T>{-e.im, -e.re}, Xb);
        }
        if (k < mt) {
            *(cplx<T>*)(F + 2 * k) = Xa;
            mx = fmax(mx, fmax(fabs(Xa.re), fabs(Xa.im)));
        }
        if (kb != k && kb < mt) {
            *(cplx<T>*)(F + 2 * kb) = Xb;
            mx = fmax(mx, fmax(fabs(Xb.re), fabs(Xb.im)));
        }
    }
    group_sync(tpf, g);
    cur = freeb;
    other = Z;
    return mx;
}

// Inverse transform of one ring spectrum into the real ring x[0..n).  The
// spectrum Fg[0..mt) was loaded into cur[0..mt) by spec_load_async (each
// output needs both F[k] and F[h-k]); it is unpacked into other[padi(k)], the
// DFT runs there, and the buffer it leaves free receives the next map's
// spectrum (load_next) while this ring is stored.  On return cur holds the
// next input.  ref != nullptr: write ref - x (Jacobi residual).
template <int KIND, typename T, typename Next>
__device__ void ring_inverse(cplx<T>*& cur, cplx<T>*& other, int shift, T* __restrict__ x,
                             const T* __restrict__ ref, const RingPair& rp, const PhaseTab<T>& tw,
                             const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
                             const PhaseTab<T>& E, int lt, int tpf, int g, Next load_next) {
    const int h = rp.h, mt = rp.mt;
    cp_async_wait<0>();
    group_sync(tpf, g);
    const cplx<T>* Fs = cur;
    cplx<T>* buf = other;
    // Entries k and h-k share F_k, F_{h-k} and one twiddle: buf_{h-k} =
    // conj(sum - i r) for buf_k = sum + i r, and conj of the ring phase of h-k
    // is i e^{-i pi k/n}.
    for (int k = lt; 2 * k <= h; k += tpf) {
        // X_k and conj(X_{h-k}) with the phase e^{+i s k pi/n}; imag of X_0, X_h dropped
        const int kb = h - k;
        const cplx<T> e = shift ? E(k) : cplx<T>{(T)1, (T)0};
        cplx<T> Xa = {(T)0, (T)0}, Xb = {(T)0, (T)0};
        if (k < mt) Xa = shift ? cmul(Fs[k], cconj(e)) : Fs[k];
        if (kb < mt) Xb = cconj(shift ? cmul(Fs[kb], cplx<T>{-e.im, e.re}) : Fs[kb]);
        if (k == 0) {
            Xa.im = (T)0;
            Xb.im = (T)0;
        }
        const cplx<T> sum = cadd(Xa, Xb), dif = csub(Xa, Xb);
        const cplx<T> r = cmul(cconj(E(2 * k)), dif);  // e^{+2 pi i k/n} (Xa - Xb)
        buf[k] = {sum.re - r.im, sum.im + r.re};  // sum + i r (unpadded: the FFT's first pass reads it)
        if (k != 0 && kb != k) buf[kb] = {sum.re + r.im, r.re - sum.im};
    }
    cplx<T>* z = ring_dft<KIND>(buf, cur, rp, tw, gtab, chirp, true, lt, tpf, g);  // starts with a group sync
    cplx<T>* freeb = (z == buf) ? cur : buf;
    load_next(freeb);
    // z holds the ring in natural unpadded order: two complex values per
    // 16-byte access when both ends are aligned (HEALPix rings of an aligned map
    // start at a multiple of 4 pixels)
    bool vec = false;
    if constexpr (sizeof(T) == 4)
        vec = !ref && (h & 1) == 0 && ((((uintptr_t)x) | ((uintptr_t)z)) & 15) == 0;
    if (vec) {
        const float4* zs = (const float4*)z;
        float4* xd = (float4*)x;
        for (int j = lt; j < h / 2; j += tpf) xd[j] = zs[j];
    } else {
        for (int j = lt; j < h; j += tpf) {
            cplx<T> v = z[j];
            if (ref) {
                const cplx<T> rv = *(const cplx<T>*)(ref + 2 * j);
                v = csub(rv, v);
            }
            *(cplx<T>*)(x + 2 * j) = v;
        }
    }
    group_sync(tpf, g);
    cur = freeb;
    other = z;
}

}  // namespace hpx
