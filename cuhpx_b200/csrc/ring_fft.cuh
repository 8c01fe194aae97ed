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
// through a Stockham radix-4/2 FFT in shared memory, otherwise through
// Bluestein's chirp-z convolution with a per-ring power-of-two size
// P >= 2h-1 (the reference pads every ring to 8*nside).  Small rings are
// transformed by sub-groups of a CTA (one warp, two, four or all eight) so
// that every thread handles ~16 points whatever the ring length.
//
// Phases are exact: the chirp e^{-i pi j^2/h} is tabulated per ring in the plan
// from the integer j^2 mod 2h in FP64, and the real-FFT split and phase-shift
// factors e^{-i pi q/n} (q <= 2n) come from a per-CTA FP64-built table --
// never from a float "pi*j*j/n" as in hpx_fft_cuda.cu:1090.
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
    int pad_;
    int64_t start_n;   // first pixel of the north ring
    int64_t start_s;   // first pixel of the south ring
    int64_t foff_n;    // spectrum offset of the north ring in F[map][.]
    int64_t foff_s;    // ... of the south ring
    int64_t gtab_off;  // offset of the chirp spectrum / chirp (complex elements), -1 if direct
    double z;          // cos(theta) of the north ring
    double w;          // quadrature weight of the ring
};

// FFT work buffers are padded by one element every 16 so that the strided
// Stockham stores of the first pass (stride 16 complex) spread over all banks.
__device__ __forceinline__ int padi(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int P) { return P + (P >> 4) + 1; }

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

// Stockham autosort FFT of length P = 2^logP on src (natural order); returns the
// buffer (src or dst) holding the natural-order result.  twP[q] = e^{-2 pi i q/P}
// for q < P/2 (shared memory).  INV: e^{+2 pi i jk/P} (unnormalised).
// First pass radix-16 in registers (contiguous 16-element stores), then radix-4
// stages, and one radix-2 stage when log2(P) is odd.
template <typename T, bool INV>
__device__ cplx<T>* stockham(cplx<T>* src, cplx<T>* dst, int logP, const cplx<T>* __restrict__ twP, int lt,
                             int tpf, int g) {
    const int P = 1 << logP;
    int Ns = 1;
    int rem = logP;
    auto swap_bufs = [&]() {
        group_sync(tpf, g);
        cplx<T>* t = src;
        src = dst;
        dst = t;
    };
    if (rem >= 4) {
        const int Q = P >> 4;
        for (int j = lt; j < Q; j += tpf) {
            cplx<T> v[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) v[r] = src[padi(j + r * Q)];
            dft16<T, INV>(v);
            // outputs 16j .. 16j+15 are one aligned 16-run: padded index 17j + r
#pragma unroll
            for (int r = 0; r < 16; ++r) dst[17 * j + r] = v[r];
        }
        Ns = 16;
        rem -= 4;
        swap_bufs();
    }
    while (rem >= 2) {
        const int Q = P >> 2;
        const int step = P / (Ns * 4);
        for (int j = lt; j < Q; j += tpf) {
            const int k = j & (Ns - 1);
            cplx<T> v0 = src[padi(j)], v1 = src[padi(j + Q)], v2 = src[padi(j + 2 * Q)], v3 = src[padi(j + 3 * Q)];
            if (Ns > 1) {
                cplx<T> w1 = twP[k * step];
                if (INV) w1.im = -w1.im;
                const cplx<T> w2 = cmul(w1, w1), w3 = cmul(w1, w2);
                v1 = cmul(v1, w1);
                v2 = cmul(v2, w2);
                v3 = cmul(v3, w3);
            }
            dft4<T, INV>(v0, v1, v2, v3);
            const int o = ((j - k) << 2) + k;
            dst[padi(o)] = v0;
            dst[padi(o + Ns)] = v1;
            dst[padi(o + 2 * Ns)] = v2;
            dst[padi(o + 3 * Ns)] = v3;
        }
        Ns <<= 2;
        rem -= 2;
        swap_bufs();
    }
    if (rem == 1) {
        const int Q = P >> 1;
        const int step = P / (Ns * 2);
        for (int j = lt; j < Q; j += tpf) {
            const int k = j & (Ns - 1);
            cplx<T> v0 = src[padi(j)], v1 = src[padi(j + Q)];
            if (Ns > 1) {
                cplx<T> w = twP[k * step];
                if (INV) w.im = -w.im;
                v1 = cmul(v1, w);
            }
            const int o = ((j - k) << 1) + k;
            dst[padi(o)] = cadd(v0, v1);
            dst[padi(o + Ns)] = csub(v0, v1);
        }
        swap_bufs();
    }
    return src;
}

// twP[q] = e^{-2 pi i q / P}, q < P/2, from the plan's table for Pmax (all threads of the CTA)
template <typename T>
__device__ void load_twiddles(cplx<T>* twP, int logP, const cplx<T>* __restrict__ tw, int logPmax) {
    const int half = 1 << (logP - 1);
    const int stride = 1 << (logPmax - logP);
    for (int q = threadIdx.x; q < half; q += blockDim.x) twP[q] = tw[q * stride];
}

// e^{-i pi q / n} for 0 <= q < 2n from two small tables: q = 64*hi + lo
template <typename T>
struct PhaseTab {
    const cplx<T>* lo;  // 64 entries
    const cplx<T>* hi;  // ceil(2n/64) entries
    __device__ __forceinline__ cplx<T> operator()(int q) const { return cmul(hi[q >> 6], lo[q & 63]); }
};

template <typename T>
__device__ void build_phase_tab(cplx<T>* lo, cplx<T>* hi, int n) {
    const int nhi = (2 * n + 63) / 64;
    for (int i = threadIdx.x; i < 64 + nhi; i += blockDim.x) {
        int q = i < 64 ? i : 64 * (i - 64);
        double s, c;
        sincospi(-(double)q / (double)n, &s, &c);
        cplx<T> v = {(T)c, (T)s};
        if (i < 64) lo[i] = v; else hi[i - 64] = v;
    }
}

// Complex DFT of length h of buf (natural order, h entries written by this
// group), forward (e^-) or inverse (e^+); returns the buffer with Z in natural order.
template <typename T>
__device__ cplx<T>* ring_dft(cplx<T>* buf, cplx<T>* buf2, const RingPair& rp, const cplx<T>* __restrict__ twP,
                             const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp, bool inv, int lt,
                             int tpf, int g) {
    group_sync(tpf, g);
    if (rp.logh >= 0) {
        if (rp.logh == 0) return buf;
        return inv ? stockham<T, true>(buf, buf2, rp.logh, twP, lt, tpf, g)
                   : stockham<T, false>(buf, buf2, rp.logh, twP, lt, tpf, g);
    }
    // Bluestein; inverse via conj(DFT(conj z)).  c_j = e^{-i pi j^2/h}.
    const int P = 1 << rp.logP;
    const int h = rp.h;
    for (int j = lt; j < P; j += tpf) {
        cplx<T> a = {(T)0, (T)0};
        if (j < h) {
            a = buf[padi(j)];
            if (inv) a.im = -a.im;
            a = cmul(a, chirp[j]);
        }
        buf[padi(j)] = a;
    }
    group_sync(tpf, g);
    cplx<T>* r = stockham<T, false>(buf, buf2, rp.logP, twP, lt, tpf, g);
    cplx<T>* o = (r == buf) ? buf2 : buf;
    const cplx<T>* G = gtab + rp.gtab_off;
    for (int j = lt; j < P; j += tpf) r[padi(j)] = cmul(r[padi(j)], G[j]);
    group_sync(tpf, g);
    r = stockham<T, true>(r, o, rp.logP, twP, lt, tpf, g);
    for (int k = lt; k < h; k += tpf) {
        cplx<T> v = cmul(r[padi(k)], chirp[k]);
        if (inv) v.im = -v.im;
        r[padi(k)] = v;
    }
    group_sync(tpf, g);
    return r;
}

// Forward transform of one real ring x[0..n) into F[0..mt) (global, contiguous).
// Returns the largest |re|, |im| this thread wrote.
template <typename T>
__device__ T ring_forward(const T* __restrict__ x, int shift, cplx<T>* buf, cplx<T>* buf2, T* __restrict__ F,
                             const RingPair& rp, const cplx<T>* __restrict__ twP, const cplx<T>* __restrict__ gtab,
                             const cplx<T>* __restrict__ chirp, const PhaseTab<T>& E, int lt, int tpf, int g) {
    const int h = rp.h;
    for (int j = lt; j < h; j += tpf) {
        buf[padi(j)] = *(const cplx<T>*)(x + 2 * j);
    }
    cplx<T>* Z = ring_dft(buf, buf2, rp, twP, gtab, chirp, false, lt, tpf, g);
    T mx = (T)0;
    for (int k = lt; k < rp.mt; k += tpf) {
        const int k1 = k == h ? 0 : k;
        const int k2 = k == 0 ? 0 : h - k;
        const cplx<T> Zk = Z[padi(k1)];
        const cplx<T> Zc = cconj(Z[padi(k2)]);
        const cplx<T> Ek = cscale(cadd(Zk, Zc), (T)0.5);
        const cplx<T> d = cscale(csub(Zk, Zc), (T)0.5);
        const cplx<T> Ok = {d.im, -d.re};  // -i * d
        cplx<T> X = cadd(Ek, cmul(E(2 * k), Ok));
        if (shift) X = cmul(E(k), X);
        *(cplx<T>*)(F + 2 * k) = X;
        mx = fmax(mx, fmax(fabs(X.re), fabs(X.im)));
    }
    group_sync(tpf, g);
    return mx;
}

// Inverse transform of the ring spectrum Fg[0..mt) (global) into one real ring
// x[0..n).  The spectrum is staged once, contiguously, into buf2 (free until
// the DFT starts), because each output needs both F[k] and F[h-k].
// ref != nullptr: write ref - x (Jacobi residual).
template <typename T>
__device__ void ring_inverse(const cplx<T>* __restrict__ Fg, int shift, cplx<T>* buf, cplx<T>* buf2, T* __restrict__ x,
                             const T* __restrict__ ref, const RingPair& rp, const cplx<T>* __restrict__ twP,
                             const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
                             const PhaseTab<T>& E, int lt, int tpf, int g) {
    const int h = rp.h, mt = rp.mt;
    for (int k = lt; k < mt; k += tpf) buf2[k] = Fg[k];
    group_sync(tpf, g);
    const cplx<T>* Fs = buf2;
    for (int k = lt; k < h; k += tpf) {
        // X_k and conj(X_{h-k}) with the phase e^{+i s k pi/n}; imag of X_0, X_h dropped
        cplx<T> Xa = {(T)0, (T)0}, Xb = {(T)0, (T)0};
        if (k < mt) Xa = shift ? cmul(Fs[k], cconj(E(k))) : Fs[k];
        const int kb = h - k;
        if (kb < mt) Xb = cconj(shift ? cmul(Fs[kb], cconj(E(kb))) : Fs[kb]);
        if (k == 0) {
            Xa.im = (T)0;
            Xb.im = (T)0;
        }
        const cplx<T> sum = cadd(Xa, Xb), dif = csub(Xa, Xb);
        const cplx<T> r = cmul(cconj(E(2 * k)), dif);  // e^{+2 pi i k/n} (Xa - Xb)
        buf[padi(k)] = {sum.re - r.im, sum.im + r.re};  // sum + i r
    }
    cplx<T>* z = ring_dft(buf, buf2, rp, twP, gtab, chirp, true, lt, tpf, g);
    for (int j = lt; j < h; j += tpf) {
        cplx<T> v = z[padi(j)];
        if (ref) {
            const cplx<T> rv = *(const cplx<T>*)(ref + 2 * j);
            v = csub(rv, v);
        }
        *(cplx<T>*)(x + 2 * j) = v;
    }
    group_sync(tpf, g);
}

}  // namespace hpx
