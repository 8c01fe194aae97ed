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

// tw[q] = e^{-2 pi i q / Pmax} for q < Pmax/2; the other half by symmetry
template <typename T>
__device__ __forceinline__ cplx<T> twid(const cplx<T>* __restrict__ tw, int q, int half) {
    if (q < half) return tw[q];
    cplx<T> v = tw[q - half];
    return {-v.re, -v.im};
}

// Stockham autosort radix-4/2 FFT of length P = 2^logP on src (natural order);
// returns the buffer (src or dst) that holds the natural-order result.
// INV: e^{+2 pi i jk/P} (unnormalised).  Threads: lt in [0, tpf) of group g.
template <typename T, bool INV>
__device__ cplx<T>* stockham(cplx<T>* src, cplx<T>* dst, int logP, const cplx<T>* __restrict__ tw, int logPmax,
                             int lt, int tpf, int g) {
    const int P = 1 << logP;
    const int half = 1 << (logPmax - 1);
    int Ns = 1;
    int rem = logP;
    while (rem > 0) {
        if (rem >= 2) {
            const int Q = P >> 2;
            const int step = (1 << logPmax) / (Ns * 4);  // twiddle index stride
            for (int j = lt; j < Q; j += tpf) {
                const int k = j & (Ns - 1);
                cplx<T> v0 = src[j], v1 = src[j + Q], v2 = src[j + 2 * Q], v3 = src[j + 3 * Q];
                if (Ns > 1) {
                    cplx<T> w1 = twid(tw, k * step, half), w2 = twid(tw, 2 * k * step, half),
                            w3 = twid(tw, 3 * k * step, half);
                    if (INV) {
                        w1.im = -w1.im;
                        w2.im = -w2.im;
                        w3.im = -w3.im;
                    }
                    v1 = cmul(v1, w1);
                    v2 = cmul(v2, w2);
                    v3 = cmul(v3, w3);
                }
                const cplx<T> t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3);
                const cplx<T> d = csub(v1, v3);
                // forward: -i*d ; inverse: +i*d
                const cplx<T> t3 = INV ? cplx<T>{-d.im, d.re} : cplx<T>{d.im, -d.re};
                const int o = ((j - k) << 2) + k;
                dst[o] = cadd(t0, t2);
                dst[o + Ns] = cadd(t1, t3);
                dst[o + 2 * Ns] = csub(t0, t2);
                dst[o + 3 * Ns] = csub(t1, t3);
            }
            Ns <<= 2;
            rem -= 2;
        } else {
            const int Q = P >> 1;
            const int step = (1 << logPmax) / (Ns * 2);
            for (int j = lt; j < Q; j += tpf) {
                const int k = j & (Ns - 1);
                cplx<T> v0 = src[j], v1 = src[j + Q];
                if (Ns > 1) {
                    cplx<T> w = twid(tw, k * step, half);
                    if (INV) w.im = -w.im;
                    v1 = cmul(v1, w);
                }
                const int o = ((j - k) << 1) + k;
                dst[o] = cadd(v0, v1);
                dst[o + Ns] = csub(v0, v1);
            }
            Ns <<= 1;
            rem -= 1;
        }
        group_sync(tpf, g);
        cplx<T>* t = src;
        src = dst;
        dst = t;
    }
    return src;
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
__device__ cplx<T>* ring_dft(cplx<T>* buf, cplx<T>* buf2, const RingPair& rp, const cplx<T>* __restrict__ tw,
                             int logPmax, const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
                             bool inv, int lt, int tpf, int g) {
    group_sync(tpf, g);
    if (rp.logh >= 0) {
        if (rp.logh == 0) return buf;
        return inv ? stockham<T, true>(buf, buf2, rp.logh, tw, logPmax, lt, tpf, g)
                   : stockham<T, false>(buf, buf2, rp.logh, tw, logPmax, lt, tpf, g);
    }
    // Bluestein; inverse via conj(DFT(conj z)).  c_j = e^{-i pi j^2/h}.
    const int P = 1 << rp.logP;
    const int h = rp.h;
    for (int j = lt; j < P; j += tpf) {
        cplx<T> a = {(T)0, (T)0};
        if (j < h) {
            a = buf[j];
            if (inv) a.im = -a.im;
            a = cmul(a, chirp[j]);
        }
        buf[j] = a;
    }
    group_sync(tpf, g);
    cplx<T>* r = stockham<T, false>(buf, buf2, rp.logP, tw, logPmax, lt, tpf, g);
    cplx<T>* o = (r == buf) ? buf2 : buf;
    const cplx<T>* G = gtab + rp.gtab_off;
    for (int j = lt; j < P; j += tpf) r[j] = cmul(r[j], G[j]);
    group_sync(tpf, g);
    r = stockham<T, true>(r, o, rp.logP, tw, logPmax, lt, tpf, g);
    for (int k = lt; k < h; k += tpf) {
        cplx<T> v = cmul(r[k], chirp[k]);
        if (inv) v.im = -v.im;
        r[k] = v;
    }
    group_sync(tpf, g);
    return r;
}

// Forward transform of one real ring x[0..n) into F[0..mt) (global, contiguous).
template <typename T>
__device__ void ring_forward(const T* __restrict__ x, int shift, cplx<T>* buf, cplx<T>* buf2, T* __restrict__ F,
                             const RingPair& rp, const cplx<T>* __restrict__ tw, int logPmax,
                             const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
                             const PhaseTab<T>& E, int lt, int tpf, int g) {
    const int h = rp.h;
    for (int j = lt; j < h; j += tpf) {
        buf[j] = *(const cplx<T>*)(x + 2 * j);
    }
    cplx<T>* Z = ring_dft(buf, buf2, rp, tw, logPmax, gtab, chirp, false, lt, tpf, g);
    for (int k = lt; k < rp.mt; k += tpf) {
        const int k1 = k == h ? 0 : k;
        const int k2 = k == 0 ? 0 : h - k;
        const cplx<T> Zk = Z[k1];
        const cplx<T> Zc = cconj(Z[k2]);
        const cplx<T> Ek = cscale(cadd(Zk, Zc), (T)0.5);
        const cplx<T> d = cscale(csub(Zk, Zc), (T)0.5);
        const cplx<T> Ok = {d.im, -d.re};  // -i * d
        cplx<T> X = cadd(Ek, cmul(E(2 * k), Ok));
        if (shift) X = cmul(E(k), X);
        *(cplx<T>*)(F + 2 * k) = X;
    }
    group_sync(tpf, g);
}

// Inverse transform of spectrum Fs[0..mt) (shared memory) into one real ring x[0..n).
// ref != nullptr: write ref - x (Jacobi residual).
template <typename T>
__device__ void ring_inverse(const cplx<T>* Fs, int shift, cplx<T>* buf, cplx<T>* buf2, T* __restrict__ x,
                             const T* __restrict__ ref, const RingPair& rp, const cplx<T>* __restrict__ tw,
                             int logPmax, const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
                             const PhaseTab<T>& E, int lt, int tpf, int g) {
    const int h = rp.h, mt = rp.mt;
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
        buf[k] = {sum.re - r.im, sum.im + r.re};       // sum + i r
    }
    cplx<T>* z = ring_dft(buf, buf2, rp, tw, logPmax, gtab, chirp, true, lt, tpf, g);
    for (int j = lt; j < h; j += tpf) {
        cplx<T> v = z[j];
        if (ref) {
            const cplx<T> rv = *(const cplx<T>*)(ref + 2 * j);
            v = csub(rv, v);
        }
        *(cplx<T>*)(x + 2 * j) = v;
    }
    group_sync(tpf, g);
}

}  // namespace hpx
