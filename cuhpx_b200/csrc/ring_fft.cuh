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
// Design (not the reference's): one CTA owns a ring pair (north ring t and its
// mirror) for a group of maps.  A real ring of length n = nphi is packed into
// a complex sequence of length h = n/2; if h is a power of two it goes through
// a radix-2 FFT in shared memory, otherwise through Bluestein's chirp-z
// convolution with a per-ring power-of-two size P >= 2h-1 (the reference pads
// every ring to 8*nside).  Every rotation factor is e^{-i pi q / n} for an
// integer q reduced mod 2n -- the phase shift (q = s*m), the real-FFT split
// (q = 2m) and the Bluestein chirp (q = 2 j^2 mod 2n) -- so phases are exact
// integer reductions evaluated from a per-CTA FP64-built table, never a float
// "pi*j*j/n" as in hpx_fft_cuda.cu:1090.
//
// The forward stage writes the north/south folded, quadrature-weighted spectra
//   S_t[m] = w_t (F_t[m] + F_t'[m]),  D_t[m] = w_t (F_t[m] - F_t'[m])
// (equator: S = w F, D = 0) into spec[m][0|1][p][c] with c = 2*map + {re,im};
// the inverse stage reads E/O = spec[m][0|1][p][c] and unfolds
// F_t = E + O, F_t' = E - O.
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
    int logP;       // Bluestein FFT size (log2), 0 when direct
    int has_south;  // 0 for the equator
    int64_t start_n;
    int64_t start_s;
    int64_t gtab_off;  // offset (complex elements) of the chirp spectrum, -1 if direct
    double z;          // cos(theta) of the north ring
    double w;          // quadrature weight of the ring
};

// ----------------------------------------------------------------- smem FFTs
// tw[q] = e^{-2 pi i q / Pmax}, q < Pmax/2
template <typename T>
__device__ __forceinline__ cplx<T> twiddle(const cplx<T>* __restrict__ tw, int q, bool inv) {
    cplx<T> w = tw[q];
    if (inv) w.im = -w.im;
    return w;
}

// natural order in, bit-reversed order out; sum_j a_j e^{-/+ 2 pi i j k / P}
template <typename T>
__device__ void fft_dif(cplx<T>* a, int logP, const cplx<T>* __restrict__ tw, int logPmax, bool inv) {
    const int P2 = 1 << (logP - 1);
    for (int s = logP; s >= 1; --s) {
        const int half = 1 << (s - 1);
        for (int b = threadIdx.x; b < P2; b += blockDim.x) {
            int j = b & (half - 1);
            int i0 = ((b >> (s - 1)) << s) + j;
            int i1 = i0 + half;
            cplx<T> u = a[i0], v = a[i1];
            a[i0] = cadd(u, v);
            a[i1] = cmul(csub(u, v), twiddle(tw, j << (logPmax - s), inv));
        }
        __syncthreads();
    }
}

// bit-reversed order in, natural order out
template <typename T>
__device__ void fft_dit(cplx<T>* a, int logP, const cplx<T>* __restrict__ tw, int logPmax, bool inv) {
    const int P2 = 1 << (logP - 1);
    for (int s = 1; s <= logP; ++s) {
        const int half = 1 << (s - 1);
        for (int b = threadIdx.x; b < P2; b += blockDim.x) {
            int j = b & (half - 1);
            int i0 = ((b >> (s - 1)) << s) + j;
            int i1 = i0 + half;
            cplx<T> u = a[i0];
            cplx<T> v = cmul(a[i1], twiddle(tw, j << (logPmax - s), inv));
            a[i0] = cadd(u, v);
            a[i1] = csub(u, v);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int bitrev(int x, int bits) { return bits == 0 ? 0 : (int)(__brev((unsigned)x) >> (32 - bits)); }

// e^{-i pi q / n} from two small tables: q = 64*hi + lo
template <typename T>
struct PhaseTab {
    const cplx<T>* lo;  // 64 entries
    const cplx<T>* hi;  // ceil(2n/64) entries
    int two_n;
    __device__ __forceinline__ cplx<T> operator()(int q) const {
        q %= two_n;
        if (q < 0) q += two_n;
        return cmul(hi[q >> 6], lo[q & 63]);
    }
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

// Complex DFT of length h held in buf: fwd computes sum_j z_j e^{-2 pi i jk/h}.
// Input z must already be in buf (natural order, h entries).  Result is
// returned through get(k) semantics: after the call, zget(buf, k) gives Z_k.
//   direct (logh >= 0): result in bit-reversed order
//   Bluestein: result in natural order, multiplied by chirp on read
template <typename T>
__device__ void ring_dft(cplx<T>* buf, const RingPair& rp, const cplx<T>* __restrict__ tw, int logPmax,
                         const cplx<T>* __restrict__ gtab, const PhaseTab<T>& E, bool inv) {
    if (rp.logh >= 0) {
        __syncthreads();
        if (rp.logh > 0) fft_dif(buf, rp.logh, tw, logPmax, inv);
        return;
    }
    // Bluestein; inverse via conj(DFT(conj z))
    __syncthreads();
    const int P = 1 << rp.logP;
    const int h = rp.h, n = rp.nphi;
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        cplx<T> a = {(T)0, (T)0};
        if (j < h) {
            a = buf[j];
            if (inv) a.im = -a.im;
            // c_j = e^{-i pi j^2 / h} = E(2 j^2 mod 2n)
            long long q = (2ll * j * j) % (2 * n);
            a = cmul(a, E((int)q));
        }
        buf[j] = a;
    }
    __syncthreads();
    fft_dif(buf, rp.logP, tw, logPmax, false);
    const cplx<T>* G = gtab + rp.gtab_off;
    for (int j = threadIdx.x; j < P; j += blockDim.x) buf[j] = cmul(buf[j], G[j]);
    __syncthreads();
    fft_dit(buf, rp.logP, tw, logPmax, true);
    for (int k = threadIdx.x; k < h; k += blockDim.x) {
        long long q = (2ll * k * k) % (2 * n);
        cplx<T> v = cmul(buf[k], E((int)q));
        if (inv) v.im = -v.im;
        buf[k] = v;
    }
    __syncthreads();
}

template <typename T>
__device__ __forceinline__ cplx<T> zget(const cplx<T>* buf, const RingPair& rp, int k) {
    return rp.logh >= 0 ? buf[bitrev(k, rp.logh)] : buf[k];
}

// Forward transform of one real ring x[0..n) into F[0..mt).
template <typename T>
__device__ void ring_forward(const T* __restrict__ x, int shift, cplx<T>* buf, cplx<T>* F, const RingPair& rp,
                             const cplx<T>* __restrict__ tw, int logPmax, const cplx<T>* __restrict__ gtab,
                             const PhaseTab<T>& E) {
    const int h = rp.h;
    for (int j = threadIdx.x; j < h; j += blockDim.x) {
        buf[j] = {x[2 * j], x[2 * j + 1]};
    }
    ring_dft(buf, rp, tw, logPmax, gtab, E, false);
    for (int k = threadIdx.x; k < rp.mt; k += blockDim.x) {
        int k1 = k == h ? 0 : k;
        int k2 = k == 0 ? 0 : h - k;
        cplx<T> Zk = zget(buf, rp, k1);
        cplx<T> Zc = cconj(zget(buf, rp, k2));
        cplx<T> Ek = cscale(cadd(Zk, Zc), (T)0.5);
        cplx<T> d = cscale(csub(Zk, Zc), (T)0.5);
        cplx<T> Ok = {d.im, -d.re};  // -i * d
        cplx<T> X = cadd(Ek, cmul(E(2 * k), Ok));
        F[k] = cmul(E(shift * k), X);
    }
}

// Inverse transform of spectrum F[0..mt) into one real ring x[0..n).
template <typename T>
__device__ void ring_inverse(const cplx<T>* F, int shift, cplx<T>* buf, T* __restrict__ x, const RingPair& rp,
                             const cplx<T>* __restrict__ tw, int logPmax, const cplx<T>* __restrict__ gtab,
                             const PhaseTab<T>& E) {
    const int h = rp.h, mt = rp.mt;
    for (int k = threadIdx.x; k < h; k += blockDim.x) {
        // X_k and conj(X_{h-k}) with the phase e^{+i s k pi/n}; imag of X_0, X_h dropped
        cplx<T> Xa = {(T)0, (T)0}, Xb = {(T)0, (T)0};
        if (k < mt) Xa = cmul(F[k], cconj(E(shift * k)));
        int kb = h - k;
        if (kb < mt) Xb = cconj(cmul(F[kb], cconj(E(shift * kb))));
        if (k == 0) {
            Xa.im = (T)0;
            Xb.im = (T)0;
        }
        cplx<T> sum = cadd(Xa, Xb), dif = csub(Xa, Xb);
        cplx<T> r = cmul(cconj(E(2 * k)), dif);  // e^{+2 pi i k/n} (Xa - Xb)
        buf[k] = {sum.re - r.im, sum.im + r.re};   // sum + i r
    }
    ring_dft(buf, rp, tw, logPmax, gtab, E, true);
    for (int j = threadIdx.x; j < h; j += blockDim.x) {
        cplx<T> z = zget(buf, rp, j);
        x[2 * j] = z.re;
        x[2 * j + 1] = z.im;
    }
}

}  // namespace hpx
