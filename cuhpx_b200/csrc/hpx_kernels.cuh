// Batched ring-stage kernels and layout helpers of the SHT pipeline.
#pragma once

#include "legendre.cuh"
#include "tc_ptx.cuh"

namespace hpx {

// Per-m ring-stage scale factors, see the adjoint derivation in hpx_plan.cu.
enum RingMode : int {
    kRingPlain = 0,    // forward: S/D weighted by w_t;  inverse: F = E +/- O
    kRingAdjoint = 1,  // forward-side adjoint of the inverse: weight c_m = 2 (1 at m=0, nphi/2)
                       // inverse-side adjoint of the forward: scale w_t * c_m/2 (w_t at m=0, nphi/2)
    kRingResidual = 2  // inverse: write ref - synthesis (Jacobi residual)
};

template <typename T>
__host__ __device__ constexpr size_t ring_smem_bytes(int bufP, int mtmax, int nmax) {
    return ((size_t)bufP + 2 * (size_t)mtmax + 64 + (2 * (size_t)nmax + 63) / 64 + 2) * sizeof(cplx<T>);
}

// map[b][npix] -> spec[m][0|1][p][c]
// With xh != nullptr (mixed-precision plans) the folded spectra are written as
// bf16 hi/lo pairs xh/xl[m][par][p][c] instead of T values in spec.
template <typename T>
__global__ void __launch_bounds__(256) k_ring_fwd(const T* __restrict__ map, int nmaps, int maps_per_cta,
                                                  T* __restrict__ spec, int C, int nside, int mtmax, int bufP,
                                                  const RingPair* __restrict__ pairs, const cplx<T>* __restrict__ tw,
                                                  int logPmax, const cplx<T>* __restrict__ gtab, int mode,
                                                  uint32_t* __restrict__ xh, uint32_t* __restrict__ xl) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = 2 * nside;
    const int p = blockIdx.x;
    const RingPair rp = pairs[p];
    cplx<T>* buf = (cplx<T>*)smem_raw;
    cplx<T>* Fn = buf + bufP;
    cplx<T>* Fs = Fn + mtmax;
    cplx<T>* elo = Fs + mtmax;
    cplx<T>* ehi = elo + 64;
    build_phase_tab(elo, ehi, rp.nphi);
    __syncthreads();
    const PhaseTab<T> E{elo, ehi, 2 * rp.nphi};
    const int64_t np = npix(nside);
    const int b0 = blockIdx.y * maps_per_cta;
    const int b1 = min(b0 + maps_per_cta, nmaps);
    for (int b = b0; b < b1; ++b) {
        const T* mp = map + (int64_t)b * np;
        ring_forward(mp + rp.start_n, rp.shift_n, buf, Fn, rp, tw, logPmax, gtab, E);
        __syncthreads();
        if (rp.has_south) {
            ring_forward(mp + rp.start_s, rp.shift_s, buf, Fs, rp, tw, logPmax, gtab, E);
            __syncthreads();
        }
        for (int k = threadIdx.x; k < rp.mt; k += blockDim.x) {
            T wk;
            if (mode == kRingAdjoint) wk = (k == 0 || k == rp.h) ? (T)1 : (T)2;
            else wk = (T)rp.w;
            cplx<T> S, D;
            if (rp.has_south) {
                S = cscale(cadd(Fn[k], Fs[k]), wk);
                D = cscale(csub(Fn[k], Fs[k]), wk);
            } else {
                S = cscale(Fn[k], wk);
                D = {(T)0, (T)0};
            }
            const int64_t i0 = (((int64_t)k * 2 + 0) * NP + p) * C + 2 * b;
            const int64_t i1 = (((int64_t)k * 2 + 1) * NP + p) * C + 2 * b;
            if (xh) {
                uint16_t h0, l0, h1, l1;
                tc::split_bf16((float)S.re, h0, l0);
                tc::split_bf16((float)S.im, h1, l1);
                xh[i0 >> 1] = (uint32_t)h0 | ((uint32_t)h1 << 16);
                xl[i0 >> 1] = (uint32_t)l0 | ((uint32_t)l1 << 16);
                tc::split_bf16((float)D.re, h0, l0);
                tc::split_bf16((float)D.im, h1, l1);
                xh[i1 >> 1] = (uint32_t)h0 | ((uint32_t)h1 << 16);
                xl[i1 >> 1] = (uint32_t)l0 | ((uint32_t)l1 << 16);
            } else {
                *(cplx<T>*)(spec + i0) = S;
                *(cplx<T>*)(spec + i1) = D;
            }
        }
        __syncthreads();
    }
}

// spec[m][0|1][p][c] -> map[b][npix]
template <typename T>
__global__ void __launch_bounds__(256) k_ring_inv(const T* __restrict__ spec, int C, T* __restrict__ map, int nmaps,
                                                  int maps_per_cta, int nside, int mtmax, int bufP,
                                                  const RingPair* __restrict__ pairs, const cplx<T>* __restrict__ tw,
                                                  int logPmax, const cplx<T>* __restrict__ gtab, int mode,
                                                  const T* __restrict__ ref) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = 2 * nside;
    const int p = blockIdx.x;
    const RingPair rp = pairs[p];
    cplx<T>* buf = (cplx<T>*)smem_raw;
    cplx<T>* Fn = buf + bufP;
    cplx<T>* Fs = Fn + mtmax;
    cplx<T>* elo = Fs + mtmax;
    cplx<T>* ehi = elo + 64;
    build_phase_tab(elo, ehi, rp.nphi);
    __syncthreads();
    const PhaseTab<T> E{elo, ehi, 2 * rp.nphi};
    const int64_t np = npix(nside);
    const int b0 = blockIdx.y * maps_per_cta;
    const int b1 = min(b0 + maps_per_cta, nmaps);
    for (int b = b0; b < b1; ++b) {
        for (int k = threadIdx.x; k < rp.mt; k += blockDim.x) {
            cplx<T> e = *(const cplx<T>*)(spec + (((int64_t)k * 2 + 0) * NP + p) * C + 2 * b);
            cplx<T> o = *(const cplx<T>*)(spec + (((int64_t)k * 2 + 1) * NP + p) * C + 2 * b);
            T sc = (T)1;
            if (mode == kRingAdjoint) sc = (k == 0 || k == rp.h) ? (T)rp.w : (T)(0.5 * rp.w);
            Fn[k] = cscale(cadd(e, o), sc);
            Fs[k] = cscale(csub(e, o), sc);
        }
        __syncthreads();
        T* mp = map + (int64_t)b * np;
        ring_inverse(Fn, rp.shift_n, buf, mp + rp.start_n, rp, tw, logPmax, gtab, E);
        __syncthreads();
        if (rp.has_south) {
            ring_inverse(Fs, rp.shift_s, buf, mp + rp.start_s, rp, tw, logPmax, gtab, E);
            __syncthreads();
        }
        if (mode == kRingResidual) {
            const T* rf = ref + (int64_t)b * np;
            for (int j = threadIdx.x; j < rp.nphi; j += blockDim.x) {
                mp[rp.start_n + j] = rf[rp.start_n + j] - mp[rp.start_n + j];
                if (rp.has_south) mp[rp.start_s + j] = rf[rp.start_s + j] - mp[rp.start_s + j];
            }
            __syncthreads();
        }
    }
}

// alm[b][l][m] (complex) -> almT[m][l][c], c = 2b + {re, im}
template <typename T>
__global__ void k_alm_to_cols(const T* __restrict__ alm, int nmaps, int L, int M, T* __restrict__ almT, int C) {
    __shared__ cplx<T> tile[16][33];
    const int m0 = blockIdx.x * 32, l = blockIdx.y, b0 = blockIdx.z * 16;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int i = ty; i < 16; i += 8) {
        const int b = b0 + i, m = m0 + tx;
        cplx<T> v = {(T)0, (T)0};
        if (b < nmaps && m < M) v = *(const cplx<T>*)(alm + 2 * (((int64_t)b * L + l) * M + m));
        tile[i][tx] = v;
    }
    __syncthreads();
    // write: for each m in tile, 32 consecutive columns (16 maps x re/im)
    for (int i = ty; i < 32; i += 8) {
        const int m = m0 + i;
        const int c = 2 * b0 + tx;
        if (m < M && c < C) {
            cplx<T> v = tile[tx >> 1][i];
            almT[((int64_t)m * L + l) * C + c] = (tx & 1) ? v.im : v.re;
        }
    }
}

// Bluestein chirp spectra: G_p = FFT_P(g) / P stored bit-reversed, g_j = e^{+i pi j^2/h}
// for |j| < h (circularly wrapped), computed in FP64 and rounded to T.
template <typename T>
__global__ void __launch_bounds__(256) k_chirp_spectra(const RingPair* __restrict__ pairs,
                                                       const cplx<double>* __restrict__ tw64, int logPmax,
                                                       cplx<T>* __restrict__ gtab) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const RingPair rp = pairs[blockIdx.x];
    if (rp.logh >= 0) return;
    cplx<double>* buf = (cplx<double>*)smem_raw;
    const int P = 1 << rp.logP, h = rp.h;
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        int d = j < h ? j : (j > P - h ? P - j : -1);
        cplx<double> v = {0.0, 0.0};
        if (d >= 0) {
            long long q = ((long long)d * d) % (2 * h);
            double s, c;
            sincospi((double)q / (double)h, &s, &c);
            v = {c, s};
        }
        buf[j] = v;
    }
    __syncthreads();
    fft_dif(buf, rp.logP, tw64, logPmax, false);
    const double inv = 1.0 / (double)P;
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        gtab[rp.gtab_off + j] = {(T)(buf[j].re * inv), (T)(buf[j].im * inv)};
    }
}

// tw[q] = e^{-2 pi i q / Pmax}
template <typename T>
__global__ void k_twiddles(cplx<T>* tw, int Pmax) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < Pmax / 2) {
        double s, c;
        sincospi(-2.0 * (double)q / (double)Pmax, &s, &c);
        tw[q] = {(T)c, (T)s};
    }
}

}  // namespace hpx
