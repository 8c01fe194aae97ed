// Batched ring-stage kernels and layout helpers of the SHT pipeline.
#pragma once

#include "legendre.cuh"
#include "tc_ptx.cuh"

namespace hpx {

// complex elements of dynamic shared memory the ring kernels need
// (the phase and twiddle tables, and the padded work buffers of every FFT
// group: groups x P <= 4096 whenever P <= 4096, so the groups' 2 padded_len(P)
// each take at most 2 padded_len(4096) + 32; 64 of slack)
__host__ __device__ constexpr size_t ring_smem_elems(int pfft_max, int nmax) {
    return (size_t)phase_tab_elems(nmax) + (size_t)phase_tab_elems(pfft_max / 2) +
           2 * (size_t)padded_len(pfft_max > 4096 ? pfft_max : 4096) + 64;
}

// CTAs per SM the ring kernels are compiled for: 3 x 256 threads of float
// (80 registers; 3 x 74 KB of shared memory at P = 4096), 2 of double
template <typename T>
constexpr int ring_min_ctas() { return sizeof(T) == 4 ? 3 : 2; }

// Per ring pair, the phase table E (e^{-i pi q/nphi}) and the FFT twiddles
// (e^{-2 pi i q/P}) one after the other, built once per plan into a slot of
// `slot` elements (k_ring_tables); each ring CTA copies its pair's slot.
template <typename T>
__global__ void __launch_bounds__(256) k_ring_tables(const RingPair* __restrict__ pairs, int slot,
                                                     cplx<T>* __restrict__ out) {
    const RingPair rp = pairs[blockIdx.x];
    cplx<T>* et = out + (size_t)blockIdx.x * slot;
    build_phase_tab(et, rp.nphi);
    if (rp.logP > 0) build_phase_tab(et + phase_tab_elems(rp.nphi), ring_fft_len(rp) / 2);
}

// complex elements of a ring pair's table slot (nmax: the largest nphi)
__host__ __device__ constexpr int ring_table_slot(int pfft_max, int nmax) {
    return (phase_tab_elems(nmax) + phase_tab_elems(pfft_max / 2) + 1) & ~1;
}

// shared-memory layout of a ring CTA: phase table E, FFT twiddles (copied from
// the pair's slot), then the work buffers
template <int KIND, typename T>
__device__ __forceinline__ cplx<T>* ring_tables(unsigned char* smem, const RingPair& rp,
                                                const cplx<T>* __restrict__ slot, PhaseTab<T>& E, PhaseTab<T>& tw) {
    cplx<T>* et = (cplx<T>*)smem;
    const int ne = phase_tab_elems(rp.nphi);
    const int half = ring_fft_len_k<KIND>(rp) / 2;
    const int n = ne + (rp.logP > 0 ? phase_tab_elems(half) : 0);
    for (int i = threadIdx.x; i < n; i += blockDim.x) et[i] = slot[i];
    E = PhaseTab<T>{et, et + 64, phase_tab_nhi(rp.nphi)};
    cplx<T>* tt = et + ne;
    tw = rp.logP > 0 ? PhaseTab<T>{tt, tt + 64, phase_tab_nhi(half)} : E;  // no FFT when h = 1
    return tt + phase_tab_elems(half);
}

// Bluestein rings: the ring's chirp (h entries) and the first half of its chirp
// spectrum G (P/2 + 1 entries; G_k = G_{P-k}) are staged in shared memory after
// the phase tables, once per CTA for all its maps; returns the start of the FFT
// buffers.
template <int KIND, typename T>
__device__ __forceinline__ cplx<T>* ring_bluestein_tables(cplx<T>* smem, const RingPair& rp,
                                                          const cplx<T>* __restrict__ gtab,
                                                          const cplx<T>* __restrict__ chirp, const cplx<T>*& Gs,
                                                          const cplx<T>*& cs) {
    const int half = ring_fft_len_k<KIND>(rp) / 2 + 1;
    cplx<T>* gsm = smem;
    cplx<T>* csm = smem + half;
    for (int i = threadIdx.x; i < half; i += blockDim.x) gsm[i] = gtab[rp.gtab_off + i];
    for (int i = threadIdx.x; i < rp.h; i += blockDim.x) csm[i] = chirp[rp.gtab_off + i];
    Gs = gsm;
    cs = csm;
    return csm + rp.h + ((half + rp.h) & 1);  // the buffers start 16-byte aligned
}

// The ring kernels come in three instantiations launched over three ring
// lists: power-of-two rings (KIND 0, 3 CTAs per SM for float), Bluestein rings
// of length 2^logP (KIND 1, 2 CTAs per SM with 128 registers and the ring's
// tables in shared memory) and of length 3 * 2^logP (KIND 2, 3072 points: one
// group of 192 threads, 2 CTAs per SM).  CTA (blockIdx.x, blockIdx.y) runs ring
// rings[blockIdx.x] for its group of maps.
template <typename T, int KIND>
constexpr int ring_kernel_ctas() { return KIND ? 2 : ring_min_ctas<T>(); }
template <int KIND>
HPX_HD constexpr int ring_kernel_threads() { return KIND == 2 ? 192 : 256; }

// One CTA per (ring t, group of maps): map[b][ring t] -> F[b][foff_t + m]
template <typename T, int KIND>
__global__ void __launch_bounds__(ring_kernel_threads<KIND>(), ring_kernel_ctas<T, KIND>())
    k_ring_fwd(const T* __restrict__ map, int nmaps, int maps_per_cta, T* __restrict__ F, int64_t Ftot, Geom geo,
               const RingPair* __restrict__ pairs, const int* __restrict__ rings, const cplx<T>* __restrict__ rtab,
               int rslot, const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
               unsigned* __restrict__ fmax) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = geo.NP, R = geo.R;
    const int t = rings[blockIdx.x];
    const bool south = t >= NP;
    const int pr = south ? R - 1 - t : t;
    const RingPair rp = pairs[pr];
    PhaseTab<T> E, tw;
    cplx<T>* bufs = ring_tables<KIND>(smem_raw, rp, rtab + (size_t)pr * rslot, E, tw);
    const cplx<T>* Gs = nullptr;
    const cplx<T>* cs = nullptr;
    if constexpr (KIND > 0) bufs = ring_bluestein_tables<KIND>(bufs, rp, gtab, chirp, Gs, cs);
    __syncthreads();
    const int tpf = rp.tpf, S = blockDim.x / tpf, g = threadIdx.x / tpf, lt = threadIdx.x % tpf;
    const int P = ring_fft_len_k<KIND>(rp);
    const int PL = padded_len(P);
    cplx<T>* buf = bufs + (size_t)g * 2 * PL;
    cplx<T>* buf2 = buf + PL;
    const int64_t start = south ? rp.start_s : rp.start_n;
    const int64_t foff = south ? rp.foff_s : rp.foff_n;
    const int shift = south ? rp.shift_s : rp.shift_n;
    const int64_t np = geo.npix;
    const int b0 = blockIdx.y * maps_per_cta;
    const int b1 = min(b0 + maps_per_cta, nmaps);
    // (bounds-checked builds) the CTA's first and last maps' ring and spectrum
    if (b1 > b0 && !(HPX_INB(b0 * np + start, kExtMap, 1) && HPX_INB((b1 - 1) * np + start + 2 * rp.h - 1, kExtMap, 1) &&
                     HPX_INB(2 * ((int64_t)(b1 - 1) * Ftot + foff + rp.mt) - 1, kExtF, 2)))
        return;
    cplx<T>* cur = buf;
    cplx<T>* other = buf2;
    if (b0 + g < b1) ring_load_async(cur, map + (int64_t)(b0 + g) * np + start, rp.h, lt, tpf);
    for (int b = b0 + g; b < b1; b += S) {
        auto load_next = [&](cplx<T>* dst) {
            if (b + S < b1) ring_load_async(dst, map + (int64_t)(b + S) * np + start, rp.h, lt, tpf);
        };
        const T mx = ring_forward<KIND>(cur, other, shift, F + 2 * ((int64_t)b * Ftot + foff), rp, tw, Gs, cs, E, lt,
                                        tpf, g, load_next);
        if (fmax) {
            // per-map max |F| (scale of the FP16 operands); a group is whole warps
            float v = (float)mx;
#pragma unroll
            for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            if ((threadIdx.x & 31) == 0 && v > 0.f) atomicMax(fmax + b, __float_as_uint(v));
        }
    }
}

// One CTA per (ring t, group of maps): F[b][foff_t + m] -> map[b][ring t]
// (ref != nullptr: write ref - synthesis)
template <typename T, int KIND>
__global__ void __launch_bounds__(ring_kernel_threads<KIND>(), ring_kernel_ctas<T, KIND>())
    k_ring_inv(const T* __restrict__ F, int64_t Ftot, T* __restrict__ map, int nmaps, int maps_per_cta, Geom geo,
               const RingPair* __restrict__ pairs, const int* __restrict__ rings, const cplx<T>* __restrict__ rtab,
               int rslot, const cplx<T>* __restrict__ gtab, const cplx<T>* __restrict__ chirp,
               const T* __restrict__ ref) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = geo.NP, R = geo.R;
    const int t = rings[blockIdx.x];
    const bool south = t >= NP;
    const int pr = south ? R - 1 - t : t;
    const RingPair rp = pairs[pr];
    PhaseTab<T> E, tw;
    cplx<T>* bufs = ring_tables<KIND>(smem_raw, rp, rtab + (size_t)pr * rslot, E, tw);
    const cplx<T>* Gs = nullptr;
    const cplx<T>* cs = nullptr;
    if constexpr (KIND > 0) bufs = ring_bluestein_tables<KIND>(bufs, rp, gtab, chirp, Gs, cs);
    __syncthreads();
    const int tpf = rp.tpf, S = blockDim.x / tpf, g = threadIdx.x / tpf, lt = threadIdx.x % tpf;
    const int P = ring_fft_len_k<KIND>(rp);
    const int PL = padded_len(P);
    cplx<T>* buf = bufs + (size_t)g * 2 * PL;
    cplx<T>* buf2 = buf + PL;
    const int64_t start = south ? rp.start_s : rp.start_n;
    const int64_t foff = south ? rp.foff_s : rp.foff_n;
    const int shift = south ? rp.shift_s : rp.shift_n;
    const int64_t np = geo.npix;
    const int b0 = blockIdx.y * maps_per_cta;
    const int b1 = min(b0 + maps_per_cta, nmaps);
    if (b1 > b0 && !(HPX_INB(b0 * np + start, kExtMap, 3) && HPX_INB((b1 - 1) * np + start + 2 * rp.h - 1, kExtMap, 3) &&
                     HPX_INB(2 * ((int64_t)(b1 - 1) * Ftot + foff + rp.mt) - 1, kExtF, 4)))
        return;
    cplx<T>* cur = buf;
    cplx<T>* other = buf2;
    auto spec = [&](int bb) { return (const cplx<T>*)(F + 2 * ((int64_t)bb * Ftot + foff)); };
    if (b0 + g < b1) spec_load_async(cur, spec(b0 + g), rp.mt, lt, tpf);
    for (int b = b0 + g; b < b1; b += S) {
        auto load_next = [&](cplx<T>* dst) {
            if (b + S < b1) spec_load_async(dst, spec(b + S), rp.mt, lt, tpf);
        };
        ring_inverse<KIND>(cur, other, shift, map + (int64_t)b * np + start,
                           ref ? ref + (int64_t)b * np + start : nullptr, rp, tw, Gs, cs, E, lt, tpf, g, load_next);
    }
}

// Per-map max |a| over the coefficients the synthesis uses, a[b][l][m] for
// m <= l (complex, 8-byte aligned): atomicMax of the float bits into out[b]
// (out zeroed by the caller).  Grid (ceil(L/8), maps); warp w scans row
// l = 8 blockIdx.x + w.
__global__ void __launch_bounds__(256) k_alm_maxabs(const float* __restrict__ alm, int L, int M,
                                                    unsigned* __restrict__ out) {
    const int b = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int l = blockIdx.x * 8 + warp;
    float v = 0.f;
    if (l < L) {
        const int n = min(l + 1, M);
        const float2* row = (const float2*)(alm + 2 * (((int64_t)b * L + l) * M));
        int m = lane;
        for (; m + 96 < n; m += 128) {
            const float2 q0 = row[m], q1 = row[m + 32], q2 = row[m + 64], q3 = row[m + 96];
            v = fmaxf(v, fmaxf(fmaxf(fabsf(q0.x), fabsf(q0.y)), fmaxf(fabsf(q1.x), fabsf(q1.y))));
            v = fmaxf(v, fmaxf(fmaxf(fabsf(q2.x), fabsf(q2.y)), fmaxf(fabsf(q3.x), fabsf(q3.y))));
        }
        for (; m < n; m += 32) v = fmaxf(v, fmaxf(fabsf(row[m].x), fabsf(row[m].y)));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ float red[8];
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) v = fmaxf(v, red[w]);
        if (v > 0.f) atomicMax(out + b, __float_as_uint(v));
    }
}

// Fold ring spectra into the m-major Legendre operand:
//   S = c (F_t + F_t'),  D = c (F_t - F_t')   (equator: S = c F_t, D = 0)
// with c = w_t (analysis) or c_m = 2, 1 at m = 0 and m = nphi/2 (adjoint of synthesis).
// Output spec[m][par][p][col] in T, or hi/lo pairs xh/xl (mixed plans): bf16,
// or, with fmax given, fp16 of the values times 2^e(map), e from the map's
// max |F| (recorded by k_ring_fwd) times the bound wb on |c| (F_t + F_t').
// CTA per (block of 32 orders, ring pair); the transpose goes through shared memory.
template <typename T>
constexpr int fold_mb() { return sizeof(T) == 4 ? 32 : 16; }

template <typename T>
__global__ void __launch_bounds__(256) k_fold(const T* __restrict__ F, int64_t Ftot, int nmaps, Geom geo,
                                              const RingPair* __restrict__ pairs, int adjoint, T* __restrict__ spec,
                                              int C, uint32_t* __restrict__ xh, uint32_t* __restrict__ xl,
                                              const unsigned* __restrict__ fmax, float wb) {
    constexpr int MB = fold_mb<T>();
    constexpr int NL = 64 * MB / 256;  // elements per thread (the kernel runs 256 threads)
    __shared__ cplx<T> tn[64][MB + 1];
    __shared__ cplx<T> ts[64][MB + 1];
    __shared__ float s_sc[64];
    const int NP = geo.NP;
    const int m0 = blockIdx.x * MB, p = blockIdx.y, bz = blockIdx.z * 64;
    const RingPair rp = pairs[p];
    if (m0 >= rp.mt) return;
    const int tid = threadIdx.x;
    // all loads of the thread are issued before the first shared-memory store
    cplx<T> vn[NL], vs[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = tid + 256 * k;
        const int b = bz + i / MB, m = m0 + i % MB;
        vn[k] = {(T)0, (T)0};
        vs[k] = {(T)0, (T)0};
        if (b < nmaps && m < rp.mt) {
            if (HPX_INB(2 * ((int64_t)b * Ftot + rp.foff_n + m) + 1, kExtF, 5))
                vn[k] = *(const cplx<T>*)(F + 2 * ((int64_t)b * Ftot + rp.foff_n + m));
            if (rp.has_south && HPX_INB(2 * ((int64_t)b * Ftot + rp.foff_s + m) + 1, kExtF, 5))
                vs[k] = *(const cplx<T>*)(F + 2 * ((int64_t)b * Ftot + rp.foff_s + m));
        }
    }
    if (xh && fmax && tid < 64) {
        // FP16 operands scaled by 2^e(map); |S|, |D| <= wb * max|F|
        const int b = bz + tid;
        s_sc[tid] = tc::pow2f(tc::f16_scale_exp(__uint_as_float(b < nmaps ? fmax[b] : 0u) * wb));
    }
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = tid + 256 * k;
        tn[i / MB][i % MB] = vn[k];
        ts[i / MB][i % MB] = vs[k];
    }
    __syncthreads();
    // each thread: one (m, map) pair -> S and D
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = tid + 256 * k;
        const int mm = i >> 6, bl = i & 63, b = bz + bl, m = m0 + mm;
        if (m >= rp.mt || 2 * b >= C) continue;
        const T wk = adjoint ? ((m == 0 || m == rp.h) ? (T)1 : (T)2) : (T)rp.w;
        const cplx<T> a = tn[bl][mm], c = ts[bl][mm];
        cplx<T> S, D;
        if (rp.has_south) {
            S = cscale(cadd(a, c), wk);
            D = cscale(csub(a, c), wk);
        } else {
            S = cscale(a, wk);
            D = {(T)0, (T)0};
        }
        const int64_t i0 = (((int64_t)m * 2 + 0) * NP + p) * C + 2 * b;
        const int64_t i1 = (((int64_t)m * 2 + 1) * NP + p) * C + 2 * b;
        if (xh ? !(HPX_INB(i0 >> 1, kExtOperX, 6) && HPX_INB(i1 >> 1, kExtOperX, 6))
               : !(HPX_INB(i0 + 1, kExtSpec, 6) && HPX_INB(i1 + 1, kExtSpec, 6)))
            continue;
        if (xh && fmax) {
            const float sc = s_sc[bl];
            uint16_t h0, l0, h1, l1;
            tc::split_f16((float)S.re * sc, h0, l0);
            tc::split_f16((float)S.im * sc, h1, l1);
            xh[i0 >> 1] = (uint32_t)h0 | ((uint32_t)h1 << 16);
            xl[i0 >> 1] = (uint32_t)l0 | ((uint32_t)l1 << 16);
            tc::split_f16((float)D.re * sc, h0, l0);
            tc::split_f16((float)D.im * sc, h1, l1);
            xh[i1 >> 1] = (uint32_t)h0 | ((uint32_t)h1 << 16);
            xl[i1 >> 1] = (uint32_t)l0 | ((uint32_t)l1 << 16);
        } else if (xh) {
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
}

// Unfold the synthesis output spec[m][par][p][col] (E = even, O = odd degrees)
// into ring spectra F_t = sc (E + O), F_t' = sc (E - O), with sc = 1, or for
// the adjoint of analysis sc = w_t (m = 0, nphi/2) and w_t/2 otherwise.
template <typename T>
__global__ void __launch_bounds__(256) k_unfold(const T* __restrict__ spec, int C, int nmaps, Geom geo,
                                                const RingPair* __restrict__ pairs, int adjoint, T* __restrict__ F,
                                                int64_t Ftot) {
    constexpr int MB = fold_mb<T>();
    constexpr int NL = 64 * MB / 256;  // elements per thread (the kernel runs 256 threads)
    __shared__ cplx<T> te[MB][65];
    __shared__ cplx<T> to[MB][65];
    const int NP = geo.NP;
    const int m0 = blockIdx.x * MB, p = blockIdx.y, bz = blockIdx.z * 64;
    const RingPair rp = pairs[p];
    if (m0 >= rp.mt) return;
    const int tid = threadIdx.x;
    // all loads of the thread are issued before the first shared-memory store
    cplx<T> ve[NL], vo[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = tid + 256 * k;
        const int mm = i >> 6, bl = i & 63, b = bz + bl, m = m0 + mm;
        ve[k] = {(T)0, (T)0};
        vo[k] = {(T)0, (T)0};
        if (m < rp.mt && 2 * b < C && HPX_INB((((int64_t)m * 2 + 1) * NP + p) * C + 2 * b + 1, kExtSpec, 7)) {
            ve[k] = *(const cplx<T>*)(spec + (((int64_t)m * 2 + 0) * NP + p) * C + 2 * b);
            vo[k] = *(const cplx<T>*)(spec + (((int64_t)m * 2 + 1) * NP + p) * C + 2 * b);
        }
    }
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = tid + 256 * k;
        te[i >> 6][i & 63] = ve[k];
        to[i >> 6][i & 63] = vo[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const int i = tid + 256 * k;
        const int bl = i / MB, mm = i % MB, b = bz + bl, m = m0 + mm;
        if (b >= nmaps || m >= rp.mt) continue;
        T sc = (T)1;
        if (adjoint) sc = (m == 0 || m == rp.h) ? (T)rp.w : (T)(0.5 * rp.w);
        const cplx<T> e = te[mm][bl], o = to[mm][bl];
        if (HPX_INB(2 * ((int64_t)b * Ftot + rp.foff_n + m) + 1, kExtF, 8))
            *(cplx<T>*)(F + 2 * ((int64_t)b * Ftot + rp.foff_n + m)) = cscale(cadd(e, o), sc);
        if (rp.has_south && HPX_INB(2 * ((int64_t)b * Ftot + rp.foff_s + m) + 1, kExtF, 8))
            *(cplx<T>*)(F + 2 * ((int64_t)b * Ftot + rp.foff_s + m)) = cscale(csub(e, o), sc);
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

// twiddles e^{-2 pi i q/P} read straight from the plan's FP64 table for Pmax
struct StrideTw64 {
    const cplx<double>* p;
    int stride;
    __device__ __forceinline__ cplx<double> operator()(int q) const { return p[q * stride]; }
};

// Bluestein tables per ring pair (FP64, rounded to T):
//   chirp[j] = e^{-i pi j^2/h}, j < h  (phase from the integer j^2 mod 2h)
//   G = FFT_P(g) / P in natural order, g_j = e^{+i pi j^2/h} for |j| < h (wrapped)
// The FP64 FFT runs in shared memory, or (GLOBAL, when two FP64 buffers of
// the largest P do not fit there: nside 2048) in a global scratch of
// 2 padded_len(Pmax) elements per block.  Plan creation only.
template <typename T, bool GLOBAL>
__global__ void __launch_bounds__(256) k_chirp_spectra(const RingPair* __restrict__ pairs,
                                                       const cplx<double>* __restrict__ tw64, int logPmax,
                                                       cplx<T>* __restrict__ gtab, cplx<T>* __restrict__ chirp,
                                                       cplx<double>* __restrict__ scratch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const RingPair rp = pairs[blockIdx.x];
    if (rp.logh >= 0) return;
    if (GLOBAL && rp.rad3) return;  // the plan gives lengths 3 * 2^K only to shared-memory builds
    const int P = ring_fft_len(rp), h = rp.h;
    cplx<double>* buf;
    cplx<double>* buf2;
    cplx<double>* twP = nullptr;
    if constexpr (GLOBAL) {
        buf = scratch + (size_t)blockIdx.x * 2 * padded_len(1 << logPmax);
        buf2 = buf + padded_len(1 << logPmax);
    } else {
        buf = (cplx<double>*)smem_raw;
        buf2 = buf + padded_len(P);
        twP = buf2 + padded_len(P);
        if (rp.rad3) {
            // twiddles of the length 3 * 2^K, in FP64
            for (int q = threadIdx.x; q < P / 2; q += blockDim.x) {
                double sn, cs;
                sincospi(-2.0 * (double)q / (double)P, &sn, &cs);
                twP[padi(q)] = {cs, sn};
            }
        } else {
            load_twiddles(twP, rp.logP, tw64, logPmax);
        }
    }
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        const int d = j < h ? j : (j > P - h ? P - j : -1);
        cplx<double> v = {0.0, 0.0};
        if (d >= 0) {
            const long long q = ((long long)d * d) % (2 * h);
            double s, c;
            sincospi((double)q / (double)h, &s, &c);
            v = {c, s};
        }
        buf[padi(j)] = v;
        if (j < h) chirp[rp.gtab_off + j] = {(T)v.re, (T)(-v.im)};
    }
    __syncthreads();
    cplx<double>* r;
    if (!GLOBAL && rp.rad3) {
        // one group of fft_tpf(P) threads (whole warps) runs the transform
        const int tpf = fft_tpf(P);
        IdentityMap id;
        if ((int)threadIdx.x < tpf) fft_ring3<double, false>(buf, buf2, rp.logP, FullTw<double>{twP}, threadIdx.x, 0, id, id);
        __syncthreads();
        r = (fft3_passes(rp.logP) & 1) ? buf2 : buf;
    } else if constexpr (GLOBAL)
        r = fft_pow2<double, false>(buf, buf2, rp.logP, StrideTw64{tw64, 1 << (logPmax - rp.logP)}, threadIdx.x,
                                    blockDim.x, 0, IdentityMap{}, IdentityMap{});
    else
        r = fft_pow2<double, false>(buf, buf2, rp.logP, FullTw<double>{twP}, threadIdx.x, blockDim.x, 0, IdentityMap{},
                                    IdentityMap{});
    const double inv = 1.0 / (double)P;
    for (int j = threadIdx.x; j < P; j += blockDim.x) {
        gtab[rp.gtab_off + j] = {(T)(r[padi(j)].re * inv), (T)(r[padi(j)].im * inv)};
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
