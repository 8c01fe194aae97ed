// Associated-Legendre recurrence and the SIMT Legendre contractions.
//
// Pbar_l^m(x) is the orthonormal associated Legendre function without the
// Condon-Shortley phase, as built by legpoly / legpoly_torch
// (cuhpx/sht_tools.py:192-256):
//   Pbar_m^m     = sqrt((2m+1)/(2m)) sin(theta) Pbar_{m-1}^{m-1},  Pbar_0^0 = 1/sqrt(4 pi)
//   Pbar_{m+1}^m = sqrt(2m+3) x Pbar_m^m
//   Pbar_l^m     = a_lm x Pbar_{l-1}^m - b_lm Pbar_{l-2}^m
// The reference tabulates it densely ([M, L, rings], 68.6 GB in FP32 at
// nside=1024, L=M=2047) and contracts with torch.einsum
// (cuhpx/hpx_sht.py:557, 599).  Here nothing is tabulated: the plan stores,
// per (m, north ring), the first degree l_s whose value is above 2^-600 and the
// FP64 pair (Pbar_{l_s}, Pbar_{l_s+1}) -- found by an exponent-scaled FP64
// recurrence so that the high-m polar seeds never underflow -- and every
// contraction kernel runs the recurrence in FP64 on the fly from there.  Values
// with l < l_s are below 2^-600 and are taken as 0.
//
// North/south symmetry: Pbar_l^m(-x) = (-1)^{l+m} Pbar_l^m(x), so a degree l
// with l-m even contracts against S = w(F_t + F_t') and l-m odd against
// D = w(F_t - F_t'); the sums run over the 2*nside north rings only.
#pragma once

#include "ring_fft.cuh"

namespace hpx {

// Three-term coefficients with the operation order of cuhpx/sht_tools.py:250-251
// (IEEE double division and square root, so they equal the reference's bitwise).
__device__ __forceinline__ double rec_a(int l, int m) {
    double dl = l, dm = m;
    return sqrt((2.0 * dl - 1.0) / (dl - dm) * (2.0 * dl + 1.0) / (dl + dm));
}
__device__ __forceinline__ double rec_b(int l, int m) {
    double dl = l, dm = m;
    return sqrt((dl + dm - 1.0) / (dl - dm) * (2.0 * dl + 1.0) / (2.0 * dl - 3.0) * (dl - dm - 1.0) / (dl + dm));
}

// Values below 2^-1000 (still normal doubles) are treated as zero.
constexpr double kSeedLog2Floor = -1000.0;

// Start values of the recurrence for (m, north ring p); see file comment.
// logc[m] = log2(Pbar_m^m / sin^m(theta)) = log2(1/sqrt(4pi)) + 0.5 sum_k log2((2k+1)/(2k)).
__global__ void k_legendre_start(int M, int L, Geom geo, const RingPair* __restrict__ pairs,
                                 const double* __restrict__ logc, int* __restrict__ lstart,
                                 double2* __restrict__ pstart) {
    const int NP = geo.NP;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)M * NP) return;
    const int m = (int)(idx / NP), p = (int)(idx % NP);
    int ls = L;
    double2 ps = make_double2(0.0, 0.0);
    const double s2 = pairs[p].s2;
    // rings from the first one that carries order m - 1: the spin-1 transforms
    // of order m - 1 read Pbar^m there (the scalar ones start at first_ring(m))
    if (m < L && p >= geo.first_ring(m > 0 ? m - 1 : 0) && (m == 0 || s2 > 0.0)) {  // poles carry m = 0 only
        const double x = pairs[p].z;
        const double lg = m == 0 ? logc[0] : logc[m] + 0.5 * (double)m * log2(s2);
        // scaled pair: value = mant * 2^E
        double E = floor(lg);
        double q0 = exp2(lg - E);
        double q1 = sqrt(2.0 * m + 3.0) * x * q0;
        int l = m;
        while (l < L) {
            if (q0 != 0.0 && log2(fabs(q0)) + E >= kSeedLog2Floor) {
                ls = l;
                ps = make_double2(ldexp(q0, (int)E), ldexp(q1, (int)E));
                break;
            }
            // advance one degree: q2 = a x q1 - b q0 at degree l+2
            double q2 = rec_a(l + 2, m) * x * q1 - rec_b(l + 2, m) * q0;
            q0 = q1;
            q1 = q2;
            ++l;
            double mx = fmax(fabs(q0), fabs(q1));
            if (mx > 0x1p400) {
                q0 = ldexp(q0, -400);
                q1 = ldexp(q1, -400);
                E += 400.0;
            }
        }
    }
    lstart[idx] = ls;
    pstart[idx] = ps;
}

// One FP64 recurrence step for degree l given (p1, p2) = (P_{l-1}, P_{l-2}).
__device__ __forceinline__ double leg_step(int l, int ls, double2 ps, double a, double b, double x, double p1,
                                           double p2) {
    double v = a * x * p1 - b * p2;
    v = (l == ls) ? ps.x : v;
    v = (l == ls + 1) ? ps.y : v;
    v = (l < ls) ? 0.0 : v;
    return v;
}

// Recurrence coefficients a_lm, b_lm for every (m, m+2 <= l < L), shared by the
// seed precompute and all contraction kernels: coef[m * Lpad + l] = (a, b).
// Rows are padded to Lpad = L + kCoefPad with zeros, so a recurrence run past
// l = L-1 yields exact zeros without a branch.
constexpr int kCoefPad = 256;
__global__ void k_legendre_coef(int M, int L, int Lpad, double2* __restrict__ coef) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)M * Lpad) return;
    const int m = (int)(idx / Lpad), l = (int)(idx % Lpad);
    coef[idx] = (l >= m + 2 && l < L) ? make_double2(rec_a(l, m), rec_b(l, m)) : make_double2(0.0, 0.0);
}

// Degree-block seeds: for every (m, block j, north ring p) the FP64 pair
// (Pbar_{l0}, Pbar_{l0+1}) at l0 = m + j*kSeedBlock, so that any block of
// degrees can be generated independently.  Thread per (m, ring).
constexpr int kSeedBlock = 64;

__host__ __device__ inline int seed_blocks(int L) { return (L + kSeedBlock - 1) / kSeedBlock; }

__global__ void k_legendre_seeds(int M, int L, int Lpad, Geom geo, const RingPair* __restrict__ pairs,
                                 const int* __restrict__ lstart, const double2* __restrict__ pstart,
                                 const double2* __restrict__ coef, double2* __restrict__ seeds) {
    const int NP = geo.NP;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)M * NP) return;
    const int m = (int)(idx / NP), p = (int)(idx % NP);
    const int nb = seed_blocks(L);
    double2* out = seeds + (int64_t)m * nb * NP + p;
    if (m >= L) return;
    const int ls = lstart[idx];
    const double2 ps = pstart[idx];
    const double x = pairs[p].z;
    double p1 = 0.0, p2 = 0.0;
    const double2* cm = coef + (int64_t)m * Lpad;
    for (int l = m; l < L; ++l) {
        double2 ab = l >= m + 2 ? cm[l] : make_double2(0.0, 0.0);
        double v = leg_step(l, ls, ps, ab.x, ab.y, x, p1, p2);
        const int off = (l - m) % kSeedBlock;
        const int j = (l - m) / kSeedBlock;
        if (off == 0) out[(int64_t)j * NP] = make_double2(v, 0.0);
        else if (off == 1) out[(int64_t)j * NP].y = v;
        p2 = p1;
        p1 = v;
    }
}

// Block-normalised recurrence used by the tensor-core producers.  Inside the
// 64-degree block that starts at l0b (seed pair P_{l0b}, P_{l0b+1}) write
// P_l = c_l q_l with c_{l0b} = c_{l0b+1} = 1 and c_l = b_l c_{l-2}; then
//   q_l = alpha_l x q_{l-1} - q_{l-2},   alpha_l = a_l c_{l-1} / c_l,
// so each step is one FP64 multiply off the dependency chain plus one FMA on
// it, and the scale c_l is applied after rounding to FP32.
struct __align__(16) AlphaC {
    double alpha;
    float c;
    float pad;
};

__global__ void k_legendre_alpha(int M, int L, int Lpad, const double2* __restrict__ coef, AlphaC* __restrict__ out) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // one thread per (m, block)
    const int nb = seed_blocks(L);
    if (idx >= (int64_t)M * nb) return;
    const int m = (int)(idx / nb), j = (int)(idx % nb);
    const int l0b = m + j * kSeedBlock;
    AlphaC* o = out + (int64_t)m * Lpad;
    if (l0b >= L && j > 0) return;
    double cm2 = 1.0, cm1 = 1.0;  // c_{l-2}, c_{l-1}
    for (int i = 0; i < kSeedBlock; ++i) {
        const int l = l0b + i;
        if (l >= Lpad) break;
        AlphaC v;
        v.pad = 0.f;
        if (i < 2 || l >= L || l < m + 2) {
            v.alpha = 0.0;
            v.c = (l < L && i < 2) ? 1.f : 0.f;
            const double c = (i < 2) ? 1.0 : 0.0;
            cm2 = cm1;
            cm1 = c;
        } else {
            const double2 ab = coef[(int64_t)m * Lpad + l];
            const double c = ab.y * cm2;
            v.alpha = ab.x * cm1 / c;
            v.c = (float)c;
            cm2 = cm1;
            cm1 = c;
        }
        o[l] = v;
    }
}

// ------------------------------------------------------------ forward (analysis)
// alm[b][l][m] = sum_{p >= t0(m)} Pbar_l^m(x_p) X[m][(l-m)&1][p][2b..2b+1]
// One CTA per (m, degree block of 64, column tile of 128 = 64 maps).  Each
// pass generates Pbar for RB rings x 64 degrees from the FP64 block seeds
// (one ring per thread), then contracts it with X chunks that cp.async
// double-buffers through shared memory.
template <typename T>
struct FwdCfg {
    static constexpr int LT = kSeedBlock;               // degrees per tile (32 even, 32 odd)
    static constexpr int CT = 128;                      // columns per CTA
    static constexpr int RB = sizeof(T) == 4 ? 256 : 128;  // rings generated per pass
    static constexpr int KC = 16;                       // rings per staged X chunk
    static constexpr int LTP = LT + 16 / sizeof(T);     // padded P row
};

template <typename T>
__host__ __device__ constexpr size_t fwd_smem_bytes() {
    using C = FwdCfg<T>;
    return (size_t)C::LT * sizeof(double2) + (size_t)C::RB * C::LTP * sizeof(T) +
           (size_t)2 * C::KC * 2 * C::CT * sizeof(T) + 64;
}


template <typename T>
__global__ void __launch_bounds__(256) k_leg_fwd_simt(const T* __restrict__ spec, int C, int nmaps,
                                                      T* __restrict__ alm, int L, int M, Geom geo,
                                                      const RingPair* __restrict__ pairs,
                                                      const int* __restrict__ lstart,
                                                      const double2* __restrict__ pstart,
                                                      const double2* __restrict__ coef, int Lpad,
                                                      const double2* __restrict__ seeds,
                                                      const int2* __restrict__ tiles, int accumulate) {
    using Cfg = FwdCfg<T>;
    constexpr int LT = Cfg::LT, CT = Cfg::CT, RB = Cfg::RB, KC = Cfg::KC, LTP = Cfg::LTP;
    constexpr int VPR = CT * sizeof(T) / 16;  // 16-byte vectors per staged row
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = geo.NP;
    const int2 tl = tiles[blockIdx.x];
    const int m = tl.x, jb = tl.y;
    const int l0 = m + jb * LT;
    const int c0 = blockIdx.y * CT;
    const int tid = threadIdx.x;
    double2* cf = (double2*)smem_raw;
    T* Pt = (T*)(cf + LT);
    T* Xs = Pt + RB * LTP;  // [2][KC][2][CT]

    const int t0 = geo.first_ring(m);
    const int K = NP - t0;
    const int nbk = seed_blocks(L);

    // zero the l < m triangle once per (m, column tile)
    if (!accumulate && jb == 0) {
        for (int i = tid; i < min(m, L) * (CT / 2); i += blockDim.x) {
            const int l = i / (CT / 2), b = c0 / 2 + i % (CT / 2);
            if (b < nmaps) *(cplx<T>*)(alm + 2 * (((int64_t)b * L + l) * M + m)) = {(T)0, (T)0};
        }
    }
    if (m >= L) return;
    for (int i = tid; i < LT; i += blockDim.x) {
        const int l = l0 + i;
        cf[i] = (l < L && l >= m + 2) ? coef[(int64_t)m * Lpad + l] : make_double2(0.0, 0.0);
    }

    const int tx = tid & 15, ty = tid >> 4;
    const int par = ty >> 3;        // 0: l-m even (S), 1: odd (D)
    const int jrow = (ty & 7) * 4;  // 4 rows of this parity
    const int cA = tx * 4, cB = 64 + tx * 4;
    T acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[i][c] = (T)0;

    auto stage = [&](int buf, int rbase, int nr) {
        T* dst = Xs + buf * (KC * 2 * CT);
        for (int i = tid; i < KC * 2 * VPR; i += blockDim.x) {
            const int v = i % VPR, row = i / VPR;
            const int q = row >> 1, pr = row & 1;
            const int r = rbase + q;
            const int c = c0 + v * (16 / (int)sizeof(T));
            const bool ok = q < nr && c < C;
            const T* src = spec + (((int64_t)m * 2 + pr) * NP + t0 + (ok ? r : 0)) * C + (ok ? c : 0);
            cp_async16(dst + row * CT + v * (16 / sizeof(T)), src, ok);
        }
        cp_async_commit();
    };

    for (int rb = 0; rb < K; rb += RB) {
        __syncthreads();  // coefficient table ready / previous pass done with Pt
        // --- generate Pbar for rings rb.., degrees l0..l0+LT from the block seeds
        if (tid < RB) {
            const int r = rb + tid;
            T* prow = Pt + tid * LTP;
            if (r < K) {
                const int p = t0 + r;
                const int64_t mi = (int64_t)m * NP + p;
                const double x = pairs[p].z;
                const int ls = lstart[mi];
                const double2 sd = seeds[((int64_t)m * nbk + jb) * NP + p];
                double p2 = 0.0, p1 = 0.0;
                if (ls <= l0) {
                    // fast path: the seed pair is exact
                    prow[0] = (T)sd.x;
                    if (LT > 1) prow[LT / 2] = (T)sd.y;
                    p2 = sd.x;
                    p1 = sd.y;
#pragma unroll 4
                    for (int i = 2; i < LT; ++i) {
                        const double2 ab = cf[i];
                        const double v = (l0 + i < L) ? ab.x * x * p1 - ab.y * p2 : 0.0;
                        p2 = p1;
                        p1 = v;
                        prow[(i & 1) * (LT / 2) + (i >> 1)] = (T)v;
                    }
                } else {
                    const double2 ps = (ls < l0 + LT && ls < L) ? pstart[mi] : make_double2(0.0, 0.0);
                    for (int i = 0; i < LT; ++i) {
                        const int l = l0 + i;
                        const double2 ab = cf[i];
                        const double v = (l < L) ? leg_step(l, ls, ps, ab.x, ab.y, x, p1, p2) : 0.0;
                        p2 = p1;
                        p1 = v;
                        prow[(i & 1) * (LT / 2) + (i >> 1)] = (T)v;
                    }
                }
            } else {
                for (int i = 0; i < LT; ++i) prow[i] = (T)0;
            }
        }
        const int rend = min(RB, K - rb);
        const int nch = (rend + KC - 1) / KC;
        stage(0, rb, min(KC, rend));
        __syncthreads();
        for (int ch = 0; ch < nch; ++ch) {
            if (ch + 1 < nch) {
                stage((ch + 1) & 1, rb + (ch + 1) * KC, min(KC, rend - (ch + 1) * KC));
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            const T* xb = Xs + (ch & 1) * (KC * 2 * CT);
            const int qn = min(KC, rend - ch * KC);
            const T* pbase = Pt + (ch * KC) * LTP + par * (LT / 2) + jrow;
#pragma unroll 4
            for (int q = 0; q < qn; ++q) {
                const T* pr = pbase + q * LTP;
                T pv[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) pv[i] = pr[i];
                const T* xr = xb + (q * 2 + par) * CT;
                T xv[8];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    xv[c] = xr[cA + c];
                    xv[4 + c] = xr[cB + c];
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int c = 0; c < 8; ++c) acc[i][c] = fma(pv[i], xv[c], acc[i][c]);
            }
            __syncthreads();
        }
    }
    // --- write this tile
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int l = l0 + 2 * (jrow + i) + par;
        if (l >= L) continue;
#pragma unroll
        for (int cc = 0; cc < 8; cc += 2) {
            const int c = c0 + (cc < 4 ? cA + cc : cB + cc - 4);
            const int b = c >> 1;
            if (b < nmaps && HPX_INB(2 * (((int64_t)b * L + l) * M + m) + 1, kExtAlm, 15)) {
                cplx<T>* dst = (cplx<T>*)(alm + 2 * (((int64_t)b * L + l) * M + m));
                cplx<T> v = {acc[i][cc], acc[i][cc + 1]};
                if (accumulate) v = cadd(*dst, v);
                *dst = v;
            }
        }
    }
}

// ------------------------------------------------------------ inverse (synthesis)
// E[m][p][c] = sum_{l-m even} Pbar_l^m(x_p) A[m][l][c],  O = sum over l-m odd,
// written to spec[m][0][p][c] and spec[m][1][p][c].  One CTA per (m, block of
// RBI rings, column tile); the FP64 recurrence of each ring runs in one thread.
template <typename T>
struct InvCfg {
    static constexpr int RBI = 64;  // rings per CTA
    static constexpr int CT = 128;  // columns per CTA
    static constexpr int LC = 32;   // degrees per staged chunk
    static constexpr int RBP = RBI + 16 / sizeof(T);
};

template <typename T>
__host__ __device__ constexpr size_t inv_smem_bytes(int L) {
    using C = InvCfg<T>;
    return (size_t)2 * L * sizeof(double) + (size_t)C::LC * C::RBP * sizeof(T) + (size_t)C::LC * C::CT * sizeof(T) + 64;
}

template <typename T>
__global__ void __launch_bounds__(256) k_leg_inv_simt(const T* __restrict__ almT, int C, T* __restrict__ spec, int L,
                                                      int M, Geom geo, const RingPair* __restrict__ pairs,
                                                      const int* __restrict__ lstart,
                                                      const double2* __restrict__ pstart,
                                                      const double2* __restrict__ coef, int Lpad,
                                                      const int2* __restrict__ work) {
    using Cfg = InvCfg<T>;
    constexpr int RBI = Cfg::RBI, CT = Cfg::CT, LC = Cfg::LC, RBP = Cfg::RBP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = geo.NP;
    const int2 wk = work[blockIdx.x];
    const int m = wk.x, rb = wk.y;
    const int c0 = blockIdx.y * CT;
    const int tid = threadIdx.x;
    double* coefA = (double*)smem_raw;
    double* coefB = coefA + L;
    T* Pt = (T*)(coefB + L);  // [LC][RBP], 16-byte aligned (2L doubles precede it)
    T* As = Pt + LC * RBP;                                          // [LC][CT]

    const int t0 = geo.first_ring(m);
    const int K = NP - t0;

    for (int l = m + 2 + tid; l < L; l += blockDim.x) {
        const double2 ab = coef[(int64_t)m * Lpad + l];
        coefA[l] = ab.x;
        coefB[l] = ab.y;
    }
    // generator state (threads tid < RBI own ring rb + tid)
    const int rg = rb + tid;
    const bool gen = tid < RBI && rg < K;
    double x = 0.0, p1 = 0.0, p2 = 0.0;
    int ls = L;
    double2 ps = make_double2(0.0, 0.0);
    if (gen) {
        x = pairs[t0 + rg].z;
        ls = lstart[(int64_t)m * NP + t0 + rg];
        if (ls < L) ps = pstart[(int64_t)m * NP + t0 + rg];
    }
    __syncthreads();

    const int tx = tid & 15, ty = tid >> 4;
    const int rrow = ty * 4;
    const int cA = tx * 4, cB = 64 + tx * 4;
    T accE[4][8], accO[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            accE[i][c] = (T)0;
            accO[i][c] = (T)0;
        }

    for (int l0 = m; l0 < L; l0 += LC) {
        if (tid < RBI) {
            for (int i = 0; i < LC; ++i) {
                const int l = l0 + i;
                double v = 0.0;
                if (gen && l < L) v = leg_step(l, ls, ps, l >= m + 2 ? coefA[l] : 0.0, l >= m + 2 ? coefB[l] : 0.0, x, p1, p2);
                p2 = p1;
                p1 = v;
                Pt[i * RBP + tid] = (T)v;
            }
        }
        for (int i = tid; i < LC * CT; i += blockDim.x) {
            const int c = i % CT, li = i / CT;
            const int l = l0 + li;
            T v = (T)0;
            if (l < L && c0 + c < C) v = almT[((int64_t)m * L + l) * C + c0 + c];
            As[li * CT + c] = v;
        }
        __syncthreads();
#pragma unroll 2
        for (int li = 0; li < LC; li += 2) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const T* pr = Pt + (li + h) * RBP + rrow;
                const T* ar = As + (li + h) * CT;
                T pv[4], av[8];
#pragma unroll
                for (int i = 0; i < 4; ++i) pv[i] = pr[i];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    av[c] = ar[cA + c];
                    av[4 + c] = ar[cB + c];
                }
                if (h == 0) {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int c = 0; c < 8; ++c) accE[i][c] = fma(pv[i], av[c], accE[i][c]);
                } else {
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int c = 0; c < 8; ++c) accO[i][c] = fma(pv[i], av[c], accO[i][c]);
                }
            }
        }
        __syncthreads();
    }
    // write E/O for rings of this CTA
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = rb + rrow + i;
        if (r >= K || !HPX_INB((((int64_t)m * 2 + 1) * NP + t0 + r) * C + c0 + min(CT, C - c0) - 1, kExtSpec, 16))
            continue;
        T* e = spec + (((int64_t)m * 2 + 0) * NP + t0 + r) * C + c0;
        T* o = spec + (((int64_t)m * 2 + 1) * NP + t0 + r) * C + c0;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int cc = c < 4 ? cA + c : cB + c - 4;
            if (c0 + cc < C) {
                e[cc] = accE[i][c];
                o[cc] = accO[i][c];
            }
        }
    }
}

}  // namespace hpx
