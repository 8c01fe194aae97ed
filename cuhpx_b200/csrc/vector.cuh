// Spin-1 (vector) Legendre contractions on CUDA cores, FP32 or FP64.
//
// cuHPX's VectorSHT / VectoriSHT (cuhpx/hpx_sht.py:286-444) transform a
// tangent field given as two real components [batch][2][npix] into
// spheroidal and toroidal coefficients [batch][2][L][M] with the table
// _precompute_dlegpoly (cuhpx/sht_tools.py:267-304), for 0 <= m <= l:
//   D0_l^m = 0.5 (sqrt((l+m)(l-m+1)) Pbar_l^{m-1} - sqrt((l-m)(l+m+1)) Pbar_l^{m+1})
//            (Pbar_l^{-1} := -Pbar_l^1, so D0_l^0 = -sqrt(l(l+1)) Pbar_l^1)
//   D1_l^m = 0.5 sqrt((2l+1)/(2l+3)) (sqrt((l-m+1)(l-m+2)) Pbar_{l+1}^{m-1}
//            + sqrt((l+m+1)(l+m+2)) Pbar_{l+1}^{m+1}),   D1_l^0 = 0
// times (-1)^m when csphase is set.  With the folded ring spectra x0, x1 of the
// two components (quadrature weights included) and nf_l = 1/(l(l+1)), nf_0 = 1:
//   S_lm = nf_l sum_t (D0 x0 - i D1 x1)       T_lm = nf_l sum_t (-D0 x1 - i D1 x0)
// and the synthesis of ring spectra (s, t) of the two components:
//   s_tm = sum_l (D0 S + i D1 T)              t_tm = sum_l (-D0 T + i D1 S).
// The reference tabulates D0, D1 densely ([2][M][L][rings], FP64) and runs
// eight einsums per call; here they are generated on the fly from FP64
// recurrences of orders m-1 and m+1, which the plan provides because the
// vector plan is built with L+1 degrees and M+1 orders.
//
// North/south symmetry: Pbar_l^m(-x) = (-1)^{l+m} Pbar_l^m(x), so D0 has the
// parity (-1)^{l+m+1} and D1 the parity (-1)^{l+m}: the analysis contracts D0
// with the fold of parity index (l-m+1)&1 and D1 with (l-m)&1 (S = w(F_t +
// F_t'), D = w(F_t - F_t')); the synthesis sums the terms whose south sign is +
// into E and the others into O, so that the scalar path's unfold (F_t = E + O,
// F_t' = E - O) and inverse ring FFTs finish the job.  The two components of
// every vector map travel through the ring stages as two consecutive maps.
#pragma once

#include "legendre.cuh"

namespace hpx {

// Running FP64 recurrence of one order o at one ring: value at degree d,
// stepping upward; degrees below o (and below the first significant degree)
// read as zero.
struct LegRun {
    int o, d, ls;
    double2 ps;
    double x, p1, p2;
    __device__ void init(int order, int m_end, int M, int64_t mi, const int* __restrict__ lstart,
                         const double2* __restrict__ pstart, double xv) {
        o = order;
        d = order;
        x = xv;
        p1 = p2 = 0.0;
        ls = (order < m_end) ? lstart[mi] : 0x7fffffff;
        ps = (order < m_end && ls < 0x7fffffff) ? pstart[mi] : make_double2(0.0, 0.0);
        (void)M;
    }
    // value at degree d, then d += 1
    __device__ double next(const double2* __restrict__ coef_o, int Lp) {
        double v = 0.0;
        if (d < Lp) {
            const double2 ab = d >= o + 2 ? coef_o[d] : make_double2(0.0, 0.0);
            v = leg_step(d, ls, ps, ab.x, ab.y, x, p1, p2);
        }
        p2 = p1;
        p1 = v;
        ++d;
        return v;
    }
};

// 0.5 sqrt(...) factors of D0 and D1 at (l, m)
__device__ __forceinline__ void vec_coefs(int l, int m, double& c1, double& c2, double& c3, double& c4) {
    const double dl = l, dm = m;
    c1 = 0.5 * sqrt((dl + dm) * (dl - dm + 1.0));
    c2 = 0.5 * sqrt((dl - dm) * (dl + dm + 1.0));
    const double h = 0.5 * sqrt((2.0 * dl + 1.0) / (2.0 * dl + 3.0));
    c3 = h * sqrt((dl - dm + 1.0) * (dl - dm + 2.0));
    c4 = h * sqrt((dl + dm + 1.0) * (dl + dm + 2.0));
}

// ------------------------------------------------------------ analysis
template <typename T>
struct VFwdCfg {
    static constexpr int LT = 32;   // degrees per tile
    static constexpr int CT = 64;   // columns per CTA: 16 vector maps x (2 components x re, im)
    static constexpr int RB = 128;  // rings generated per pass
    static constexpr int KC = 16;   // rings per staged spectrum chunk
};

template <typename T>
__host__ __device__ constexpr size_t vfwd_smem_bytes() {
    using C = VFwdCfg<T>;
    return (size_t)4 * C::LT * sizeof(double) + (size_t)C::RB * (C::LT + 1) * sizeof(double) +
           (size_t)C::RB * 2 * C::LT * sizeof(T) + (size_t)2 * C::KC * 2 * C::CT * sizeof(T) + 64;
}

// Grid (Mv * ceil(Lv / LT), column tiles); CTA (m, jb) = blockIdx.x / nj, % nj.
// spec: folded spectra [Mp][2][NP][C] of 2 * nvec scalar maps (column
// 2 (2b + c) + {re, im}); alm: [nvec][2][Lv][Mv] complex.  use_nf = 0 leaves
// out the 1/(l(l+1)) factor (the adjoint of the synthesis).
template <typename T>
__global__ void __launch_bounds__(256) k_vleg_fwd(const T* __restrict__ spec, int C, int nvec, T* __restrict__ alm,
                                                  int Lv, int Mv, int Lp, int Mp, int Lpad, Geom geo,
                                                  const RingPair* __restrict__ pairs, const int* __restrict__ lstart,
                                                  const double2* __restrict__ pstart,
                                                  const double2* __restrict__ coef, const double2* __restrict__ seeds,
                                                  int csphase, int use_nf) {
    using Cfg = VFwdCfg<T>;
    constexpr int LT = Cfg::LT, CT = Cfg::CT, RB = Cfg::RB, KC = Cfg::KC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = geo.NP;
    const int nj = (Lv + LT - 1) / LT;
    const int m = blockIdx.x / nj, jb = blockIdx.x % nj;
    const int l0 = m + jb * LT;
    const int c0 = blockIdx.y * CT;
    const int tid = threadIdx.x;
    double* cf = (double*)smem_raw;              // [4][LT]
    double* Pa = cf + 4 * LT;                    // [RB][LT+1] Pbar^{m-1}
    T* Dt = (T*)(Pa + RB * (LT + 1));            // [RB][2][LT]
    T* Xs = Dt + RB * 2 * LT;                    // [2][KC][2][CT]
    const int vb0 = c0 / 4;

    // the l < m triangle (and whole orders m >= Lv) are zero
    if (jb == 0) {
        const int lz = min(m, Lv);
        for (int i = tid; i < lz * (CT / 4) * 2; i += blockDim.x) {
            const int comp = i & 1, vb = vb0 + (i >> 1) % (CT / 4), l = (i >> 1) / (CT / 4);
            if (vb < nvec && HPX_INB(2 * ((((int64_t)vb * 2 + comp) * Lv + l) * Mv + m) + 1, kExtAlm, 17))
                *(cplx<T>*)(alm + 2 * ((((int64_t)vb * 2 + comp) * Lv + l) * Mv + m)) = {(T)0, (T)0};
        }
    }
    if (m >= Lv || l0 >= Lv) return;
    if (tid < LT) {
        double c1, c2, c3, c4;
        vec_coefs(l0 + tid, m, c1, c2, c3, c4);
        cf[tid] = c1;
        cf[LT + tid] = c2;
        cf[2 * LT + tid] = c3;
        cf[3 * LT + tid] = c4;
    }
    const int t0 = geo.first_ring(m);
    const int K = NP - t0;
    const int nbk = seed_blocks(Lp);

    const int bl = tid & 15;   // vector map within the tile
    const int dg = tid >> 4;   // degrees l0 + 2 dg, + 1
    T A[2][4], B[2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int k = 0; k < 4; ++k) A[i][k] = B[i][k] = (T)0;

    auto stage = [&](int buf, int rbase, int nr) {
        T* dst = Xs + buf * (KC * 2 * CT);
        constexpr int VPR = CT * sizeof(T) / 16;
        for (int i = tid; i < KC * 2 * VPR; i += blockDim.x) {
            const int v = i % VPR, row = i / VPR;
            const int q = row >> 1, pr = row & 1;
            const int c = c0 + v * (16 / (int)sizeof(T));
            const bool ok = q < nr && c < C;
            const T* src = spec + (((int64_t)m * 2 + pr) * NP + t0 + (ok ? rbase + q : 0)) * C + (ok ? c : 0);
            cp_async16(dst + row * CT + v * (16 / sizeof(T)), src, ok);
        }
        cp_async_commit();
    };

    for (int rb = 0; rb < K; rb += RB) {
        __syncthreads();  // coefficient factors ready / previous pass done with Pa, Dt
        if (tid < RB) {
            const int r = rb + tid;
            double* pa = Pa + tid * (LT + 1);
            T* d0 = Dt + tid * 2 * LT;
            T* d1 = d0 + LT;
            if (r < K) {
                const int p = t0 + r;
                const double x = pairs[p].z;
                // order m+1 from its degree-block seed at or below l0 (values below m+1 are zero)
                const int ob = m + 1;
                const int jbb = l0 > ob ? (l0 - ob) / kSeedBlock : 0;
                // order m-1 likewise (m = 0 uses Pbar^{-1} = -Pbar^1)
                if (m >= 1) {
                    const int oa = m - 1;
                    const int jba = (l0 - oa) / kSeedBlock;
                    const int64_t mia = (int64_t)oa * NP + p;
                    const int ls = lstart[mia];
                    const double2 ps = pstart[mia];
                    const double2 sd = seeds[((int64_t)oa * nbk + jba) * NP + p];
                    const double2* ca = coef + (int64_t)oa * Lpad;
                    const int lsb = oa + jba * kSeedBlock;
                    double q1 = 0.0, q2 = 0.0;
                    for (int l = lsb; l <= l0 + LT; ++l) {
                        double v;
                        if (l == lsb && ls <= lsb) v = sd.x;
                        else if (l == lsb + 1 && ls <= lsb) v = sd.y;
                        else {
                            const double2 ab = (l >= oa + 2 && l < Lp) ? ca[l] : make_double2(0.0, 0.0);
                            v = l < Lp ? leg_step(l, ls, ps, ab.x, ab.y, x, q1, q2) : 0.0;
                        }
                        q2 = q1;
                        q1 = v;
                        if (l >= l0) pa[l - l0] = v;
                    }
                }
                const int64_t mib = (int64_t)ob * NP + p;
                const int ls = ob < Mp ? lstart[mib] : Lp;
                const double2 ps = ob < Mp ? pstart[mib] : make_double2(0.0, 0.0);
                const int lsb = ob + jbb * kSeedBlock;
                const double2 sd = (ob < Mp && lsb < Lp) ? seeds[((int64_t)ob * nbk + jbb) * NP + p] : make_double2(0.0, 0.0);
                const double2* cb = coef + (int64_t)(ob < Mp ? ob : 0) * Lpad;
                double q1 = 0.0, q2 = 0.0, prev = 0.0;
                const int lstart_b = min(lsb, l0);
                for (int l = lstart_b; l <= l0 + LT; ++l) {
                    double v = 0.0;
                    if (l >= ob && ob < Mp && l < Lp) {
                        if (l == lsb && ls <= lsb) v = sd.x;
                        else if (l == lsb + 1 && ls <= lsb) v = sd.y;
                        else {
                            const double2 ab = l >= ob + 2 ? cb[l] : make_double2(0.0, 0.0);
                            v = leg_step(l, ls, ps, ab.x, ab.y, x, q1, q2);
                        }
                    }
                    q2 = q1;
                    q1 = v;
                    if (l >= l0) {
                        const int i = l - l0;
                        const double pm = m >= 1 ? pa[i] : -v;  // Pbar_l^{m-1}
                        if (i < LT) d0[i] = (T)((l >= m && l < Lv) ? cf[i] * pm - cf[LT + i] * v : 0.0);
                        if (i > 0) {
                            // D1 at degree l - 1 uses Pbar_l^{m-1} and Pbar_l^{m+1}
                            const int ld = l - 1;
                            d1[i - 1] = (T)((m >= 1 && ld >= m && ld < Lv) ? cf[2 * LT + i - 1] * pm + cf[3 * LT + i - 1] * v
                                                                             : 0.0);
                        }
                    }
                    prev = v;
                }
                (void)prev;
            } else {
                for (int i = 0; i < LT; ++i) d0[i] = d1[i] = (T)0;
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
            for (int q = 0; q < qn; ++q) {
                const T* drow = Dt + (ch * KC + q) * 2 * LT;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int li = 2 * dg + i;
                    const int par0 = (li + 1) & 1;  // l - m = jb*LT + li, LT even
                    const T d0 = drow[li], d1 = drow[LT + li];
                    const T* x0 = xb + (q * 2 + par0) * CT + 4 * bl;
                    const T* x1 = xb + (q * 2 + (par0 ^ 1)) * CT + 4 * bl;
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        A[i][k] = fma(d0, x0[k], A[i][k]);
                        B[i][k] = fma(d1, x1[k], B[i][k]);
                    }
                }
            }
            __syncthreads();
        }
    }
    // S = nf (A0 - i B1), T = nf (-A1 - i B0); A0 = (A[0], A[1]), A1 = (A[2], A[3]), likewise B
    const int vb = vb0 + bl;
    if (vb >= nvec) return;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int l = l0 + 2 * dg + i;
        if (l >= Lv) continue;
        T nf = (l == 0 || !use_nf) ? (T)1 : (T)(1.0 / ((double)l * (double)(l + 1)));
        if (csphase && (m & 1)) nf = -nf;
        if (!HPX_INB(2 * ((((int64_t)vb * 2 + 1) * Lv + l) * Mv + m) + 1, kExtAlm, 18)) continue;
        const cplx<T> S = {nf * (A[i][0] + B[i][3]), nf * (A[i][1] - B[i][2])};
        const cplx<T> Tt = {nf * (B[i][1] - A[i][2]), -nf * (A[i][3] + B[i][0])};
        *(cplx<T>*)(alm + 2 * ((((int64_t)vb * 2 + 0) * Lv + l) * Mv + m)) = S;
        *(cplx<T>*)(alm + 2 * ((((int64_t)vb * 2 + 1) * Lv + l) * Mv + m)) = Tt;
    }
}

// ------------------------------------------------------------ synthesis
template <typename T>
struct VInvCfg {
    static constexpr int RBI = 64;  // rings per CTA
    static constexpr int CT = 64;   // columns per CTA (16 vector maps)
    static constexpr int LC = 32;   // degrees per staged chunk
};

template <typename T>
__host__ __device__ constexpr size_t vinv_smem_bytes() {
    using C = VInvCfg<T>;
    return (size_t)4 * C::LC * sizeof(double) + (size_t)2 * C::LC * C::RBI * sizeof(T) +
           (size_t)C::LC * C::CT * sizeof(T) + 64;
}

// Grid (Mp * ceil(NP / RBI), column tiles); CTA (m, ring block) = blockIdx.x / nr, % nr.
// Writes E/O spectra spec[m][0|1][p][C] of the 2 nvec scalar maps for every
// m < Mp and ring p >= first_ring(m) (zeros for orders the coefficients do not carry).
// use_nf = 1 first scales the coefficients by 1/(l(l+1)) (the adjoint of the analysis).
template <typename T>
__global__ void __launch_bounds__(256) k_vleg_inv(const T* __restrict__ alm, int nvec, T* __restrict__ spec, int C,
                                                  int Lv, int Mv, int Lp, int Mp, int Lpad, Geom geo,
                                                  const RingPair* __restrict__ pairs, const int* __restrict__ lstart,
                                                  const double2* __restrict__ pstart,
                                                  const double2* __restrict__ coef, int csphase, int use_nf) {
    using Cfg = VInvCfg<T>;
    constexpr int RBI = Cfg::RBI, CT = Cfg::CT, LC = Cfg::LC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = geo.NP;
    const int nr = (NP + RBI - 1) / RBI;
    const int m = blockIdx.x / nr, rb = (blockIdx.x % nr) * RBI;
    const int c0 = blockIdx.y * CT;
    const int tid = threadIdx.x;
    const int t0 = geo.first_ring(m);
    const int K = NP - t0;
    if (rb >= K) return;
    double* cf = (double*)smem_raw;       // [4][LC]
    T* D0 = (T*)(cf + 4 * LC);            // [LC][RBI]
    T* D1 = D0 + LC * RBI;                // [LC][RBI]
    T* As = D1 + LC * RBI;                // [LC][CT]: per vector map S re, S im, T re, T im

    const int tx = tid & 15, ty = tid >> 4;
    const int rrow = ty * 4;
    T E[4][4], O[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int k = 0; k < 4; ++k) E[i][k] = O[i][k] = (T)0;

    if (m < Mv && m < Lv) {
        // generator threads: one ring each, running orders m-1 and m+1 one degree ahead
        const int rg = rb + tid;
        const bool gen = tid < RBI && rg < K;
        LegRun ra, rbn;
        double cur_a = 0.0, nxt_a = 0.0, cur_b = 0.0, nxt_b = 0.0;
        const double2* ca = coef + (int64_t)(m >= 1 ? m - 1 : 0) * Lpad;
        const double2* cb = coef + (int64_t)(m + 1) * Lpad;
        if (gen) {
            const int p = t0 + rg;
            const double x = pairs[p].z;
            if (m >= 1) ra.init(m - 1, Mp, Mp, (int64_t)(m - 1) * NP + p, lstart, pstart, x);
            rbn.init(m + 1, Mp, Mp, (int64_t)(m + 1) * NP + p, lstart, pstart, x);
            // degree m: Pbar_m^{m-1} needs the run from m-1; Pbar_m^{m+1} = 0
            if (m >= 1) {
                ra.next(ca, Lp);           // degree m-1
                cur_a = ra.next(ca, Lp);   // degree m
                nxt_a = ra.next(ca, Lp);   // degree m+1
            }
            cur_b = 0.0;
            nxt_b = rbn.next(cb, Lp);      // degree m+1
        }
        for (int l0 = m; l0 < Lv; l0 += LC) {
            __syncthreads();  // previous chunk consumed
            if (tid < LC) {
                double c1, c2, c3, c4;
                vec_coefs(l0 + tid, m, c1, c2, c3, c4);
                cf[tid] = c1;
                cf[LC + tid] = c2;
                cf[2 * LC + tid] = c3;
                cf[3 * LC + tid] = c4;
            }
            for (int i = tid; i < LC * CT; i += blockDim.x) {
                const int c = i % CT, li = i / CT, l = l0 + li;
                const int vb = (c0 + c) >> 2, k = c & 3;  // k: S re, S im, T re, T im
                T v = (T)0;
                if (l < Lv && vb < nvec) v = alm[2 * ((((int64_t)vb * 2 + (k >> 1)) * Lv + l) * Mv + m) + (k & 1)];
                if (use_nf && l > 0) v = (T)((double)v / ((double)l * (double)(l + 1)));
                As[li * CT + c] = v;
            }
            __syncthreads();
            if (tid < RBI) {
                for (int i = 0; i < LC; ++i) {
                    const int l = l0 + i;
                    double d0 = 0.0, d1 = 0.0;
                    if (gen && l < Lv) {
                        const double pa = m >= 1 ? cur_a : -cur_b;
                        d0 = cf[i] * pa - cf[LC + i] * cur_b;
                        d1 = m >= 1 ? cf[2 * LC + i] * nxt_a + cf[3 * LC + i] * nxt_b : 0.0;
                        cur_a = nxt_a;
                        cur_b = nxt_b;
                        if (m >= 1) nxt_a = ra.next(ca, Lp);
                        nxt_b = rbn.next(cb, Lp);
                    }
                    if (csphase && (m & 1)) {
                        d0 = -d0;
                        d1 = -d1;
                    }
                    D0[i * RBI + tid] = (T)d0;
                    D1[i * RBI + tid] = (T)d1;
                }
            }
            __syncthreads();
            for (int li = 0; li < LC; ++li) {
                const int l = l0 + li;
                const bool even = ((l + m) & 1) == 0;
                const T* ar = As + li * CT + 4 * tx;
                const T sr = ar[0], si = ar[1], tr = ar[2], ti = ar[3];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const T d0 = D0[li * RBI + rrow + i], d1 = D1[li * RBI + rrow + i];
                    // D0 part (south sign -(-1)^{l+m}) and D1 part (south sign (-1)^{l+m})
                    const T p0[4] = {d0 * sr, d0 * si, -d0 * tr, -d0 * ti};
                    const T p1[4] = {-d1 * ti, d1 * tr, -d1 * si, d1 * sr};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        E[i][k] += even ? p1[k] : p0[k];
                        O[i][k] += even ? p0[k] : p1[k];
                    }
                }
            }
        }
    }
    // write E/O for the rings of this CTA
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = rb + rrow + i;
        if (r >= K || c0 + 4 * tx >= C || !HPX_INB((((int64_t)m * 2 + 1) * NP + t0 + r) * C + c0 + 4 * tx + 3, kExtSpec, 19))
            continue;
        T* e = spec + (((int64_t)m * 2 + 0) * NP + t0 + r) * C + c0 + 4 * tx;
        T* o = spec + (((int64_t)m * 2 + 1) * NP + t0 + r) * C + c0 + 4 * tx;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (c0 + 4 * tx + k < C) {
                e[k] = E[i][k];
                o[k] = O[i][k];
            }
        }
    }
}

}  // namespace hpx
