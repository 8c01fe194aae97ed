// Tensor-core (tcgen05) Legendre contraction, BF16 3-term split, FP32 accumulate.
//
// Same mathematics as the SIMT kernels in legendre.cuh (orthonormal Pbar_l^m,
// north/south folding, per-m contraction), mapped onto the 5th-generation
// tensor cores:
//
//  * the Pbar operand is generated on the fly by producer warps running the
//    FP64 three-term recurrence from the plan's 64-degree block seeds, rounded
//    to FP32 and split into bf16 hi + lo, and stored straight into shared
//    memory in the UMMA SWIZZLE_128B (analysis) / SWIZZLE_64B (synthesis)
//    canonical layout;
//  * the data operand (folded spectra for analysis, coefficients for
//    synthesis) is pre-split into bf16 hi/lo in global memory and brought in by
//    TMA (cp.async.bulk.tensor, 128B swizzle, no multicast);
//  * one thread issues tcgen05.mma (M=128, N=128, K=16) for the three products
//    hi*hi + hi*lo + lo*hi into FP32 accumulators in TMEM; tcgen05.commit
//    frees a pipeline stage when its MMAs retire;
//  * four epilogue warps drain TMEM (tcgen05.ld) while the next tile
//    accumulates into the other half of TMEM.
//
// Analysis tile  = (m, 256 consecutive degrees): D_par[128 l][128 cols] +=
//                   Pbar_par[128 l][32 rings] * X_par[32 rings][128 cols]
// Synthesis tile = (m, 128 rings):   D_par[128 rings][128 cols] +=
//                   Pbar^T[128 rings][32 l] * A_par[32 l][128 cols]
// where par is the parity of l-m and cols = 2*map + {re, im}.
//
// Persistent kernels, one CTA per SM, static round-robin over a tile list.
// Every mbarrier wait is bounded (tc_ptx.cuh); a timeout writes an error code
// to the plan's device flag and the kernel drains and returns.
#pragma once

#include "legendre.cuh"
#include "tc_ptx.cuh"

namespace hpx {

constexpr int kTcCols = 128;      // N: columns per tile (64 maps)
constexpr int kTcStages = 3;      // smem pipeline depth
constexpr int kTcRingChunk = 32;  // K per analysis stage (rings)
constexpr int kTcFwdDeg = 256;    // degrees per analysis tile (128 per parity)
constexpr int kTcInvRings = 128;  // rings per synthesis tile
constexpr int kTcDegChunk = 64;   // degrees per synthesis stage (32 per parity)
constexpr int kTcThreads = 512;   // 16 warps
constexpr int kTcStageBytes = 65536;
constexpr int kTcSmem = kTcStages * kTcStageBytes + 8 * 1024 + 1024 + 1024;

// Host-side state of the tensor-core path, owned by the plan.
struct TcPlan {
    int active = 0;
    int nsm = 0;
    int* d_err = nullptr;     // device error flag written by bounded waits
    int2* d_fwd_tiles = nullptr;
    int n_fwd_tiles = 0;
    int2* d_inv_tiles = nullptr;
    int n_inv_tiles = 0;
    int m_tc_end = 0;         // orders m < m_tc_end go through the tensor cores
    int Lh = 0;               // rows per (m, parity) of the synthesis operand
    void* encode = nullptr;   // cuTensorMapEncodeTiled (driver entry point)
};

// ------------------------------------------------------------------ shared layout
struct TcShared {
    uint64_t full_tma[kTcStages];
    uint64_t full_prod[kTcStages];
    uint64_t empty[kTcStages];
    uint64_t acc_full[2];
    uint64_t acc_empty[2];
    uint64_t drain;
    uint32_t tmem_base;
};

__device__ __forceinline__ uint32_t pack_bf16x2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

// split 8 doubles into bf16 hi/lo 16-byte vectors
__device__ __forceinline__ void split8(const double* v, uint4& hi, uint4& lo) {
    uint16_t h[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) tc::split_bf16((float)v[i], h[i], l[i]);
    hi = make_uint4(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]), pack_bf16x2(h[4], h[5]), pack_bf16x2(h[6], h[7]));
    lo = make_uint4(pack_bf16x2(l[0], l[1]), pack_bf16x2(l[2], l[3]), pack_bf16x2(l[4], l[5]), pack_bf16x2(l[6], l[7]));
}

// On exit (normal or after a timeout) the TMA thread waits, bounded, for the
// loads it issued into the last pipeline stages, so no bulk copy lands in
// shared memory after the CTA has finished.
__device__ __forceinline__ void tma_drain(TcShared* sh, int issued, int* err) {
    (void)err;
    for (int k = 1; k <= kTcStages && issued - k >= 0; ++k) {
        const int it = issued - k;
        int local = 0;  // bounded wait that does not stop early on another role's error
        tc::mbar_wait(&sh->full_tma[it % kTcStages], (it / kTcStages) & 1, &local, 0);
    }
}
// The MMA thread commits once more and waits, bounded, so that every MMA it
// issued has retired before TMEM is released.
__device__ __forceinline__ void mma_drain(TcShared* sh, int* err) {
    tc::mma_commit(&sh->drain);
    int dummy = 0;
    tc::mbar_wait(&sh->drain, 0, &dummy, 0);
    (void)err;
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

// Generate 64 consecutive degrees l0b..l0b+63 of one ring from its block seed,
// handing every 16 degrees (8 of each parity) to `emit(s, even8, odd8)`.
template <typename Emit>
__device__ __forceinline__ void gen_block64(int l0b, int L, int ls, double2 ps, double2 sd, double x,
                                            const double2* __restrict__ cf, bool fast, Emit&& emit) {
    double p2 = 0.0, p1 = 0.0;
    double ev[8], od[8];
    if (fast) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int i = s * 16 + k;
                double v;
                if (i == 0) v = sd.x;
                else if (i == 1) v = sd.y;
                else {
                    const double2 ab = cf[i];
                    v = ab.x * x * p1 - ab.y * p2;
                }
                p2 = p1;
                p1 = v;
                if (k & 1) od[k >> 1] = v; else ev[k >> 1] = v;
            }
            emit(s, ev, od);
        }
    } else {
#pragma unroll 1
        for (int s = 0; s < 4; ++s) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int i = s * 16 + k;
                const int l = l0b + i;
                const double2 ab = cf[i];
                double v = (l < L) ? leg_step(l, ls, ps, ab.x, ab.y, x, p1, p2) : 0.0;
                p2 = p1;
                p1 = v;
                if (k & 1) od[k >> 1] = v; else ev[k >> 1] = v;
            }
            emit(s, ev, od);
        }
    }
}

// ================================================================== analysis
// Xh/Xl: bf16 [2M][NP][128] (hi and lo of S (par 0) and D (par 1)) via tensor maps.
__global__ void __launch_bounds__(kTcThreads, 1)
    k_leg_fwd_tc(const __grid_constant__ CUtensorMap xh_map, const __grid_constant__ CUtensorMap xl_map, int nmaps,
                 float* __restrict__ alm, int L, int M, int Lpad, int nside, const RingPair* __restrict__ pairs,
                 const int* __restrict__ lstart, const double2* __restrict__ pstart, const double2* __restrict__ coef,
                 const double2* __restrict__ seeds, const int2* __restrict__ tiles, int ntiles, int accumulate,
                 int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* stages = base;                                           // kTcStages x 64 KB
    double2* coef_s = (double2*)(base + kTcStages * kTcStageBytes);         // 8 producer warps x 64
    TcShared* sh = (TcShared*)(base + kTcStages * kTcStageBytes + 8 * 1024);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NP = 2 * nside;
    const int nbk = seed_blocks(L);

    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            tc::mbar_init(&sh->full_tma[s], 1);
            tc::mbar_init(&sh->full_prod[s], 4);
            tc::mbar_init(&sh->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&sh->acc_full[a], 1);
            tc::mbar_init(&sh->acc_empty[a], 4);
        }
        tc::mbar_init(&sh->drain, 1);
        tc::fence_mbar_init();
    }
    if (warp == 1) {
        tc::tmem_alloc(&sh->tmem_base, 512);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sh->tmem_base;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            tc::tma_prefetch_desc(&xh_map);
            tc::tma_prefetch_desc(&xl_map);
            int it = 0;
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
                const int m = tiles[t].x;
                const int t0 = first_ring_for_m(m, nside);
                const int nch = (NP - t0 + kTcRingChunk - 1) / kTcRingChunk;
                for (int c = 0; c < nch; ++c, ++it) {
                    const int s = it % kTcStages;
                    if (!tc::mbar_wait(&sh->empty[s], ((it / kTcStages) & 1) ^ 1, err, 11)) goto tma_done;
                    unsigned char* st = stages + s * kTcStageBytes + 32768;  // B region
                    tc::mbar_arrive_tx(&sh->full_tma[s], 32768);
                    const int y = t0 + c * kTcRingChunk;
#pragma unroll
                    for (int par = 0; par < 2; ++par)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            tc::tma_load_3d(st + (par * 2 + 0) * 8192 + h * 4096, &xh_map, h * 64, y, 2 * m + par,
                                            &sh->full_tma[s]);
                            tc::tma_load_3d(st + (par * 2 + 1) * 8192 + h * 4096, &xl_map, h * 64, y, 2 * m + par,
                                            &sh->full_tma[s]);
                        }
                }
            }
        tma_done:
            tma_drain(sh, it, err);
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_bf16(128, kTcCols, true, true);
            int it = 0, tcount = 0;
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tcount) {
                const int m = tiles[t].x;
                const int t0 = first_ring_for_m(m, nside);
                const int nch = (NP - t0 + kTcRingChunk - 1) / kTcRingChunk;
                const int a = tcount & 1;
                if (!tc::mbar_wait(&sh->acc_empty[a], ((tcount >> 1) & 1) ^ 1, err, 12)) break;
                tc::tc_fence_after();
                const uint32_t dbase = tmem + a * 2 * kTcCols;
                for (int c = 0; c < nch; ++c, ++it) {
                    const int s = it % kTcStages;
                    const uint32_t ph = (it / kTcStages) & 1;
                    if (!tc::mbar_wait(&sh->full_tma[s], ph, err, 13)) goto mma_done;
                    if (!tc::mbar_wait(&sh->full_prod[s], ph, err, 14)) goto mma_done;
                    tc::tc_fence_after();
                    const uint32_t sa = tc::smem_u32(stages + s * kTcStageBytes);
                    const uint32_t sb = sa + 32768;
#pragma unroll
                    for (int par = 0; par < 2; ++par) {
                        const uint32_t d = dbase + par * kTcCols;
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            const uint64_t ah = tc::smem_desc_sw128(sa + (par * 2 + 0) * 8192 + ks * 2048, 4096, 1024);
                            const uint64_t al = tc::smem_desc_sw128(sa + (par * 2 + 1) * 8192 + ks * 2048, 4096, 1024);
                            const uint64_t bh = tc::smem_desc_sw128(sb + (par * 2 + 0) * 8192 + ks * 2048, 4096, 1024);
                            const uint64_t bl = tc::smem_desc_sw128(sb + (par * 2 + 1) * 8192 + ks * 2048, 4096, 1024);
                            tc::mma_bf16(d, ah, bh, idesc, (c > 0 || ks > 0) ? 1u : 0u);
                            tc::mma_bf16(d, ah, bl, idesc, 1u);
                            tc::mma_bf16(d, al, bh, idesc, 1u);
                        }
                    }
                    tc::mma_commit(&sh->empty[s]);
                }
                tc::mma_commit(&sh->acc_full[a]);
            }
        mma_done:
            mma_drain(sh, err);
        }
    } else if (warp >= 4 && warp < 8) {
        // ------------------------------------------------ epilogue: TMEM -> alm
        const int ew = warp & 3;  // TMEM lanes 32*ew .. +31
        int tcount = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tcount) {
            const int m = tiles[t].x, jb = tiles[t].y;
            const int l0 = m + jb * kTcFwdDeg;
            const int a = tcount & 1;
            // zero the l < m triangle of this column while the tile accumulates
            if (!accumulate && jb == 0) {
                const int nz = min(m, L);
                for (int i = (warp - 4) * 32 + lane; i < nz * 64; i += 128) {
                    const int l = i >> 6, b = i & 63;
                    if (b < nmaps) *(float2*)(alm + 2 * (((int64_t)b * L + l) * M + m)) = make_float2(0.f, 0.f);
                }
            }
            if (!tc::mbar_wait_warp(&sh->acc_full[a], (tcount >> 1) & 1, err, 15)) break;
            tc::tc_fence_after();
            const int row = ew * 32 + lane;
#pragma unroll 1
            for (int par = 0; par < 2; ++par) {
                const int l = l0 + 2 * row + par;
                const uint32_t taddr = tmem + ((uint32_t)(ew * 32) << 16) + a * 2 * kTcCols + par * kTcCols;
#pragma unroll 1
                for (int c = 0; c < kTcCols; c += 16) {
                    float v[16];
                    tc::tmem_ld16(taddr + c, v);
                    if (l < L) {
#pragma unroll
                        for (int j = 0; j < 16; j += 2) {
                            const int b = (c + j) >> 1;
                            if (b < nmaps) {
                                float2* dst = (float2*)(alm + 2 * (((int64_t)b * L + l) * M + m));
                                float2 o = make_float2(v[j], v[j + 1]);
                                if (accumulate) {
                                    const float2 q = *dst;
                                    o.x += q.x;
                                    o.y += q.y;
                                }
                                *dst = o;
                            }
                        }
                    }
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sh->acc_empty[a]);
        }
    } else if (warp >= 8) {
        // ------------------------------------------------ Pbar producers
        const int pw = warp - 8;    // 0..7
        const int grp = pw >> 2;    // chunk parity handled by this group
        const int q = pw & 3;       // 64-degree block within the tile
        double2* cfw = coef_s + pw * 64;
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int m = tiles[t].x, jb = tiles[t].y;
            const int l0 = m + jb * kTcFwdDeg;
            const int l0b = l0 + 64 * q;
            const int t0 = first_ring_for_m(m, nside);
            const int nch = (NP - t0 + kTcRingChunk - 1) / kTcRingChunk;
            // coefficients of this warp's 64 degrees (zero beyond L)
            __syncwarp();
            for (int i = lane; i < 64; i += 32) cfw[i] = coef[(int64_t)m * Lpad + min(l0b + i, Lpad - 1)];
            __syncwarp();
            for (int c = 0; c < nch; ++c, ++it) {
                if ((it & 1) != grp) continue;
                const int s = it % kTcStages;
                if (!tc::mbar_wait_warp(&sh->empty[s], ((it / kTcStages) & 1) ^ 1, err, 16)) goto prod_done;
                const int p = t0 + c * kTcRingChunk + lane;
                const uint32_t sa = tc::smem_u32(stages + s * kTcStageBytes);
                // A tile layout (per parity, hi/lo): atom (i/64) * 4096 + ring group (lane/8) * 1024
                const uint32_t rowbase = (uint32_t)((q >> 1) * 4096 + (lane >> 3) * 1024);
                auto emit = [&](int sidx, const double* ev, const double* od) {
                    uint4 eh, el, oh, ol;
                    split8(ev, eh, el);
                    split8(od, oh, ol);
                    const uint32_t off = rowbase + tc::sw128_offset(lane & 7, ((q & 1) << 2) + sidx);
                    st_shared_v4(sa + 0 * 8192 + off, eh);
                    st_shared_v4(sa + 1 * 8192 + off, el);
                    st_shared_v4(sa + 2 * 8192 + off, oh);
                    st_shared_v4(sa + 3 * 8192 + off, ol);
                };
                const bool valid = p < NP && l0b < L;
                const int64_t mi = (int64_t)m * NP + (valid ? p : 0);
                const int ls = valid ? lstart[mi] : L;
                const bool fast = __all_sync(0xffffffffu, !valid || ls <= l0b);
                if (valid) {
                    const double2 sd = seeds[((int64_t)m * nbk + (l0b - m) / 64) * NP + p];
                    const double2 ps = fast ? make_double2(0.0, 0.0) : pstart[mi];
                    gen_block64(l0b, L, ls, ps, sd, pairs[p].z, cfw, fast, emit);
                } else {
                    const double z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
                    for (int sidx = 0; sidx < 4; ++sidx) emit(sidx, z8, z8);
                }
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh->full_prod[s]);
            }
        }
    prod_done:;
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

// ================================================================== synthesis
// Ah/Al: bf16 [2M][Lh][128] coefficient operand (row i of (m, par) is degree
// l = m + 2i + par) via tensor maps; writes E/O into spec[m][par][p][c] (FP32).
__global__ void __launch_bounds__(kTcThreads, 1)
    k_leg_inv_tc(const __grid_constant__ CUtensorMap ah_map, const __grid_constant__ CUtensorMap al_map,
                 float* __restrict__ spec, int C, int L, int M, int Lpad, int nside, const RingPair* __restrict__ pairs,
                 const int* __restrict__ lstart, const double2* __restrict__ pstart, const double2* __restrict__ coef,
                 const double2* __restrict__ seeds, const int2* __restrict__ tiles, int ntiles, int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* stages = base;
    double2* coef_s = (double2*)(base + kTcStages * kTcStageBytes);
    TcShared* sh = (TcShared*)(base + kTcStages * kTcStageBytes + 8 * 1024);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NP = 2 * nside;
    const int nbk = seed_blocks(L);

    if (tid == 0) {
        for (int s = 0; s < kTcStages; ++s) {
            tc::mbar_init(&sh->full_tma[s], 1);
            tc::mbar_init(&sh->full_prod[s], 4);
            tc::mbar_init(&sh->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&sh->acc_full[a], 1);
            tc::mbar_init(&sh->acc_empty[a], 4);
        }
        tc::mbar_init(&sh->drain, 1);
        tc::fence_mbar_init();
    }
    if (warp == 1) {
        tc::tmem_alloc(&sh->tmem_base, 512);
        tc::tmem_relinquish();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = sh->tmem_base;

    auto nchunks = [&](int m) { return m < L ? (L - m + kTcDegChunk - 1) / kTcDegChunk : 0; };

    if (warp == 0) {
        if (lane == 0) {
            tc::tma_prefetch_desc(&ah_map);
            tc::tma_prefetch_desc(&al_map);
            int it = 0;
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
                const int m = tiles[t].x;
                const int nch = nchunks(m);
                for (int c = 0; c < nch; ++c, ++it) {
                    const int s = it % kTcStages;
                    if (!tc::mbar_wait(&sh->empty[s], ((it / kTcStages) & 1) ^ 1, err, 21)) goto tma_done;
                    unsigned char* st = stages + s * kTcStageBytes + 32768;
                    tc::mbar_arrive_tx(&sh->full_tma[s], 32768);
#pragma unroll
                    for (int par = 0; par < 2; ++par)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            tc::tma_load_3d(st + (par * 2 + 0) * 8192 + h * 4096, &ah_map, h * 64, c * 32, 2 * m + par,
                                            &sh->full_tma[s]);
                            tc::tma_load_3d(st + (par * 2 + 1) * 8192 + h * 4096, &al_map, h * 64, c * 32, 2 * m + par,
                                            &sh->full_tma[s]);
                        }
                }
            }
        tma_done:
            tma_drain(sh, it, err);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // A (Pbar^T) K-major SW64, B (coefficients) MN-major SW128
            const uint32_t idesc = tc::idesc_bf16(128, kTcCols, false, true);
            int it = 0, tcount = 0;
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tcount) {
                const int m = tiles[t].x;
                const int nch = nchunks(m);
                const int a = tcount & 1;
                if (!tc::mbar_wait(&sh->acc_empty[a], ((tcount >> 1) & 1) ^ 1, err, 22)) break;
                tc::tc_fence_after();
                const uint32_t dbase = tmem + a * 2 * kTcCols;
                for (int c = 0; c < nch; ++c, ++it) {
                    const int s = it % kTcStages;
                    const uint32_t ph = (it / kTcStages) & 1;
                    if (!tc::mbar_wait(&sh->full_tma[s], ph, err, 23)) goto mma_done;
                    if (!tc::mbar_wait(&sh->full_prod[s], ph, err, 24)) goto mma_done;
                    tc::tc_fence_after();
                    const uint32_t sa = tc::smem_u32(stages + s * kTcStageBytes);
                    const uint32_t sb = sa + 32768;
#pragma unroll
                    for (int par = 0; par < 2; ++par) {
                        const uint32_t d = dbase + par * kTcCols;
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            const uint64_t ah = tc::smem_desc_kmajor_sw64(sa + (par * 2 + 0) * 8192 + ks * 32, 512);
                            const uint64_t al = tc::smem_desc_kmajor_sw64(sa + (par * 2 + 1) * 8192 + ks * 32, 512);
                            const uint64_t bh = tc::smem_desc_sw128(sb + (par * 2 + 0) * 8192 + ks * 2048, 4096, 1024);
                            const uint64_t bl = tc::smem_desc_sw128(sb + (par * 2 + 1) * 8192 + ks * 2048, 4096, 1024);
                            tc::mma_bf16(d, ah, bh, idesc, (c > 0 || ks > 0) ? 1u : 0u);
                            tc::mma_bf16(d, ah, bl, idesc, 1u);
                            tc::mma_bf16(d, al, bh, idesc, 1u);
                        }
                    }
                    tc::mma_commit(&sh->empty[s]);
                }
                tc::mma_commit(&sh->acc_full[a]);
            }
        mma_done:
            mma_drain(sh, err);
        }
    } else if (warp >= 4 && warp < 8) {
        // ------------------------------------------------ epilogue: TMEM -> spec (E, O)
        const int ew = warp & 3;
        int tcount = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++tcount) {
            const int m = tiles[t].x, rb = tiles[t].y;
            const int t0 = first_ring_for_m(m, nside);
            const int a = tcount & 1;
            const int r = rb + ew * 32 + lane;
            const int p = t0 + r;
            if (!tc::mbar_wait_warp(&sh->acc_full[a], (tcount >> 1) & 1, err, 25)) break;
            tc::tc_fence_after();
#pragma unroll 1
            for (int par = 0; par < 2; ++par) {
                float* dst = spec + (((int64_t)m * 2 + par) * NP + p) * C;
                const uint32_t taddr = tmem + ((uint32_t)(ew * 32) << 16) + a * 2 * kTcCols + par * kTcCols;
#pragma unroll 1
                for (int c = 0; c < kTcCols; c += 16) {
                    float v[16];
                    tc::tmem_ld16(taddr + c, v);
                    if (p < NP && c < C) {
#pragma unroll
                        for (int j = 0; j < 16; j += 4) *(float4*)(dst + c + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                    }
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sh->acc_empty[a]);
        }
    } else if (warp >= 8) {
        // ------------------------------------------------ Pbar^T producers
        const int pw = warp - 8;
        const int grp = pw >> 2;  // chunk parity handled by this group
        const int rw = pw & 3;    // 32-ring slice of the 128-ring tile
        double2* cfw = coef_s + pw * 64;
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const int m = tiles[t].x, rb = tiles[t].y;
            const int t0 = first_ring_for_m(m, nside);
            const int nch = nchunks(m);
            const int r = rw * 32 + lane;  // row of the A tile
            const int p = t0 + rb + r;
            const bool valid = p < NP;
            const int64_t mi = (int64_t)m * NP + (valid ? p : 0);
            const int ls = valid ? lstart[mi] : L;
            const double x = valid ? pairs[p].z : 0.0;
            for (int c = 0; c < nch; ++c, ++it) {
                if ((it & 1) != grp) continue;
                const int s = it % kTcStages;
                const int l0b = m + c * kTcDegChunk;
                __syncwarp();
                for (int i = lane; i < 64; i += 32) cfw[i] = coef[(int64_t)m * Lpad + min(l0b + i, Lpad - 1)];
                __syncwarp();
                if (!tc::mbar_wait_warp(&sh->empty[s], ((it / kTcStages) & 1) ^ 1, err, 26)) goto prod_done;
                const uint32_t sa = tc::smem_u32(stages + s * kTcStageBytes);
                // K-major SW64: row r (ring), 32 bf16 per row; 8-row groups of 512 B
                const uint32_t rowbase = (uint32_t)((r >> 3) * 512);
                auto emit = [&](int sidx, const double* ev, const double* od) {
                    uint4 eh, el, oh, ol;
                    split8(ev, eh, el);
                    split8(od, oh, ol);
                    const uint32_t off = rowbase + tc::sw64_offset(r & 7, sidx);
                    st_shared_v4(sa + 0 * 8192 + off, eh);
                    st_shared_v4(sa + 1 * 8192 + off, el);
                    st_shared_v4(sa + 2 * 8192 + off, oh);
                    st_shared_v4(sa + 3 * 8192 + off, ol);
                };
                const bool fast = __all_sync(0xffffffffu, !valid || ls <= l0b);
                if (valid) {
                    const double2 sd = seeds[((int64_t)m * nbk + c) * NP + p];
                    const double2 ps = fast ? make_double2(0.0, 0.0) : pstart[mi];
                    gen_block64(l0b, L, ls, ps, sd, x, cfw, fast, emit);
                } else {
                    const double z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
                    for (int sidx = 0; sidx < 4; ++sidx) emit(sidx, z8, z8);
                }
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh->full_prod[s]);
            }
        }
    prod_done:;
    }

    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc::tc_fence_after();
        tc::tmem_dealloc(tmem, 512);
    }
}

// ================================================================== operand preparation
// alm[b][l][m] (FP32 complex) -> Ah/Al bf16 [2M][Lh][128]: row i of (m, par) is
// degree l = m + 2i + par; rows with l >= L (up to L+63) are written as zeros.
__global__ void k_alm_to_tc(const float* __restrict__ alm, int nmaps, int L, int M, int Lh,
                            uint16_t* __restrict__ ah, uint16_t* __restrict__ al) {
    __shared__ float2 tile[64][33];
    const int m0 = blockIdx.x * 32, l = blockIdx.y;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int i = ty; i < 64; i += 8) {
        const int m = m0 + tx;
        float2 v = make_float2(0.f, 0.f);
        if (i < nmaps && m < M && l < L) v = *(const float2*)(alm + 2 * (((int64_t)i * L + l) * M + m));
        tile[i][tx] = v;
    }
    __syncthreads();
    // each warp writes rows for 4 m's: 128 columns as 64 bf16x2 (hi) + 64 (lo)
    for (int mi = ty; mi < 32; mi += 8) {
        const int m = m0 + mi;
        if (m >= M || l < m) continue;
        const int d = l - m, par = d & 1, i = d >> 1;
        if (i >= Lh) continue;
        uint32_t* rh = (uint32_t*)(ah + (((int64_t)(2 * m + par)) * Lh + i) * kTcCols);
        uint32_t* rl = (uint32_t*)(al + (((int64_t)(2 * m + par)) * Lh + i) * kTcCols);
        for (int b = tx; b < 64; b += 32) {
            const float2 v = tile[b][mi];
            uint16_t h0, l0, h1, l1;
            tc::split_bf16(v.x, h0, l0);
            tc::split_bf16(v.y, h1, l1);
            rh[b] = pack_bf16x2(h0, h1);
            rl[b] = pack_bf16x2(l0, l1);
        }
    }
}

}  // namespace hpx
