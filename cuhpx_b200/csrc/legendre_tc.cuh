// Tensor-core (tcgen05) Legendre contraction, BF16 or FP16 3-term split, FP32 accumulate.
//
// Same mathematics as the SIMT kernels in legendre.cuh (orthonormal Pbar_l^m,
// north/south folding, per-m contraction), mapped onto the 5th-generation
// tensor cores:
//
//  * the Pbar operand comes from the plan's resident table (fp16 or bf16 hi
//    and lo halves) by TMA, or, without the table, is generated on the fly by
//    producer warps running the FP64 three-term recurrence from the plan's
//    64-degree block seeds, rounded to FP32, split into hi + lo and stored
//    straight into shared memory; either way in the UMMA SWIZZLE_128B
//    (analysis) / SWIZZLE_64B (synthesis) canonical layout;
//  * the data operand (folded spectra for analysis, coefficients for
//    synthesis) is pre-split into hi/lo halves in global memory and brought in
//    by TMA (cp.async.bulk.tensor, 128B swizzle, no multicast);
//  * one thread issues tcgen05.mma (M=128, N=128, K=16) for the three products
//    into FP32 accumulators in TMEM; tcgen05.commit frees a pipeline stage
//    when its MMAs retire;
//  * epilogue warps (four, or eight with the table) drain TMEM (tcgen05.ld)
//    and add the accumulators.
//
// TMEM (512 columns) holds, per parity, a main accumulator (hi*hi) and a cross
// accumulator (hi*lo + lo*hi), at column (2 par + part) * 128.  The tensor
// cores' FP32 accumulation rounds toward zero at every MMA (an MMA adding
// 0.99 ulp to 1.0 leaves it unchanged), so each MMA into an accumulator can
// lose up to one ulp of its magnitude, always in the same direction; the bias
// grows with the number of MMAs chained into it.  Keeping the cross products,
// 2^-8 (bf16) or 2^-11 (fp16) smaller, in their own accumulator leaves one MMA
// per K-step on the main one, and the epilogue adds the two with
// round-to-nearest FP32.
//
// Analysis tile  = (m, 256 consecutive degrees): D_par[128 l][128 cols] +=
//                   Pbar_par[128 l][16 or 32 rings] * X_par[rings][128 cols]
// Synthesis tile = (m, 128 rings):   D_par[128 rings][128 cols] +=
//                   Pbar^T[128 rings][32 l] * A_par[32 l][128 cols]
// where par is the parity of l-m and cols = 2*map + {re, im}.
//
// Persistent kernels, one CTA per SM; each CTA runs its own contiguous range of
// the plan's tile list (tile_off[cta] .. tile_off[cta+1]), balanced on the host.
// Every mbarrier wait is bounded (tc_ptx.cuh); a timeout writes an error code
// to the plan's device flag and the kernel drains and returns.
#pragma once

#include <vector>

#include "legendre.cuh"
#include "tc_ptx.cuh"

namespace hpx {

// Optional per-CTA role timers (built only with -DHPX_TC_PROFILE): cycles each
// role spends waiting vs working, summed in registers and added to
// g_tc_prof once when the role finishes (so no global atomic sits between a
// role's stores and its release-arrive), read back by hpx_tc_profile_read.
// Slots: 0-2 MMA waits (TMA data, producers, accumulator free); 3 producer
// wait for a free stage, 4 producer work (wait end to arrive), 7 recurrence,
// 8 producer loop between chunks, 9 proxy fence + arrive; 5-6 epilogue wait
// and work; 10 the MMA thread's whole run.
#ifdef HPX_TC_PROFILE
constexpr int kTcpSlots = 16;
__device__ unsigned long long g_tc_prof[2][148 * 2][kTcpSlots];
#define TCP_DECL unsigned long long tcp_acc[kTcpSlots] = {}
#define TCP_T0(v) long long v = clock64()
#define TCP_SET(v) v = clock64()
#define TCP_ADD(k, slot, v) (tcp_acc[slot] += (unsigned long long)(clock64() - (v)))
#define TCP_FLUSH(k)                                                                          \
    do {                                                                                      \
        _Pragma("unroll") for (int i_ = 0; i_ < kTcpSlots; ++i_) if (tcp_acc[i_])             \
            atomicAdd(&g_tc_prof[k][blockIdx.x % 296][i_], tcp_acc[i_]);                      \
    } while (0)
#else
#define TCP_DECL
#define TCP_T0(v)
#define TCP_SET(v)
#define TCP_ADD(k, slot, v)
#define TCP_FLUSH(k)
#endif

constexpr int kTcCols = 128;      // N: columns per tile (64 maps)
constexpr int kTcThreads = 512;   // 16 warps
// Table-driven epilogues stage each warp's 32 rows x 16 columns in shared
// memory (row stride 20 floats: the row writes of 8 lanes fall on distinct
// banks) and store them as 8 rows x 64 contiguous bytes per instruction,
// instead of one 16-byte piece of each of 32 rows 512 bytes apart.
constexpr int kEpiStride = 20;
constexpr int kEpiStageFloats = 32 * kEpiStride;  // per warp
constexpr int kEpiStageBytes = 8 * kEpiStageFloats * 4;

// Tile words.  Analysis tile (m, y): degree tile jb = y & 255 and, with the
// resident table, the first pipeline chunk c0 = y >> 8 whose rings hold a
// nonzero table entry for the tile's degrees (the chunks before it are all
// zeros -- polar rings below the turning point -- and are skipped, which
// leaves the sums bit for bit unchanged).  Synthesis tile (m, y): ring block
// rb = y & 0xffff and first degree chunk c0 = y >> 16, likewise.
__host__ __device__ constexpr int fwd_tile_jb(int y) { return y & 255; }
__host__ __device__ constexpr int fwd_tile_c0(int y) { return y >> 8; }
__host__ __device__ constexpr int inv_tile_rb(int y) { return y & 0xffff; }
__host__ __device__ constexpr int inv_tile_c0(int y) { return y >> 16; }

// Failure-detection test builds only (-DHPX_TEST_WITHHOLD_TMA_LOADS): the TMA
// thread announces each stage's bytes but issues no load, so the MMA thread's
// bounded wait for the stage runs out, the kernel drains and returns, and
// hpx_plan_check reports HPX_ERR_TIMEOUT.  The product library never has it.
#ifdef HPX_TEST_WITHHOLD_TMA_LOADS
constexpr bool kWithholdTmaLoads = true;
#else
constexpr bool kWithholdTmaLoads = false;
#endif

// analysis: 6 stages of 16 rings (32 KB: A 4 x 4 KB, B 4 x 4 KB)
constexpr int kFStages = 6;
constexpr int kFRing = 16;
constexpr int kFStageBytes = 32768;
constexpr int kTcFwdDeg = 256;    // degrees per analysis tile (128 per parity)
constexpr int kFCoef = 256;       // per-producer-warp coefficient window (AlphaC)
constexpr int kFSmem = kFStages * kFStageBytes + 8 * kFCoef * 16 + 1024 + 1024;
// The table-driven analysis runs the same 192 KB as 3 stages of 32 rings
// (4 KB TMA boxes, two K-steps of 16 rings per stage): half the boxes, barrier
// round trips and commits per byte.  Producer-fed stages stay at 16 rings.
template <bool TAB>
constexpr int kFRingS = TAB ? 32 : kFRing;
template <bool TAB>
constexpr int kFStagesS = TAB ? 3 : kFStages;
template <bool TAB>
constexpr int kFStageBytesS = TAB ? 65536 : kFStageBytes;
static_assert(kFStagesS<true> * kFStageBytesS<true> == kFStages * kFStageBytes, "same stage memory");
// synthesis: 3 stages of 64 degrees (64 KB: A 4 x 8 KB, B 4 x 8 KB)
constexpr int kIStages = 3;
constexpr int kIStageBytes = 65536;
constexpr int kTcInvRings = 128;  // rings per synthesis tile
constexpr int kTcDegChunk = 64;   // degrees per synthesis stage (32 per parity)
constexpr int kISmem = kIStages * kIStageBytes + 8 * 64 * 16 + 1024 + kEpiStageBytes + 1024;
constexpr int kMaxStages = 6;
// Epilogue warps (4..4+n): 4 drain both parities; the table-driven kernels have
// no producer warps, so 8 drain one parity each (warp w reads TMEM lanes
// 32 (w mod 4) .. +31 either way).
template <bool TAB>
constexpr int kEpiWarps = TAB ? 8 : 4;
// One 32 x 16 block: lane r holds v[0..16) of row r; row r goes to row_ptr(r)
// (nullptr: skipped).  Ends with the warp's staging buffer free again.
template <typename RowPtr>
__device__ __forceinline__ void epi_store_block(float* stg, const float (&v)[16], int lane, RowPtr row_ptr) {
#pragma unroll
    for (int j = 0; j < 16; j += 4) *(float4*)(stg + lane * kEpiStride + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = k * 8 + (lane >> 2), q = lane & 3;
        float* dst = row_ptr(r);
        if (dst) *(float4*)(dst + 4 * q) = *(const float4*)(stg + r * kEpiStride + 4 * q);
    }
    __syncwarp();
}

// Host-side state of the tensor-core path, owned by the plan.
struct TcPlan {
    int active = 0;
    int nsm = 0;
    int* d_err = nullptr;     // device error flag written by bounded waits
    int2* d_fwd_tiles = nullptr;  // tiles grouped by CTA
    int* d_fwd_off = nullptr;     // CTA c runs tiles d_fwd_off[c] .. d_fwd_off[c+1]
    int n_fwd_tiles = 0, n_fwd_ctas = 0;
    int2* d_inv_tiles = nullptr;
    int* d_inv_off = nullptr;
    int n_inv_tiles = 0, n_inv_ctas = 0;
    int m_tc_end = 0;         // orders m < m_tc_end go through the tensor cores
    int table = 0;            // 1: Pbar read from the resident table, 0: generated by producer warps
    int Lt = 0;               // table row length (halves)
    size_t table_bytes = 0;
    size_t stream_fwd = 0, stream_inv = 0;  // table bytes one pass streams (TMA boxes of the tiles' chunks)
    uint16_t* d_table = nullptr;  // [m_tc_end][2 par][2 hl][2N][Lt]
    CUtensorMap tab_fwd{}, tab_inv{};
    int Lh = 0;               // rows per (m, parity) of the synthesis operand
    void* encode = nullptr;   // cuTensorMapEncodeTiled (driver entry point)
    // the tile lists in generation order and their costs, kept on the host so
    // that a new schedule (hpx_plan_set_schedule) can deal them again
    std::vector<int2> fwd_list, inv_list;
    std::vector<double> fwd_cost, inv_cost;
    int fwd_deal = 0, inv_deal = 0, ctas = 0;
};

// ------------------------------------------------------------------ shared layout
struct TcShared {
    uint64_t full_tma[kMaxStages];
    uint64_t full_prod[kMaxStages];
    uint64_t empty[kMaxStages];
    uint64_t acc_full[2];
    uint64_t acc_empty[2];
    uint64_t drain;
    uint32_t tmem_base;
};

__device__ __forceinline__ uint32_t pack_bf16x2(uint16_t a, uint16_t b) { return (uint32_t)a | ((uint32_t)b << 16); }

// x ~ hi + lo for two floats: hi = bf16_rn(x), lo = bf16_rn(x - hi) (packed conversions)
__device__ __forceinline__ uint32_t split_pair(float fa, float fb, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(fa, fb);
    const uint32_t hb = *(const uint32_t*)&h;
    const float ha = __uint_as_float(hb << 16), hbf = __uint_as_float(hb & 0xffff0000u);
    const __nv_bfloat162 l = __floats2bfloat162_rn(fa - ha, fb - hbf);
    lo = *(const uint32_t*)&l;
    return hb;
}
// the same with fp16 halves: hi = f16_rn(x), lo = f16_rn(x - hi)
__device__ __forceinline__ uint32_t split_pair_h(float fa, float fb, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(fa, fb);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(fa - hf.x, fb - hf.y);
    lo = *(const uint32_t*)&l;
    return *(const uint32_t*)&h;
}
template <bool F16>
__device__ __forceinline__ void split8f(const float* v, uint4& hi, uint4& lo) {
    if constexpr (F16) {
        hi.x = split_pair_h(v[0], v[1], lo.x);
        hi.y = split_pair_h(v[2], v[3], lo.y);
        hi.z = split_pair_h(v[4], v[5], lo.z);
        hi.w = split_pair_h(v[6], v[7], lo.w);
    } else {
        hi.x = split_pair(v[0], v[1], lo.x);
        hi.y = split_pair(v[2], v[3], lo.y);
        hi.z = split_pair(v[4], v[5], lo.z);
        hi.w = split_pair(v[6], v[7], lo.w);
    }
}

// 1 / 2^e(map) of the FP16 operand scale for the first kTcCols/2 maps (1 for BF16)
template <bool F16>
__device__ __forceinline__ void load_inv_scales(float* s_inv, const unsigned* __restrict__ vmax, float bound_mul,
                                                int nmaps) {
    const int b = threadIdx.x;
    if (b < kTcCols / 2) {
        float v = 1.f;
        if (F16 && b < nmaps) v = tc::pow2f(-tc::f16_scale_exp(__uint_as_float(vmax[b]) * bound_mul));
        s_inv[b] = v;
    }
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w)
                 : "memory");
}

// On exit (normal or after a timeout) the TMA thread waits, bounded, for the
// loads it issued into the last pipeline stages, so no bulk copy lands in
// shared memory after the CTA has finished.
__device__ __forceinline__ void tma_drain(TcShared* sh, int issued, int stages) {
    for (int k = 1; k <= stages && issued - k >= 0; ++k) {
        const int it = issued - k;
        tc::mbar_wait_quiet(&sh->full_tma[it % stages], (it / stages) & 1);
    }
}
// The MMA thread commits once more and waits, bounded, so that every MMA it
// issued has retired before TMEM is released.
__device__ __forceinline__ void mma_drain(TcShared* sh) {
    tc::mma_commit(&sh->drain);
    tc::mbar_wait_quiet(&sh->drain, 0);
}

// acc_arrivals: epilogue warps that drain one accumulator (4, or 8 when the
// table-driven kernels, which have no producer warps, split the two parities)
__device__ __forceinline__ void tc_setup(TcShared* sh, int stages, int prod_arrivals, int warp, int acc_arrivals) {
    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            tc::mbar_init(&sh->full_tma[s], 1);
            tc::mbar_init(&sh->full_prod[s], prod_arrivals);
            tc::mbar_init(&sh->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            tc::mbar_init(&sh->acc_full[a], 1);
            tc::mbar_init(&sh->acc_empty[a], acc_arrivals);
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
}

// Two independent block-normalised recurrences (64 degrees each) from their
// seeds, interleaved for latency hiding.  Every 16 degrees, emit(chain, s,
// even8, odd8) receives the FP32 values Pbar = c * q of 8 even and 8 odd degrees.
template <typename Emit>
__device__ __forceinline__ void gen2_fast(double2 sa, double2 sb, double xa, double xb, const AlphaC* __restrict__ ca,
                                          const AlphaC* __restrict__ cb, Emit&& emit) {
    double qa2 = 0.0, qa1 = 0.0, qb2 = 0.0, qb1 = 0.0;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        float ea[8], oa[8], eb[8], ob[8];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int i = s * 16 + k;
            const AlphaC A = ca[i];
            const AlphaC B = cb[i];
            double va, vb;
            if (i == 0) {
                va = sa.x;
                vb = sb.x;
            } else if (i == 1) {
                va = sa.y;
                vb = sb.y;
            } else {
                va = fma(A.alpha * xa, qa1, -qa2);
                vb = fma(B.alpha * xb, qb1, -qb2);
            }
            qa2 = qa1;
            qa1 = va;
            qb2 = qb1;
            qb1 = vb;
            const float fa = (float)va * A.c, fb = (float)vb * B.c;
            if (k & 1) {
                oa[k >> 1] = fa;
                ob[k >> 1] = fb;
            } else {
                ea[k >> 1] = fa;
                eb[k >> 1] = fb;
            }
        }
        emit(0, s, ea, oa);
        emit(1, s, eb, ob);
    }
}

// Reference-form recurrence with the l_s injection (orders whose first
// significant degree lies inside this block; rare), coefficients from global memory.
template <typename Emit>
__device__ __forceinline__ void gen1_slow(int chain, int m, int l0b, int L, int Lpad, int ls, double2 ps, double2 sd,
                                          double x, const double2* __restrict__ coef, Emit&& emit) {
    double p2 = 0.0, p1 = 0.0;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        float ev[8], od[8];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int i = s * 16 + k;
            const int l = l0b + i;
            double v;
            if (i == 0 && ls <= l0b) v = sd.x;
            else if (i == 1 && ls <= l0b) v = sd.y;
            else {
                const double2 ab = l < L && l >= m + 2 ? coef[(int64_t)m * Lpad + l] : make_double2(0.0, 0.0);
                v = (l < L) ? leg_step(l, ls, ps, ab.x, ab.y, x, p1, p2) : 0.0;
            }
            p2 = p1;
            p1 = v;
            if (k & 1) od[k >> 1] = (float)v; else ev[k >> 1] = (float)v;
        }
        emit(chain, s, ev, od);
    }
}

// ================================================================== resident table
// Legendre table of the tensor-core contraction: tab[m][par][hl][p][i] (2-byte
// halves; row length Lt, a multiple of 8) holds Pbar_l^m(z_p) for l = m + 2i +
// par, rounded from FP64 to FP32 and split into hi + lo halves (fp16 or bf16).
// The rows are l-contiguous, so TMA boxes of {64 i, 16 rings} (128B swizzle)
// and {32 i, 128 rings} (64B swizzle) land exactly in the analysis and
// synthesis A-operand layouts.  Thread per (m, north ring p >= first ring of
// m, 64-degree block), starting from the block seed (or, inside the block
// holding the first significant degree, from the start pair), as gen1_slow.
// Entries never written (rings before the first ring of m, degrees >= L)
// must be zero: the caller clears the table first.
template <bool F16>
__global__ void __launch_bounds__(128) k_legendre_table(int m_end, int L, int Lpad, Geom geo, int Lt,
                                                        const double* __restrict__ zr, const int* __restrict__ lstart,
                                                        const double2* __restrict__ pstart,
                                                        const double2* __restrict__ coef,
                                                        const double2* __restrict__ seeds, uint16_t* __restrict__ tab) {
    const int NP = geo.NP;
    const int nbk = seed_blocks(L);
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)m_end * nbk * NP) return;
    const int p = (int)(idx % NP);
    const int j = (int)((idx / NP) % nbk);
    const int m = (int)(idx / ((int64_t)NP * nbk));
    const int l0 = m + j * kSeedBlock;
    if (l0 >= L || p < geo.first_ring(m)) return;
    const int64_t mi = (int64_t)m * NP + p;
    const int ls = lstart[mi];
    const double2 ps = pstart[mi];
    const double2 sd = seeds[((int64_t)m * nbk + j) * NP + p];
    const double x = zr[p];
    double p1 = 0.0, p2 = 0.0;
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {  // 16 degrees -> 8 values of each parity
        uint32_t hi[2][4], lo[2][4];
#pragma unroll
        for (int k = 0; k < 16; k += 2) {
            float f[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int kk = q * 16 + k + u, l = l0 + kk;
                double v;
                if (kk == 0 && ls <= l0) v = sd.x;
                else if (kk == 1 && ls <= l0) v = sd.y;
                else {
                    const double2 ab = (l < L && l >= m + 2) ? coef[(int64_t)m * Lpad + l] : make_double2(0.0, 0.0);
                    v = (l < L) ? leg_step(l, ls, ps, ab.x, ab.y, x, p1, p2) : 0.0;
                }
                p2 = p1;
                p1 = v;
                f[u] = (float)v;
            }
            // f[0]: even offset (par 0), f[1]: odd offset (par 1), index i = 8q + k/2
            const int w = (k >> 1) >> 1, half = (k >> 1) & 1;
#pragma unroll
            for (int par = 0; par < 2; ++par) {
                uint16_t h, g;
                if (F16) tc::split_f16(f[par], h, g);
                else tc::split_bf16(f[par], h, g);
                if (half == 0) {
                    hi[par][w] = h;
                    lo[par][w] = g;
                } else {
                    hi[par][w] |= (uint32_t)h << 16;
                    lo[par][w] |= (uint32_t)g << 16;
                }
            }
        }
        const int i0 = j * (kSeedBlock / 2) + q * 8;
        if (i0 < Lt) {
#pragma unroll
            for (int par = 0; par < 2; ++par) {
                uint16_t* rh = tab + ((((int64_t)m * 2 + par) * 2 + 0) * NP + p) * Lt + i0;
                uint16_t* rl = tab + ((((int64_t)m * 2 + par) * 2 + 1) * NP + p) * Lt + i0;
                *(uint4*)rh = make_uint4(hi[par][0], hi[par][1], hi[par][2], hi[par][3]);
                *(uint4*)rl = make_uint4(lo[par][0], lo[par][1], lo[par][2], lo[par][3]);
            }
        }
    }
}

// First nonzero entry of each (m, ring) of the table: out[m * NP + p] = the
// smallest d = l - m whose hi half is nonzero in either parity, or 1 << 30.
// A zero hi half means a zero lo half too (|Pbar| below the smallest
// subnormal of the half type).  Block of 64 threads per (ring, m): warp w
// scans parity w.
__global__ void __launch_bounds__(64) k_table_first_nz(const uint16_t* __restrict__ tab, int NP, int Lt,
                                                       int* __restrict__ out) {
    const int p = blockIdx.x, m = blockIdx.y, par = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint16_t* row = tab + ((((int64_t)m * 2 + par) * 2 + 0) * NP + p) * Lt;
    int first = 1 << 30;
    for (int i0 = 0; i0 < Lt; i0 += 32) {
        const int i = i0 + lane;
        const unsigned nz = __ballot_sync(0xffffffffu, i < Lt && row[i] != 0);
        if (nz) {
            first = 2 * (i0 + __ffs(nz) - 1) + par;
            break;
        }
    }
    __shared__ int s_first[2];
    if (lane == 0) s_first[par] = first;
    __syncthreads();
    if (threadIdx.x == 0) out[(int64_t)m * NP + p] = min(s_first[0], s_first[1]);
}

// ================================================================== analysis
// Xh/Xl: bf16 [2M][NP][128] (hi and lo of S (par 0) and D (par 1)) via tensor maps.
// Tile (m, 256 degrees); pipeline chunk = 16 rings.  Stage layout:
//   A_par,hl (Pbar, MN-major SW128, 128 l x 16 rings, 4 KB) at (par*2+hl)*4096
//   B_par,hl (X,    MN-major SW128, 16 rings x 128 cols, 4 KB) at 16384 + (par*2+hl)*4096
// Producer warp w < 6 owns pipeline stage w and takes the chunks it = w (mod 6):
// a producer never runs more than one barrier phase ahead of the MMAs (with more
// producer groups than stages an mbarrier parity wait could pass on a stale
// phase).  Lane = (ring r = lane&15, block pair bp = lane>>4) runs the two
// blocks 2bp, 2bp+1 of its ring.
template <bool F16, bool TAB>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_leg_fwd_tc(const __grid_constant__ CUtensorMap xh_map, const __grid_constant__ CUtensorMap xl_map,
                 const __grid_constant__ CUtensorMap tab_map, int nmaps,
                 float* __restrict__ ycols, int L, int Lpad, Geom geo, const double* __restrict__ zr,
                 const int* __restrict__ lstart, const int* __restrict__ lsmax, const double2* __restrict__ pstart,
                 const double2* __restrict__ coef, const AlphaC* __restrict__ alphac, const double2* __restrict__ seeds,
                 const int2* __restrict__ tiles, const int* __restrict__ tile_off, const unsigned* __restrict__ fmax,
                 float wb, int* __restrict__ err) {
    __shared__ float s_inv[kTcCols / 2];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // align by pointer arithmetic on the shared array (keeps the shared address space known)
    unsigned char* base = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    unsigned char* stages = base;
    AlphaC* coef_s = (AlphaC*)(base + kFStages * kFStageBytes);
    TcShared* sh = (TcShared*)(base + kFStages * kFStageBytes + 8 * kFCoef * 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NP = geo.NP;
    const int nbk = seed_blocks(L);
    const int t_begin = tile_off[blockIdx.x], t_end = tile_off[blockIdx.x + 1];  // this CTA's tiles
    load_inv_scales<F16>(s_inv, fmax, wb, nmaps);
    tc_setup(sh, kFStagesS<TAB>, 1, warp, kEpiWarps<TAB>);
    const uint32_t tmem = sh->tmem_base;
    constexpr int RS = kFRingS<TAB>, NS = kFStagesS<TAB>, SB = kFStageBytesS<TAB>;
    // stage s: A (Pbar) at s SB, B (operand) at s SB + SB/2; within each, the
    // (par, hl) blocks are SB/8 apart and their two 64-wide halves SB/16 apart
    auto nchunks = [&](int m) { return (NP - geo.first_ring(m) + RS - 1) / RS; };

    if (warp == 0) {
        if (lane == 0) {
            tc::tma_prefetch_desc(&xh_map);
            tc::tma_prefetch_desc(&xl_map);
            if (TAB) tc::tma_prefetch_desc(&tab_map);
            int it = 0;
            for (int t = t_begin; t < t_end; ++t) {
                const int m = tiles[t].x, jb = fwd_tile_jb(tiles[t].y), c0 = fwd_tile_c0(tiles[t].y);
                const int t0 = geo.first_ring(m);
                const int nch = nchunks(m);
                for (int c = c0; c < nch; ++c, ++it) {
                    const int s = it % NS;
                    if (!tc::mbar_wait(&sh->empty[s], ((it / NS) & 1) ^ 1, err, 11)) goto tma_done;
                    unsigned char* st = stages + s * SB + SB / 2;
                    tc::mbar_arrive_tx(&sh->full_tma[s], TAB ? SB : SB / 2);
                    if (kWithholdTmaLoads) continue;
                    const int y = t0 + c * RS;  // rings past NP read as zeros (TMA out-of-bounds fill)
                    if (TAB) {
                        // A operand: Pbar for 128 degrees of each parity x RS rings, hi and lo
#pragma unroll
                        for (int ph = 0; ph < 4; ++ph)
#pragma unroll
                            for (int h = 0; h < 2; ++h)
                                tc::tma_load_3d(stages + s * SB + ph * (SB / 8) + h * (SB / 16), &tab_map,
                                                jb * (kTcFwdDeg / 2) + h * 64, y, 4 * m + ph, &sh->full_tma[s]);
                    }
#pragma unroll
                    for (int par = 0; par < 2; ++par)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            tc::tma_load_3d(st + (par * 2 + 0) * (SB / 8) + h * (SB / 16), &xh_map, h * 64, y,
                                            2 * m + par, &sh->full_tma[s]);
                            tc::tma_load_3d(st + (par * 2 + 1) * (SB / 8) + h * (SB / 16), &xl_map, h * 64, y,
                                            2 * m + par, &sh->full_tma[s]);
                        }
                }
            }
        tma_done:
            tma_drain(sh, it, NS);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            TCP_DECL;
            TCP_T0(role);
            const uint32_t idesc = F16 ? tc::idesc_f16(128, kTcCols, true, true) : tc::idesc_bf16(128, kTcCols, true, true);
            int it = 0, tcount = 0;
            for (int t = t_begin; t < t_end; ++t, ++tcount) {
                const int m = tiles[t].x, c0 = fwd_tile_c0(tiles[t].y);
                const int nch = nchunks(m);
                TCP_T0(w2);
                if (!tc::mbar_wait(&sh->acc_empty[0], (tcount & 1) ^ 1, err, 12)) break;
                TCP_ADD(0, 2, w2);
                tc::tc_fence_after();
                for (int c = c0; c < nch; ++c, ++it) {
                    const int s = it % NS;
                    const uint32_t ph = (it / NS) & 1;
                    TCP_T0(w0);
                    if (!tc::mbar_wait(&sh->full_tma[s], ph, err, 13)) goto mma_done;
                    TCP_ADD(0, 0, w0);
                    TCP_T0(w1);
                    if (!TAB && !tc::mbar_wait(&sh->full_prod[s], ph, err, 14)) goto mma_done;
                    TCP_ADD(0, 1, w1);
                    tc::tc_fence_after();
                    const uint32_t sa = tc::smem_u32(stages + s * SB);
                    const uint32_t sb = sa + SB / 2;
#pragma unroll
                    for (int par = 0; par < 2; ++par) {
                        const uint32_t dm = tmem + par * 2 * kTcCols, dc = dm + kTcCols;
#pragma unroll
                        for (int ks = 0; ks < RS / 16; ++ks) {
                            // K-step ks: rings 16 ks .. +15, 16 rows of 128 B into each 64-wide half
                            const uint32_t ko = ks * 2048;
                            const uint64_t ah = tc::smem_desc_sw128(sa + (par * 2 + 0) * (SB / 8) + ko, SB / 16, 1024);
                            const uint64_t al = tc::smem_desc_sw128(sa + (par * 2 + 1) * (SB / 8) + ko, SB / 16, 1024);
                            const uint64_t bh = tc::smem_desc_sw128(sb + (par * 2 + 0) * (SB / 8) + ko, SB / 16, 1024);
                            const uint64_t bl = tc::smem_desc_sw128(sb + (par * 2 + 1) * (SB / 8) + ko, SB / 16, 1024);
                            const uint32_t acc = (c > c0 || ks > 0) ? 1u : 0u;
                            tc::mma_bf16(dm, ah, bh, idesc, acc);
                            tc::mma_bf16(dc, ah, bl, idesc, acc);
                            tc::mma_bf16(dc, al, bh, idesc, 1u);
                        }
                    }
                    tc::mma_commit(&sh->empty[s]);
                }
                tc::mma_commit(&sh->acc_full[0]);
            }
        mma_done:
            mma_drain(sh);
            TCP_ADD(0, 10, role);
            TCP_FLUSH(0);
        }
    } else if (warp >= 4 && warp < 4 + kEpiWarps<TAB>) {
        // ------------------------------------------------ epilogue: TMEM -> ycols[m][l][128]
        // Each row (m, l) is written whole by one thread (512 contiguous bytes),
        // so no two CTAs write the same sector; k_tc_to_alm scatters the rows
        // into alm[b][l][m] with coalesced stores.
        TCP_DECL;
        const int ew = warp & 3;  // TMEM lanes 32*ew .. +31
        const int par_lo = kEpiWarps<TAB> == 8 ? (warp - 4) >> 2 : 0;
        const int par_hi = kEpiWarps<TAB> == 8 ? par_lo + 1 : 2;
        int tcount = 0;
        for (int t = t_begin; t < t_end; ++t, ++tcount) {
            const int m = tiles[t].x, jb = fwd_tile_jb(tiles[t].y);
            const int l0 = m + jb * kTcFwdDeg;
            TCP_T0(e0);
            if (!tc::mbar_wait_warp(&sh->acc_full[0], tcount & 1, err, 15)) break;
            if (lane == 0) TCP_ADD(0, 5, e0);
            TCP_T0(e1);
            tc::tc_fence_after();
            const int row = ew * 32 + lane;
#pragma unroll 1
            for (int par = par_lo; par < par_hi; ++par) {
                const int l = l0 + 2 * row + par;
                const uint32_t taddr = tmem + ((uint32_t)(ew * 32) << 16) + par * 2 * kTcCols;
#pragma unroll 1
                for (int c = 0; c < kTcCols; c += 16) {
                    float v[16], w[16];
                    tc::tmem_ld16(taddr + c, v);
                    tc::tmem_ld16(taddr + kTcCols + c, w);
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] += w[j];
                    if constexpr (TAB) {
#pragma unroll
                        for (int j = 0; j < 16; j += 2) {
                            const float sc = s_inv[(c + j) >> 1];
                            v[j] *= sc;
                            v[j + 1] *= sc;
                        }
                        float* stg = (float*)coef_s + (warp - 4) * kEpiStageFloats;
                        const int lr0 = l0 + 2 * ew * 32 + par;  // degree of row 0 of this warp
                        epi_store_block(stg, v, lane, [&](int r) -> float* {
                            const int lr = lr0 + 2 * r;
                            return (lr < L && HPX_INB(((int64_t)m * L + lr) * kTcCols + c + 15, kExtYcols, 13))
                                       ? ycols + ((int64_t)m * L + lr) * kTcCols + c
                                       : nullptr;
                        });
                    } else if (l < L && HPX_INB(((int64_t)m * L + l) * kTcCols + c + 15, kExtYcols, 13)) {
                        float* dst = ycols + ((int64_t)m * L + l) * kTcCols + c;
#pragma unroll
                        for (int j = 0; j < 16; j += 4) {
                            const float s0 = s_inv[(c + j) >> 1], s1 = s_inv[((c + j) >> 1) + 1];
                            *(float4*)(dst + j) = make_float4(v[j] * s0, v[j + 1] * s0, v[j + 2] * s1, v[j + 3] * s1);
                        }
                    }
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sh->acc_empty[0]);
            if (lane == 0) TCP_ADD(0, 6, e1);
        }
        if (lane == 0) TCP_FLUSH(0);
    } else if (!TAB && warp >= 8 && warp < 8 + kFStages) {
        // ------------------------------------------------ Pbar producers
        TCP_DECL;
        const int pw = warp - 8;
        const int r = lane & 15, bp = lane >> 4;
        AlphaC* cfw = coef_s + pw * kFCoef;
        int t = t_begin, c = 0, it = 0, cur_tile = -1;
        int m = 0, jb = 0, t0 = 0, nch = 0;
        auto load_tile = [&]() {
            if (t < t_end) {
                const int2 tt = tiles[t];
                m = tt.x;
                jb = fwd_tile_jb(tt.y);
                t0 = geo.first_ring(m);
                nch = nchunks(m);
            }
        };
        auto to_mine = [&]() {
            while (t < t_end) {
                if (c >= nch) {
                    ++t;
                    c = 0;
                    load_tile();
                    continue;
                }
                if (it % kFStages == pw) return;
                ++c;
                ++it;
            }
        };
        struct In {
            double2 s0, s1;
            double x;
            int p, l0, tile, m, it, lsm;
        };
        auto fetch = [&]() {
            In in;
            in.p = t0 + c * kFRing + r;
            in.l0 = m + jb * kTcFwdDeg;
            in.tile = t;
            in.m = m;
            in.it = it;
            const int b0 = in.l0 + 128 * bp, b1 = b0 + 64;
            const bool v = in.p < NP;
            const int64_t sb = ((int64_t)m * nbk + (b0 - m) / kSeedBlock) * NP + in.p;
            in.s0 = (v && b0 < L) ? seeds[sb] : make_double2(0.0, 0.0);
            in.s1 = (v && b1 < L) ? seeds[sb + NP] : make_double2(0.0, 0.0);
            in.x = v ? zr[in.p] : 0.0;
            in.lsm = lsmax[m];
            return in;
        };
        load_tile();
        to_mine();
        if (t < t_end) {
            In cur = fetch();
            TCP_T0(lp);
            while (true) {
                const int s = cur.it % kFStages;
                if (cur.tile != cur_tile) {
                    // coefficient window of this tile's 256 degrees
                    __syncwarp();
                    const AlphaC* src = alphac + (int64_t)cur.m * Lpad + cur.l0;
                    for (int i = lane; i < kFCoef; i += 32) cfw[i] = src[i];
                    __syncwarp();
                    cur_tile = cur.tile;
                }
                if (lane == 0) TCP_ADD(0, 8, lp);
                TCP_T0(pw0);
                if (!tc::mbar_wait_warp(&sh->empty[s], ((cur.it / kFStages) & 1) ^ 1, err, 16)) break;
                if (lane == 0) TCP_ADD(0, 3, pw0);
                TCP_T0(pw1);
                const uint32_t sa = tc::smem_u32(stages + s * kFStageBytes);
                const uint32_t gbase = (uint32_t)((r >> 3) * 1024);
                auto emit = [&](int chain, int sidx, const float* ev, const float* od) {
                    const int q = 2 * bp + chain;  // 64-degree block within the tile
                    uint4 eh, el, oh, ol;
                    split8f<F16>(ev, eh, el);
                    split8f<F16>(od, oh, ol);
                    const uint32_t off = (uint32_t)((q >> 1) * 2048) + gbase + tc::sw128_offset(r & 7, ((q & 1) << 2) + sidx);
                    st_shared_v4(sa + 0 * 4096 + off, eh);
                    st_shared_v4(sa + 1 * 4096 + off, el);
                    st_shared_v4(sa + 2 * 4096 + off, oh);
                    st_shared_v4(sa + 3 * 4096 + off, ol);
                };
                const int b0 = cur.l0 + 128 * bp;
                const bool fast = cur.l0 >= cur.lsm;  // warp-uniform
                TCP_T0(gg);
                if (fast) {
                    gen2_fast(cur.s0, cur.s1, cur.x, cur.x, cfw + 128 * bp, cfw + 128 * bp + 64, emit);
                } else {
                    const bool v = cur.p < NP;
                    const int64_t mi = (int64_t)cur.m * NP + (v ? cur.p : 0);
                    const int ls = v ? lstart[mi] : L;
                    const double2 ps = v ? pstart[mi] : make_double2(0.0, 0.0);
                    gen1_slow(0, cur.m, b0, L, Lpad, ls, ps, cur.s0, v ? cur.x : 0.0, coef, emit);
                    gen1_slow(1, cur.m, b0 + 64, L, Lpad, ls, ps, cur.s1, v ? cur.x : 0.0, coef, emit);
                }
                if (lane == 0) TCP_ADD(0, 7, gg);
                TCP_T0(ff);
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh->full_prod[s]);
                if (lane == 0) TCP_ADD(0, 9, ff);
                if (lane == 0) TCP_ADD(0, 4, pw1);
                TCP_SET(lp);
                // next chunk's inputs: issued after this chunk is published, so the
                // proxy fence and the release-arrive above never wait on them
                ++c;
                ++it;
                to_mine();
                if (t >= t_end) break;
                cur = fetch();
            }
        }
        if (lane == 0) TCP_FLUSH(0);
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
// Tile (m, 128 rings); pipeline chunk = one 64-degree seed block.  Stage:
//   A_par,hl (Pbar^T, K-major SW64, 128 rings x 32 l, 8 KB) at (par*2+hl)*8192
//   B_par,hl (coefficients, MN-major SW128, 32 l x 128 cols, 8 KB) at 32768 + ...
// Chunk it goes to producer pair g = it mod 3 (warps 8+2g, 9+2g), which owns
// stage g (one barrier phase of run-ahead at most); lane runs rings 32w + lane
// and 64 + 32w + lane of the tile.
template <bool F16, bool TAB>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_leg_inv_tc(const __grid_constant__ CUtensorMap ah_map, const __grid_constant__ CUtensorMap al_map,
                 const __grid_constant__ CUtensorMap tab_map, const __grid_constant__ CUtensorMap spec_map,
                 float* __restrict__ spec, int C, int nmaps, int L, int M, int Lpad, Geom geo,
                 const double* __restrict__ zr, const int* __restrict__ lstart, const int* __restrict__ lsmax,
                 const double2* __restrict__ pstart, const double2* __restrict__ coef,
                 const AlphaC* __restrict__ alphac, const double2* __restrict__ seeds, const int2* __restrict__ tiles,
                 const int* __restrict__ tile_off, const unsigned* __restrict__ amax, int* __restrict__ err) {
    __shared__ float s_inv[kTcCols / 2];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // align by pointer arithmetic on the shared array (keeps the shared address space known)
    unsigned char* base = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
    unsigned char* stages = base;
    AlphaC* coef_s = (AlphaC*)(base + kIStages * kIStageBytes);
    TcShared* sh = (TcShared*)(base + kIStages * kIStageBytes + 8 * 64 * 16);
    float* epi_stage = (float*)(base + kIStages * kIStageBytes + 8 * 64 * 16 + 1024);  // table mode
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int NP = geo.NP;
    const int nbk = seed_blocks(L);
    const int t_begin = tile_off[blockIdx.x], t_end = tile_off[blockIdx.x + 1];  // this CTA's tiles
    load_inv_scales<F16>(s_inv, amax, 1.f, nmaps);
    tc_setup(sh, kIStages, 2, warp, kEpiWarps<TAB>);
    const uint32_t tmem = sh->tmem_base;
    auto nchunks = [&](int m) { return m < L ? (L - m + kTcDegChunk - 1) / kTcDegChunk : 0; };

    if (warp == 0) {
        if (lane == 0) {
            tc::tma_prefetch_desc(&ah_map);
            tc::tma_prefetch_desc(&al_map);
            if (TAB) tc::tma_prefetch_desc(&tab_map);
            int it = 0;
            for (int t = t_begin; t < t_end; ++t) {
                const int m = tiles[t].x, rb = inv_tile_rb(tiles[t].y), c0 = inv_tile_c0(tiles[t].y);
                const int t0 = geo.first_ring(m);
                const int nch = nchunks(m);
                for (int c = c0; c < nch; ++c, ++it) {
                    const int s = it % kIStages;
                    if (!tc::mbar_wait(&sh->empty[s], ((it / kIStages) & 1) ^ 1, err, 21)) goto tma_done;
                    unsigned char* st = stages + s * kIStageBytes + 32768;
                    tc::mbar_arrive_tx(&sh->full_tma[s], TAB ? 65536 : 32768);
                    if (kWithholdTmaLoads) continue;
                    if (TAB) {
                        // A operand: Pbar^T for 128 rings x 32 degrees of each parity, hi and lo
#pragma unroll
                        for (int ph = 0; ph < 4; ++ph)
                            tc::tma_load_3d(stages + s * kIStageBytes + ph * 8192, &tab_map, c * (kTcDegChunk / 2),
                                            t0 + rb, 4 * m + ph, &sh->full_tma[s]);
                    }
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
            tma_drain(sh, it, kIStages);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            TCP_DECL;
            TCP_T0(role);
            const uint32_t idesc = F16 ? tc::idesc_f16(128, kTcCols, false, true) : tc::idesc_bf16(128, kTcCols, false, true);
            int it = 0, tcount = 0;
            for (int t = t_begin; t < t_end; ++t, ++tcount) {
                const int m = tiles[t].x, c0 = inv_tile_c0(tiles[t].y);
                const int nch = nchunks(m);
                TCP_T0(w2);
                if (!tc::mbar_wait(&sh->acc_empty[0], (tcount & 1) ^ 1, err, 22)) break;
                TCP_ADD(1, 2, w2);
                tc::tc_fence_after();
                for (int c = c0; c < nch; ++c, ++it) {
                    const int s = it % kIStages;
                    const uint32_t ph = (it / kIStages) & 1;
                    TCP_T0(w0);
                    if (!tc::mbar_wait(&sh->full_tma[s], ph, err, 23)) goto mma_done;
                    TCP_ADD(1, 0, w0);
                    TCP_T0(w1);
                    if (!TAB && !tc::mbar_wait(&sh->full_prod[s], ph, err, 24)) goto mma_done;
                    TCP_ADD(1, 1, w1);
                    tc::tc_fence_after();
                    const uint32_t sa = tc::smem_u32(stages + s * kIStageBytes);
                    const uint32_t sb = sa + 32768;
#pragma unroll
                    for (int par = 0; par < 2; ++par) {
                        const uint32_t dm = tmem + par * 2 * kTcCols, dc = dm + kTcCols;
#pragma unroll
                        for (int ks = 0; ks < 2; ++ks) {
                            const uint64_t ah = tc::smem_desc_kmajor_sw64(sa + (par * 2 + 0) * 8192 + ks * 32, 512);
                            const uint64_t al = tc::smem_desc_kmajor_sw64(sa + (par * 2 + 1) * 8192 + ks * 32, 512);
                            const uint64_t bh = tc::smem_desc_sw128(sb + (par * 2 + 0) * 8192 + ks * 2048, 4096, 1024);
                            const uint64_t bl = tc::smem_desc_sw128(sb + (par * 2 + 1) * 8192 + ks * 2048, 4096, 1024);
                            const uint32_t acc = (c > c0 || ks > 0) ? 1u : 0u;
                            tc::mma_bf16(dm, ah, bh, idesc, acc);
                            tc::mma_bf16(dc, ah, bl, idesc, acc);
                            tc::mma_bf16(dc, al, bh, idesc, 1u);
                        }
                    }
                    tc::mma_commit(&sh->empty[s]);
                }
                tc::mma_commit(&sh->acc_full[0]);
            }
        mma_done:
            mma_drain(sh);
            TCP_ADD(1, 10, role);
            TCP_FLUSH(1);
        }
    } else if (warp >= 4 && warp < 4 + kEpiWarps<TAB>) {
        // ------------------------------------------------ epilogue: TMEM -> spec (E, O)
        TCP_DECL;
        const int ew = warp & 3;  // TMEM lanes 32*ew .. +31
        const int par_lo = kEpiWarps<TAB> == 8 ? (warp - 4) >> 2 : 0;
        const int par_hi = kEpiWarps<TAB> == 8 ? par_lo + 1 : 2;
        int tcount = 0;
        for (int t = t_begin; t < t_end; ++t, ++tcount) {
            const int m = tiles[t].x, rb = inv_tile_rb(tiles[t].y);
            const int t0 = geo.first_ring(m);
            const int rr = rb + ew * 32 + lane;
            const int p = t0 + rr;
            TCP_T0(e0);
            if (!tc::mbar_wait_warp(&sh->acc_full[0], tcount & 1, err, 25)) break;
            if (lane == 0) TCP_ADD(1, 5, e0);
            TCP_T0(e1);
            tc::tc_fence_after();
#pragma unroll 1
            for (int par = par_lo; par < par_hi; ++par) {
                float* dst = spec + (((int64_t)m * 2 + par) * NP + p) * C;
                const uint32_t taddr = tmem + ((uint32_t)(ew * 32) << 16) + par * 2 * kTcCols;
#pragma unroll 1
                for (int c = 0; c < kTcCols; c += 16) {
                    float v[16], w[16];
                    tc::tmem_ld16(taddr + c, v);
                    tc::tmem_ld16(taddr + kTcCols + c, w);
#pragma unroll
                    for (int j = 0; j < 16; ++j) v[j] += w[j];
                    if constexpr (TAB) {
#pragma unroll
                        for (int j = 0; j < 16; j += 2) {
                            const float sc = s_inv[(c + j) >> 1];
                            v[j] *= sc;
                            v[j + 1] *= sc;
                        }
                        // the warp's 32 rings x 16 columns, dense in the 64-byte swizzle of
                        // spec_map, go out as one TMA store (rings past NP are clipped)
                        unsigned char* stg = (unsigned char*)(epi_stage + (warp - 4) * kEpiStageFloats);
                        if (lane == 0) tc::bulk_wait_read0();  // the previous store has read the buffer
                        __syncwarp();
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            *(float4*)(stg + tc::sw64_offset(lane, j)) =
                                make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                        tc::fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) {
                            tc::tma_store_3d(&spec_map, stg, c, t0 + rb + ew * 32, 2 * m + par);
                            tc::bulk_commit();
                        }
                    } else if (p < NP && c < C && HPX_INB(dst - spec + c + 15, kExtSpec, 14)) {
#pragma unroll
                        for (int j = 0; j < 16; j += 4) {
                            const float s0 = s_inv[(c + j) >> 1], s1 = s_inv[((c + j) >> 1) + 1];
                            *(float4*)(dst + c + j) = make_float4(v[j] * s0, v[j + 1] * s0, v[j + 2] * s1, v[j + 3] * s1);
                        }
                    }
                }
            }
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&sh->acc_empty[0]);
            if (lane == 0) TCP_ADD(1, 6, e1);
        }
        if (TAB && lane == 0) tc::bulk_wait0();  // every TMA store of this warp is done
        if (lane == 0) TCP_FLUSH(1);
    } else if (!TAB && warp >= 8 && warp < 8 + 2 * kIStages) {
        // ------------------------------------------------ Pbar^T producers
        TCP_DECL;
        const int pw = warp - 8;
        const int g = pw >> 1, w = pw & 1;
        AlphaC* cfw = coef_s + pw * 64;
        const int r0 = 32 * w + lane, r1 = 64 + 32 * w + lane;  // tile rows of the two chains
        int t = t_begin, c = 0, it = 0;
        int m = 0, rb = 0, t0 = 0, nch = 0;
        auto load_tile = [&]() {
            if (t < t_end) {
                const int2 tt = tiles[t];
                m = tt.x;
                rb = inv_tile_rb(tt.y);
                t0 = geo.first_ring(m);
                nch = nchunks(m);
            }
        };
        auto to_mine = [&]() {
            while (t < t_end) {
                if (c >= nch) {
                    ++t;
                    c = 0;
                    load_tile();
                    continue;
                }
                if (it % kIStages == g) return;
                ++c;
                ++it;
            }
        };
        struct In {
            double2 s0, s1;
            double x0, x1;
            AlphaC c0, c1;
            int p0, p1, l0b, m, it, lsm;
        };
        auto fetch = [&]() {
            In in;
            in.m = m;
            in.it = it;
            in.l0b = m + c * kTcDegChunk;
            in.p0 = t0 + rb + r0;
            in.p1 = t0 + rb + r1;
            const int64_t sb = ((int64_t)m * nbk + c) * NP;
            in.s0 = in.p0 < NP ? seeds[sb + in.p0] : make_double2(0.0, 0.0);
            in.s1 = in.p1 < NP ? seeds[sb + in.p1] : make_double2(0.0, 0.0);
            in.x0 = in.p0 < NP ? zr[in.p0] : 0.0;
            in.x1 = in.p1 < NP ? zr[in.p1] : 0.0;
            const AlphaC* src = alphac + (int64_t)m * Lpad + in.l0b;
            in.c0 = src[lane];
            in.c1 = src[lane + 32];
            in.lsm = lsmax[m];
            return in;
        };
        load_tile();
        to_mine();
        if (t < t_end) {
            In cur = fetch();
            TCP_T0(lp);
            while (true) {
                const int s = cur.it % kIStages;
                if (lane == 0) TCP_ADD(1, 8, lp);
                TCP_T0(pw0);
                if (!tc::mbar_wait_warp(&sh->empty[s], ((cur.it / kIStages) & 1) ^ 1, err, 26)) break;
                if (lane == 0) TCP_ADD(1, 3, pw0);
                TCP_T0(pw1);
                __syncwarp();
                cfw[lane] = cur.c0;
                cfw[lane + 32] = cur.c1;
                __syncwarp();
                const uint32_t sa = tc::smem_u32(stages + s * kIStageBytes);
                auto emit = [&](int chain, int sidx, const float* ev, const float* od) {
                    const int rr = chain ? r1 : r0;
                    uint4 eh, el, oh, ol;
                    split8f<F16>(ev, eh, el);
                    split8f<F16>(od, oh, ol);
                    const uint32_t off = (uint32_t)((rr >> 3) * 512) + tc::sw64_offset(rr & 7, sidx);
                    st_shared_v4(sa + 0 * 8192 + off, eh);
                    st_shared_v4(sa + 1 * 8192 + off, el);
                    st_shared_v4(sa + 2 * 8192 + off, oh);
                    st_shared_v4(sa + 3 * 8192 + off, ol);
                };
                TCP_T0(gg);
                if (cur.l0b >= cur.lsm) {
                    gen2_fast(cur.s0, cur.s1, cur.x0, cur.x1, cfw, cfw, emit);
                } else {
                    const bool v0 = cur.p0 < NP, v1 = cur.p1 < NP;
                    const int64_t mb = (int64_t)cur.m * NP;
                    gen1_slow(0, cur.m, cur.l0b, L, Lpad, v0 ? lstart[mb + cur.p0] : L,
                              v0 ? pstart[mb + cur.p0] : make_double2(0.0, 0.0), cur.s0, cur.x0, coef, emit);
                    gen1_slow(1, cur.m, cur.l0b, L, Lpad, v1 ? lstart[mb + cur.p1] : L,
                              v1 ? pstart[mb + cur.p1] : make_double2(0.0, 0.0), cur.s1, cur.x1, coef, emit);
                }
                if (lane == 0) TCP_ADD(1, 7, gg);
                TCP_T0(ff);
                tc::fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(&sh->full_prod[s]);
                if (lane == 0) TCP_ADD(1, 9, ff);
                if (lane == 0) TCP_ADD(1, 4, pw1);
                TCP_SET(lp);
                ++c;
                ++it;
                to_mine();
                if (t >= t_end) break;
                cur = fetch();
            }
        }
        if (lane == 0) TCP_FLUSH(1);
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
// amax != nullptr: fp16 halves of the values times 2^e(map), e from the map's
// max |a| (k_alm_maxabs); otherwise bf16 halves.
__global__ void k_alm_to_tc(const float* __restrict__ alm, int nmaps, int L, int M, int Lh,
                            uint16_t* __restrict__ ah, uint16_t* __restrict__ al, const unsigned* __restrict__ amax) {
    __shared__ float2 tile[64][33];
    __shared__ float s_sc[64];
    const int m0 = blockIdx.x * 32, l = blockIdx.y;
    if (l < m0) return;  // only m <= l is used: nothing to convert in this block
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    // all loads of the thread are issued before the first shared-memory store
    float2 vv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int i = ty + 8 * k, m = m0 + tx;
        vv[k] = make_float2(0.f, 0.f);
        if (i < nmaps && m < M && m <= l && l < L && HPX_INB(2 * (((int64_t)i * L + l) * M + m) + 1, kExtAlm, 9))
            vv[k] = *(const float2*)(alm + 2 * (((int64_t)i * L + l) * M + m));
    }
    if (amax && ty < 2) {
        const int b = ty * 32 + tx;
        s_sc[b] = tc::pow2f(tc::f16_scale_exp(__uint_as_float(b < nmaps ? amax[b] : 0u)));
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) tile[ty + 8 * k][tx] = vv[k];
    __syncthreads();
    // each warp writes rows for 4 m's: 128 columns as 64 bf16x2 (hi) + 64 (lo)
    for (int mi = ty; mi < 32; mi += 8) {
        const int m = m0 + mi;
        if (m >= M || l < m) continue;
        const int d = l - m, par = d & 1, i = d >> 1;
        if (i >= Lh || !HPX_INB((((int64_t)(2 * m + par)) * Lh + i) * kTcCols + kTcCols - 1, kExtOperA, 10)) continue;
        uint32_t* rh = (uint32_t*)(ah + (((int64_t)(2 * m + par)) * Lh + i) * kTcCols);
        uint32_t* rl = (uint32_t*)(al + (((int64_t)(2 * m + par)) * Lh + i) * kTcCols);
        for (int b = tx; b < 64; b += 32) {
            const float2 v = tile[b][mi];
            uint16_t h0, l0, h1, l1;
            if (amax) {
                const float sc = s_sc[b];
                tc::split_f16(v.x * sc, h0, l0);
                tc::split_f16(v.y * sc, h1, l1);
            } else {
                tc::split_bf16(v.x, h0, l0);
                tc::split_bf16(v.y, h1, l1);
            }
            rh[b] = pack_bf16x2(h0, h1);
            rl[b] = pack_bf16x2(l0, l1);
        }
    }
}

// ycols[m][l][2b + {re, im}] (analysis output of the tensor cores, orders
// m < m_end) -> alm[b][l][m] (FP32 complex), storing or (accumulate) adding;
// l < m entries are set to zero unless accumulating.  Grid (ceil(m_end/32), L),
// block 32 x 8; the transpose goes through shared memory so that both the
// 512-byte row reads and the 32-order stores are coalesced.
__global__ void k_tc_to_alm(const float* __restrict__ ycols, int nmaps, int L, int M, int m_end,
                            float* __restrict__ alm, int accumulate) {
    __shared__ float2 tile[64][33];
    const int m0 = blockIdx.x * 32, l = blockIdx.y;
    const int tx = threadIdx.x, ty = threadIdx.y;
    // all loads of the thread are issued before the first shared-memory store
    float2 vv[4][2];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int m = m0 + ty + 8 * k;
        const bool live = m < m_end && m <= l && HPX_INB(((int64_t)m * L + l) * kTcCols + kTcCols - 1, kExtYcols, 11);
        const float2* row = (const float2*)(ycols + ((int64_t)m * L + l) * kTcCols);
#pragma unroll
        for (int h = 0; h < 2; ++h) vv[k][h] = live ? row[tx + 32 * h] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int h = 0; h < 2; ++h) tile[tx + 32 * h][ty + 8 * k] = vv[k][h];
    __syncthreads();
    const int m = m0 + tx;
    if (m >= m_end) return;
    for (int b = ty; b < nmaps && b < 64; b += 8) {
        if (!HPX_INB(2 * (((int64_t)b * L + l) * M + m) + 1, kExtAlm, 12)) continue;
        float2* dst = (float2*)(alm + 2 * (((int64_t)b * L + l) * M + m));
        float2 v = tile[b][tx];
        if (accumulate) {
            const float2 q = *dst;
            v.x += q.x;
            v.y += q.y;
        }
        *dst = v;
    }
}

}  // namespace hpx
