// Thin inline-PTX layer for the sm_100a tensor-core (tcgen05) kernels:
// TMEM allocation, UMMA shared-memory / instruction descriptors, MMA issue and
// commit, TMEM loads, mbarriers with bounded waits, and TMA tile loads.
//
// Every wait here is bounded: after kWaitLimitNs of %globaltimer time it records
// an error code in the caller's flag and gives up, so a broken pipeline ends
// the kernel with a status the host can read instead of hanging the GPU.  Polls
// suspend in hardware (suspend-time hint), and the flag and the clock are only
// read every 16 polls, so waiting warps cost almost nothing.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hpx {
namespace tc {

// Limit of every bounded wait: 2 s.  The failure-detection test builds a copy
// of the library with a 1 ms limit (-DHPX_WAIT_LIMIT_NS=1000000ull).
#ifndef HPX_WAIT_LIMIT_NS
#define HPX_WAIT_LIMIT_NS 2000000000ull
#endif
constexpr uint64_t kWaitLimitNs = HPX_WAIT_LIMIT_NS;

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// ---------------------------------------------------------------- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::); }
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
// try_wait with a suspend-time hint: a waiting thread is parked by the hardware
// (for at most kSuspendHintNs) until the phase completes, instead of spinning
// and taking issue slots from the producer warps on the same SM sub-partition.
constexpr uint32_t kSuspendHintNs = 20000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}
// Bounded wait; on timeout sets *err (if not set) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 15) == 0) {
            if (*(volatile int*)err) return false;
            if (globaltimer_ns() - t0 > kWaitLimitNs) {
                atomicCAS(err, 0, code);
                return false;
            }
        }
    }
}

// Bounded wait without an error flag (exit drains): true if the phase completed.
__device__ __forceinline__ bool mbar_wait_quiet(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 15) == 0 && globaltimer_ns() - t0 > kWaitLimitNs) return false;
    }
}

// Warp-uniform bounded wait: lane 0 polls, every lane gets the same answer, so
// warp-collective instructions after it never see a partial warp.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, int* err, int code) {
    int ok = 1;
    if ((threadIdx.x & 31) == 0) ok = mbar_wait(bar, parity, err, code) ? 1 : 0;
    ok = __shfl_sync(0xffffffffu, ok, 0);
    return ok != 0;
}

// ---------------------------------------------------------------- fences
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// ---------------------------------------------------------------- TMEM
// Warp-wide: allocate ncols TMEM columns, address written to *dst (smem).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread i of the warp gets lane (base+i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---------------------------------------------------------------- descriptors
// UMMA shared-memory descriptor, SWIZZLE_128B, sm_100 (version 1).
//   lbo/sbo in bytes; for MN-major operands lbo = stride between 64-element
//   (128-byte) MN atoms and sbo = stride between groups of 8 K rows; for
//   K-major operands sbo = stride between groups of 8 M/N rows, lbo unused.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // version for sm_100
    d |= (uint64_t)layout << 61;
    return d;
}
constexpr uint32_t kLayoutSW128 = 2;
constexpr uint32_t kLayoutSW64 = 4;
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return smem_desc(saddr, lbo, sbo, kLayoutSW128);
}
// K-major, SWIZZLE_64B: rows of 64 bytes, 8-row groups `sbo` bytes apart.
__device__ __forceinline__ uint64_t smem_desc_kmajor_sw64(uint32_t saddr, uint32_t sbo) {
    return smem_desc(saddr, 16, sbo, kLayoutSW64);
}

// Instruction descriptor for kind::f16 with BF16 A/B, FP32 accumulate.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4)                      // D format F32
           | (1u << 7)                    // A format BF16
           | (1u << 10)                   // B format BF16
           | ((a_mn ? 1u : 0u) << 15)     // A major
           | ((b_mn ? 1u : 0u) << 16)     // B major
           | ((uint32_t)(N >> 3) << 17)   // N
           | ((uint32_t)(M >> 4) << 24);  // M
}

// Instruction descriptor for kind::f16 with FP16 A/B (format code 0), FP32 accumulate.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4)                      // D format F32
           | ((a_mn ? 1u : 0u) << 15)     // A major
           | ((b_mn ? 1u : 0u) << 16)     // B major
           | ((uint32_t)(N >> 3) << 17)   // N
           | ((uint32_t)(M >> 4) << 24);  // M
}

// D[tmem] (+)= A[smem] * B[smem]; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrive on an mbarrier once all previously issued MMAs of this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---------------------------------------------------------------- TMA
__device__ __forceinline__ void tma_load_3d(void* smem_dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(smem_dst)),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
// TMA tiled store shared -> global, in the issuing thread's bulk async-group;
// elements outside the tensor are not written.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* smem_src, int x, int y, int z) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n" ::"l"((uint64_t)map),
                 "r"(smem_u32(smem_src)), "r"(x), "r"(y), "r"(z)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// wait until the thread's committed bulk stores have read their shared-memory source
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// ... and until they are complete
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"((uint64_t)map) : "memory");
}

// ---------------------------------------------------------------- bf16 split
// x = hi + lo with hi = bf16(x) and lo = bf16(x - hi): about 16 significant bits.
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
    __nv_bfloat16 h = __float2bfloat16_rn(x);
    __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

// ---------------------------------------------------------------- fp16 split
// x = hi + lo with hi = f16(x) and lo = f16(x - hi): about 22 significant bits
// for |x| in [2^-3, 2^15]; below that lo is subnormal and the absolute error
// stays under 2^-25.
__device__ __forceinline__ void split_f16(float x, uint16_t& hi, uint16_t& lo) {
    const __half h = __float2half_rn(x);
    const __half l = __float2half_rn(x - __half2float(h));
    hi = __half_as_ushort(h);
    lo = __half_as_ushort(l);
}

// Power-of-two scale of the FP16 operands of one map: e such that a bound B
// on the map's operand magnitudes maps below 2^14 (fp16 max is 65504), so
// every value keeps 22 bits down to 2^-17 of the bound.  0, inf and NaN
// bounds give e = 0.
__device__ __forceinline__ int f16_scale_exp(float bound) {
    if (!(bound > 0.f) || !(bound < 3.0e38f)) return 0;
    int ex = 0;
    (void)frexpf(bound, &ex);  // bound < 2^ex
    const int e = 14 - ex;
    return e < -120 ? -120 : (e > 120 ? 120 : e);
}
// 2^e for |e| <= 126, exactly
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }

// Byte offset of the 16-byte chunk `chunk` (0..7) of row `row` inside a
// SWIZZLE_128B atom (8 rows x 128 bytes), the pattern TMA and UMMA share.
__device__ __forceinline__ uint32_t sw128_offset(int row, int chunk) {
    return (uint32_t)(row * 128 + ((chunk ^ (row & 7)) << 4));
}
// Same for SWIZZLE_64B (rows of 64 bytes, chunk 0..3, 512-byte atoms).
__device__ __forceinline__ uint32_t sw64_offset(int row, int chunk) {
    return (uint32_t)(row * 64 + ((chunk ^ ((row >> 1) & 3)) << 4));
}

}  // namespace tc
}  // namespace hpx
