// healpy a_lm packing: dense [batch][L][M] coefficients <-> healpy's packed
// order-major vector (cuHPX states the index map in
// tests/reproduce_difference_between_healpy_cuhpx.py:58-81):
//   packed[m (2L - 1 - m) / 2 + l] = a[l][m],  m <= l < L, m < min(M, L)
// optionally times (-1)^m (Condon-Shortley factor between the two phase
// conventions).  The dense side is contiguous in m, the packed side in l, so
// each CTA moves one 32 x 32 (l, m) tile through shared memory: coalesced
// reads of 32 orders of a degree row, coalesced writes of 32 degrees of an
// order run.  HBM-bound: 2 x element bytes per kept entry (plus the zeros of
// the dense side when unpacking).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hpx {

constexpr int kHpTile = 32;

__device__ __forceinline__ float2 neg(float2 v) { return make_float2(-v.x, -v.y); }
__device__ __forceinline__ double2 neg(double2 v) { return make_double2(-v.x, -v.y); }

__host__ __device__ inline int64_t healpy_index(int L, int l, int m) {
    return (int64_t)m * (2 * L - 1 - m) / 2 + l;
}
__host__ __device__ inline int64_t healpy_size(int L, int M) {
    const int64_t Mk = M < L ? M : L;
    return Mk * L - Mk * (Mk - 1) / 2;
}

// E: float2 (complex float) or double2 (complex double).  Grid (ceil(min(M,L)/32)
// tiles of orders when packing, ceil(M/32) when unpacking (the dense side's
// orders m >= L are written as zeros), ceil(L/32), maps); block (32, 8).
template <typename E, bool PACK>
__global__ void __launch_bounds__(256) k_healpy(const E* __restrict__ src, E* __restrict__ dst, int L, int M,
                                                int cs_phase) {
    __shared__ E tile[kHpTile][kHpTile + 1];
    const int m0 = blockIdx.x * kHpTile, l0 = blockIdx.y * kHpTile;
    const int64_t b = blockIdx.z;
    const int Mk = M < L ? M : L;
    const int64_t dense = (int64_t)L * M, packed = healpy_size(L, M);
    const int tx = threadIdx.x, ty = threadIdx.y;
    // tiles wholly above the diagonal (every m > l) hold nothing to pack
    if (PACK && m0 > l0 + kHpTile - 1) return;
    if (PACK) {
        // read dense rows: thread (tx, ty + 8k) reads a[l0 + ty + 8k][m0 + tx]
#pragma unroll
        for (int k = 0; k < kHpTile; k += 8) {
            const int l = l0 + ty + k, m = m0 + tx;
            E v{};
            if (l < L && m < Mk && m <= l) {
                v = src[b * dense + (int64_t)l * M + m];
                if (cs_phase && (m & 1)) v = neg(v);
            }
            tile[ty + k][tx] = v;
        }
        __syncthreads();
        // write packed runs: thread (tx, ty + 8k) writes order m0 + ty + k, degree l0 + tx
#pragma unroll
        for (int k = 0; k < kHpTile; k += 8) {
            const int m = m0 + ty + k, l = l0 + tx;
            if (m < Mk && l < L && m <= l) dst[b * packed + healpy_index(L, l, m)] = tile[tx][ty + k];
        }
    } else {
        // read packed runs (zeros above the diagonal)
#pragma unroll
        for (int k = 0; k < kHpTile; k += 8) {
            const int m = m0 + ty + k, l = l0 + tx;
            E v{};
            if (m < Mk && l < L && m <= l) {
                v = src[b * packed + healpy_index(L, l, m)];
                if (cs_phase && (m & 1)) v = neg(v);
            }
            tile[tx][ty + k] = v;
        }
        __syncthreads();
        // write dense rows, zeros for m > l and for orders m >= L
#pragma unroll
        for (int k = 0; k < kHpTile; k += 8) {
            const int l = l0 + ty + k, m = m0 + tx;
            if (l < L && m < M) dst[b * dense + (int64_t)l * M + m] = m < Mk ? tile[ty + k][tx] : E{};
        }
    }
}

}  // namespace hpx
