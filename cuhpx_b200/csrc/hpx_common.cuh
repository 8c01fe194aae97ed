// Shared device/host helpers of the hpx_b200 library: HEALPix ring geometry,
// complex arithmetic, status plumbing.
//
// Ring geometry restates cuhpx/sht_tools.py:161-189, 319-332 (nphi_ring,
// cumulative_nphi_ring, p2phi_ring) and the z formula of
// cuhpx/sht_tools.py:114-140.  Rings are numbered t = 0 .. 4*nside-2 from north
// to south; ring t and ring 4*nside-2-t are mirror images (z -> -z), the
// equator is t = 2*nside-1.  "Ring pair" p in [0, 2*nside) names the north ring
// t=p and its mirror (the equator pairs with itself).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define HPX_HD __host__ __device__ __forceinline__

namespace hpx {

// ------------------------------------------------------------------ geometry
HPX_HD int nrings(int nside) { return 4 * nside - 1; }
HPX_HD int64_t npix(int nside) { return 12ll * nside * nside; }

// pixels on ring t
HPX_HD int ring_nphi(int t, int nside) {
    if (t < nside - 1) return 4 * (t + 1);
    if (t <= 3 * nside - 1) return 4 * nside;
    return 4 * (4 * nside - t - 1);
}

// first pixel of ring t (RING order)
HPX_HD int64_t ring_start(int t, int nside) {
    if (t < nside) return 2ll * t * (t + 1);
    if (t < 3 * nside) return 2ll * nside * (nside + 1) + (int64_t)(t - nside) * 4 * nside;
    int64_t r = 4 * nside - t - 1;
    return 12ll * nside * nside - 2 * r * (r + 1);
}

// phi0 of ring t is s*pi/nphi with s in {0,1} (cuhpx/sht_tools.py:161-176):
// polar rings always have s=1, equatorial rings alternate.
HPX_HD int ring_shift(int t, int nside) {
    if (t + 1 >= nside && t + 1 <= 3 * nside) return (t - nside + 2) & 1;
    return 1;
}

// z = cos(theta) of ring t, exact formula in double
HPX_HD double ring_z(int t, int nside) {
    double n = (double)nside;
    if (t < nside - 1) {
        double a = (double)(t + 1);
        return 1.0 - a * a / (3.0 * n * n);
    }
    if (t <= 3 * nside - 1) return 4.0 / 3.0 - 2.0 * (double)(t + 1) / (3.0 * n);
    double a = (double)(4 * nside - 1 - t);
    return a * a / (3.0 * n * n) - 1.0;
}

// sin^2(theta) of ring t computed without cancellation near the poles
HPX_HD double ring_sin2(int t, int nside) {
    double n = (double)nside;
    int tn = t < 2 * nside ? t : 4 * nside - 2 - t;  // north-hemisphere ring
    if (tn < nside - 1) {
        double a = (double)(tn + 1);
        double omz = a * a / (3.0 * n * n);  // 1 - z
        return omz * (2.0 - omz);
    }
    double z = ring_z(tn, nside);
    return (1.0 - z) * (1.0 + z);
}

// the first north ring that carries order m: F_m(t) is kept only for
// m <= nphi_t/2 (cuhpx/hpx_sht.py:47-48 truncates at min(L, nphi/2+1))
HPX_HD int first_ring_for_m(int m, int nside) {
    if (m > 2 * nside) return 2 * nside;  // no ring carries this order
    // polar ring t has nphi = 4(t+1): need 2(t+1) >= m
    int t = (m + 1) / 2 - 1;
    if (t < 0) t = 0;
    if (t > nside - 1) t = nside - 1;  // equatorial rings carry m <= 2*nside
    return t;
}

// ------------------------------------------------------------------ grid of rings
// What the kernels need to know about the iso-latitude grid of a plan: NP
// ring pairs (north ring p and its mirror), R rings, npix samples per map, and
// which north rings carry order m.  HEALPix grids (nside > 0) truncate order m
// to the rings with nphi/2 >= m; latitude-longitude grids (nside = 0) keep
// orders m < mt_all on every ring.
struct Geom {
    int NP;
    int R;
    int64_t npix;
    int nside;
    int mt_all;
    HPX_HD int first_ring(int m) const {
        if (nside > 0) return first_ring_for_m(m, nside);
        return m < mt_all ? 0 : NP;
    }
};

// ------------------------------------------------------------------ bounds-checked builds
// Built with -DHPX_CHECK_BOUNDS (cuhpx_b200.build VARIANTS["bounds"]), the ring,
// layout, contraction-epilogue and spin-1 kernels check the index of their
// global accesses against the extents of the current chunk's buffers
// (g_hpx_ext, written by the host before every chunk), skip any access outside
// and record the first violation's code in g_hpx_oob; hpx_plan_check reports
// it as HPX_ERR_BOUNDS.  Extents count elements from each buffer's base as the
// kernels receive it: maps and ring spectra in real elements, coefficients in
// real elements, ycols in floats, the synthesis operand in halves (per plane)
// and the analysis operand in 32-bit words (per plane).  Without the define
// every check is the constant true.
enum HpxExtent { kExtMap = 0, kExtF, kExtSpec, kExtAlm, kExtYcols, kExtOperA, kExtOperX, kExtN };
#ifdef HPX_CHECK_BOUNDS
__device__ long long g_hpx_ext[kExtN];
__device__ int g_hpx_oob;
__device__ __forceinline__ bool hpx_inb(int64_t i, int ext, int code) {
    if (i >= 0 && i < g_hpx_ext[ext]) return true;
    atomicCAS(&g_hpx_oob, 0, code);
    return false;
}
#define HPX_INB(i, ext, code) ::hpx::hpx_inb((int64_t)(i), (ext), (code))
#else
#define HPX_INB(i, ext, code) true
#endif

// ------------------------------------------------------------------ complex
template <typename T>
struct __align__(2 * sizeof(T)) cplx {
    T re, im;
};

template <typename T>
HPX_HD cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
HPX_HD cplx<T> cmulc(cplx<T> a, cplx<T> b) {  // a * conj(b)
    return {a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im};
}
template <typename T>
HPX_HD cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
HPX_HD cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T>
HPX_HD cplx<T> cconj(cplx<T> a) { return {a.re, -a.im}; }
template <typename T>
HPX_HD cplx<T> cscale(cplx<T> a, T s) { return {a.re * s, a.im * s}; }

// ------------------------------------------------------------------ async copies
// cp.async global -> shared: 16 bytes (zero fill when !valid), or 8 bytes
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid = true) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace hpx
