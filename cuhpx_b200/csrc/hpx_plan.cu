// hpx_b200 plan object and C ABI (see include/hpx_b200.h).
//
// A plan owns, on one device: the ring-pair table (geometry, quadrature
// weight, Bluestein sizes), FFT twiddles, the Bluestein chirp spectra and the
// per-(m, ring) Legendre start values.  It replaces the reference's
// construction-time precompute (cuhpx/hpx_sht.py:645-683: FITS weights, the
// dense FP64 legpoly_torch table built by an O(L^2) Python loop, W) and its
// process-global cuFFT plan singletons (src/harmonic_transform/hpx_fft.h:69-255,
// hpx_fft.cpp:49,125), which were neither thread-safe nor batch-size
// independent.  Plans here are immutable after creation; every call brings its
// own workspace, so calls on different streams with different workspaces may
// run concurrently.
//
// Adjoints (exact, w.r.t. <x,y> = sum x*y on maps and Re sum conj(a)*b on alm):
//   forward  a = P^T W F f  ->  adjoint  f_bar = F^H W P a_bar
//     where F^H of the truncated, phase-shifted real DFT is the inverse ring
//     transform with the m = 0 and m = nphi/2 terms weighted 1 and all other
//     orders weighted 1/2 (the irfft counts them twice);
//   inverse  f = F^{-1} P a  ->  adjoint a_bar = P^T c F f_bar
//     with c_m = 2 for 0 < m < nphi/2 and 1 for m = 0, nphi/2.
// The reference's hand-written backward (cuhpx/hpx_sht.py:565-583, 614-641)
// halves the m = 0 term and mishandles the ring Nyquist terms; these do not.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/hpx_b200.h"
#include "hpx_kernels.cuh"
#include "legendre_tc.cuh"
#include "hpx_remap.cuh"
#include "hpx_healpy.cuh"
#include "vector.cuh"

using namespace hpx;

namespace {

thread_local std::string g_last_error;

int set_err(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define HPX_CUDA_TRY(expr)                                                                            \
    do {                                                                                              \
        cudaError_t _e = (expr);                                                                      \
        if (_e != cudaSuccess)                                                                        \
            return set_err(_e == cudaErrorMemoryAllocation ? HPX_ERR_OOM : HPX_ERR_CUDA,              \
                           std::string(#expr) + ": " + cudaGetErrorString(_e));                      \
    } while (0)

int ilog2_exact(int v) {
    if (v <= 0 || (v & (v - 1))) return -1;
    int r = 0;
    while ((1 << r) < v) ++r;
    return r;
}
int ceil_log2(int v) {
    int r = 0;
    while ((1 << r) < v) ++r;
    return r;
}

enum Stage { kStRingFwd = 0, kStRingInv, kStLegFwd, kStLegInv, kStAlmCols, kStFold, kStUnfold, kStColsAlm, kNumStages };
const char* kStageNames[kNumStages] = {"ring_fft_forward", "ring_fft_inverse", "legendre_forward", "legendre_inverse",
                                       "alm_to_columns",   "fold",             "unfold",           "columns_to_alm"};

}  // namespace

struct hpx_plan_s {
    hpx_desc_t desc{};
    int device = 0;
    int nside = 0, L = 0, M = 0, NP = 0, R = 0;  // nside = 0: latitude-longitude grid
    Geom geo{};
    int64_t npix = 0;
    int prec = HPX_PREC_FP32;
    bool f64 = false;
    int batch_chunk = 64;
    int logPmax = 0;
    int bufP = 0;   // complex slots of the ring FFT buffer
    int mtmax = 0;  // max orders per ring
    int nmax = 0;   // max nphi
    std::vector<RingPair> h_pairs;
    RingPair* d_pairs = nullptr;
    // ring lists of the three ring-kernel instantiations: power-of-two rings,
    // Bluestein rings of length 2^K, then of length 3 * 2^K (largest first
    // within each), as ring indices t
    int* d_rings = nullptr;
    int n_rings_pow2 = 0, n_rings_blue = 0, n_rings_blue3 = 0;
    int hblue = 0, pblue = 0;    // largest h and FFT length of the Bluestein rings of length 2^K
    int hblue3 = 0, pblue3 = 0;  // ... and of length 3 * 2^K
    // auxiliary stream and fork/join events: the power-of-two ring launch of a
    // transform runs on aux beside the Bluestein launches; the mutex keeps
    // the record/wait pairs of concurrent callers of one plan apart
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    mutable std::mutex fork_mu;
    void* d_rtab = nullptr; // cplx<T> per ring pair: phase table and FFT twiddles (ring_table_slot elements)
    int rslot = 0;
    void* d_gtab = nullptr; // cplx<T> Bluestein chirp spectra (natural order)
    void* d_chirp = nullptr; // cplx<T> Bluestein chirps
    int64_t Ftot = 0;        // complex spectrum entries per map over all rings
    int* d_lstart = nullptr;
    double2* d_pstart = nullptr;
    int2* d_invwork = nullptr;
    int n_invwork = 0;
    int Lpad = 0;                // coefficient row length (L + kCoefPad)
    double2* d_coef = nullptr;   // [M][Lpad] recurrence coefficients
    double2* d_seeds = nullptr;  // [M][seed_blocks(L)][2*nside] block seeds
    int2* d_fwdtiles = nullptr;  // (m, degree block) tiles of the forward contraction
    double* d_z = nullptr;       // cos(theta) of the north rings
    AlphaC* d_alphac = nullptr;  // [M][Lpad] block-normalised recurrence (tensor-core producers)
    int* d_lsmax = nullptr;      // per order: max over its rings of the first significant degree
    std::vector<int> h_lsmax;
    int n_fwdtiles = 0;
    float wmax = 0.f;            // largest ring weight w_t
    int ring_g = 16;             // maps per ring-FFT CTA (hpx_plan_set_schedule)
    int ring_streams = 2;        // 2: ring launches overlap on the aux stream; 1: serial
    size_t ring_smem = 0, blue_smem = 0, blue3_smem = 0, fwd_smem = 0, inv_smem = 0;
    TcPlan tc;  // tensor-core contraction state (mixed precision plans)

    // per-kernel event timing (hpx_stats_*)
    struct EvRec {
        int stage;
        cudaEvent_t a, b;
    };
    std::mutex stats_mu;
    bool stats_on = false;
    std::vector<EvRec> stats_recs;
    std::vector<cudaEvent_t> ev_pool;
    int64_t stat_launch[kNumStages] = {};
    double stat_ms[kNumStages] = {};

    cudaEvent_t take_event() {
        if (!ev_pool.empty()) {
            cudaEvent_t e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }

    ~hpx_plan_s() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        cudaFree(d_pairs);
        cudaFree(d_rings);
        if (aux) cudaStreamDestroy(aux);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        cudaFree(d_gtab);
        cudaFree(d_rtab);
        cudaFree(d_chirp);
        cudaFree(d_lstart);
        cudaFree(d_pstart);
        cudaFree(d_invwork);
        cudaFree(d_coef);
        cudaFree(d_seeds);
        cudaFree(d_fwdtiles);
        cudaFree(d_z);
        cudaFree(d_alphac);
        cudaFree(d_lsmax);
        cudaFree(tc.d_err);
        cudaFree(tc.d_fwd_tiles);
        cudaFree(tc.d_inv_tiles);
        cudaFree(tc.d_fwd_off);
        cudaFree(tc.d_inv_off);
        cudaFree(tc.d_table);
        for (auto& r : stats_recs) {
            cudaEventDestroy(r.a);
            cudaEventDestroy(r.b);
        }
        for (auto e : ev_pool) cudaEventDestroy(e);
        cudaSetDevice(prev);
    }

    size_t real_size() const { return f64 ? sizeof(double) : sizeof(float); }
    int cols() const { return ((2 * batch_chunk) + 3) & ~3; }
    size_t spec_bytes() const { return (size_t)M * 2 * NP * cols() * real_size(); }
    size_t almT_bytes() const { return (size_t)M * L * cols() * real_size(); }
    size_t resid_bytes() const { return (size_t)batch_chunk * npix * real_size(); }
    size_t F_bytes() const { return (size_t)batch_chunk * Ftot * 2 * real_size(); }
    bool mixed() const { return prec == HPX_PREC_BF16X3 || prec == HPX_PREC_F16X3; }
    bool f16() const { return prec == HPX_PREC_F16X3; }
    // bf16/fp16 hi/lo synthesis operand [2M][Lh][128] x 2
    size_t tcA_bytes() const { return mixed() ? (size_t)2 * 2 * M * tc.Lh * kTcCols * sizeof(uint16_t) : 0; }
    // per-map max |F| and max |a| (FP16 operand scales)
    size_t scale_bytes() const { return f16() ? (size_t)2 * 4 * batch_chunk : 0; }
    // order-major analysis output of the tensor cores, ycols[m][l][128]; it
    // reuses the ring-spectra region (dead after the fold) when that is large
    // enough, else the SIMT column region
    size_t ycols_bytes() const { return mixed() ? (size_t)tc.m_tc_end * L * kTcCols * sizeof(float) : 0; }
    bool ycols_in_F() const { return F_bytes() >= ycols_bytes(); }
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

template <typename T>
int create_typed(hpx_plan_s* P) {
    using C = cplx<T>;
    const int Pmax = 1 << P->logPmax;
    // chirp spectra computed in FP64 with FP64 twiddles
    int64_t gsize = 0;
    for (auto& rp : P->h_pairs)
        if (rp.logh < 0) gsize = std::max<int64_t>(gsize, rp.gtab_off + ring_fft_len(rp));
    if (gsize > 0) {
        cplx<double>* tw64 = nullptr;
        HPX_CUDA_TRY(cudaMalloc(&tw64, (size_t)(Pmax / 2) * sizeof(cplx<double>)));
        k_twiddles<double><<<(Pmax / 2 + 255) / 256, 256>>>(tw64, Pmax);
        HPX_CUDA_TRY(cudaMalloc(&P->d_gtab, (size_t)gsize * sizeof(C)));
        HPX_CUDA_TRY(cudaMalloc(&P->d_chirp, (size_t)gsize * sizeof(C)));
        const int Pbig = std::max(Pmax, P->bufP);  // lengths 3 * 2^K included
        size_t sm = (size_t)(2 * padded_len(Pbig) + padded_len(Pbig / 2)) * sizeof(cplx<double>);
        int dmax = 0;
        HPX_CUDA_TRY(cudaDeviceGetAttribute(&dmax, cudaDevAttrMaxSharedMemoryPerBlockOptin, P->device));
        cplx<double>* scratch = nullptr;
        if (P->n_rings_blue3 > 0 && (int)sm > dmax) {
            cudaFree(tw64);
            return set_err(HPX_ERR_UNSUPPORTED, "chirp precompute of the 3 * 2^K lengths needs shared memory");
        }
        if ((int)sm <= dmax) {
            HPX_CUDA_TRY(cudaFuncSetAttribute(k_chirp_spectra<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmax));
            k_chirp_spectra<T, false><<<P->NP, 256, sm>>>(P->d_pairs, tw64, P->logPmax, (C*)P->d_gtab, (C*)P->d_chirp,
                                                          nullptr);
        } else {
            const size_t n = (size_t)P->NP * 2 * padded_len(Pmax);
            if (cudaMalloc(&scratch, n * sizeof(cplx<double>)) != cudaSuccess) {
                cudaFree(tw64);
                return set_err(HPX_ERR_OOM, "chirp precompute scratch");
            }
            k_chirp_spectra<T, true><<<P->NP, 256>>>(P->d_pairs, tw64, P->logPmax, (C*)P->d_gtab, (C*)P->d_chirp,
                                                     scratch);
        }
        cudaError_t e = cudaGetLastError();
        cudaError_t e2 = cudaDeviceSynchronize();
        cudaFree(tw64);
        cudaFree(scratch);
        if (e != cudaSuccess || e2 != cudaSuccess)
            return set_err(HPX_ERR_CUDA, std::string("chirp spectra: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    // per ring pair: phase table and FFT twiddles, copied by each ring CTA
    P->rslot = ring_table_slot(P->bufP, P->nmax);
    HPX_CUDA_TRY(cudaMalloc(&P->d_rtab, (size_t)P->NP * P->rslot * sizeof(C)));
    k_ring_tables<T><<<P->NP, 256>>>(P->d_pairs, P->rslot, (C*)P->d_rtab);
    HPX_CUDA_TRY(cudaGetLastError());
    // shared memory budgets
    P->ring_smem = ring_smem_elems(P->bufP, P->nmax) * sizeof(C);
    // Bluestein CTAs also hold the ring's chirp and half of its chirp spectrum
    P->blue_smem = P->n_rings_blue ? (ring_smem_elems(P->bufP, P->nmax) + P->pblue / 2 + 2 + P->hblue) * sizeof(C) : 0;
    // (192-thread CTAs: one group of 192 at 3072 points, 2 x 3072 padded points
    // of buffers, within ring_smem_elems' 2 x 4096)
    P->blue3_smem =
        P->n_rings_blue3 ? (ring_smem_elems(P->bufP, P->nmax) + P->pblue3 / 2 + 2 + P->hblue3) * sizeof(C) : 0;
    P->fwd_smem = fwd_smem_bytes<T>();
    P->inv_smem = inv_smem_bytes<T>(P->L);
    int dev_max = 0;
    HPX_CUDA_TRY(cudaDeviceGetAttribute(&dev_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, P->device));
    if ((int)P->ring_smem > dev_max || (int)P->blue_smem > dev_max || (int)P->blue3_smem > dev_max ||
        (int)P->fwd_smem > dev_max ||
        (int)P->inv_smem > dev_max)
        return set_err(HPX_ERR_UNSUPPORTED, "nside/lmax too large for the shared-memory kernels of this precision");
    // The attribute is per function, not per plan: always raise it to the device
    // maximum so that a plan needing less never lowers it under another plan.
    HPX_CUDA_TRY(cudaStreamCreateWithFlags(&P->aux, cudaStreamNonBlocking));
    HPX_CUDA_TRY(cudaEventCreateWithFlags(&P->ev_fork, cudaEventDisableTiming));
    HPX_CUDA_TRY(cudaEventCreateWithFlags(&P->ev_join, cudaEventDisableTiming));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_ring_fwd<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_ring_fwd<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_ring_fwd<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_ring_inv<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_ring_inv<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_ring_inv<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_fwd_simt<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_vleg_fwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_vleg_inv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_inv_simt<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_max));
    return HPX_OK;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Assignment of tiles to at most `nsm` CTAs (the m-to-CTA schedule of the
// persistent tensor-core kernels).  `deal` picks the strategy
// (HPX_DEAL_*):
//   ORDER_SNAKE  tiles sorted by decreasing total cost of their order (ties in
//                list order, so the tiles of one order stay together, are dealt
//                to neighbouring CTAs in the same rounds and share the order's
//                data operand in L2), dealt in rounds of one tile per CTA,
//                alternating direction each round (balanced sums);
//   TILE_SNAKE   the same rounds over tiles sorted by their own cost;
//   GREEDY       longest tile first onto the least-loaded CTA;
//   CONTIGUOUS   tiles in order sequence cut into ranges of equal cost, so a
//                CTA keeps the tiles of few orders.
// Returns the CTA count; `order` receives the tiles grouped by CTA and `off`
// the CTA boundaries.
int schedule_tiles(const std::vector<int2>& tiles, const std::vector<double>& cost, int nsm, int deal,
                   std::vector<int2>& order, std::vector<int>& off) {
    const int n = (int)tiles.size();
    const int nc = std::max(1, std::min(nsm, n));
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::vector<std::vector<int>> per(nc);
    if (deal == HPX_DEAL_CONTIGUOUS) {
        double total = 0.0;
        for (double c : cost) total += c;
        double acc = 0.0;
        int cta = 0;
        for (int i = 0; i < n; ++i) {
            // move on once this CTA holds its share (keeping at least one tile for each later CTA)
            if (cta < nc - 1 && acc >= total * (cta + 1) / nc && n - i > nc - 1 - cta) ++cta;
            per[cta].push_back(i);
            acc += cost[i];
        }
    } else {
        if (deal == HPX_DEAL_TILE_SNAKE || deal == HPX_DEAL_GREEDY) {
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        } else {
            std::vector<double> mcost(n);
            for (int i = 0; i < n;) {
                int j = i;
                double c = 0.0;
                while (j < n && tiles[j].x == tiles[i].x) c += cost[j++];
                for (int k = i; k < j; ++k) mcost[k] = c;
                i = j;
            }
            std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return mcost[a] > mcost[b]; });
        }
        if (deal == HPX_DEAL_GREEDY) {
            std::vector<double> load(nc, 0.0);
            for (int k = 0; k < n; ++k) {
                const int c = (int)(std::min_element(load.begin(), load.end()) - load.begin());
                per[c].push_back(idx[k]);
                load[c] += cost[idx[k]];
            }
        } else {
            for (int k = 0; k < n; ++k) {
                const int round = k / nc, pos = k % nc;
                per[(round & 1) ? nc - 1 - pos : pos].push_back(idx[k]);
            }
        }
    }
    order.clear();
    off.assign(1, 0);
    for (auto& v : per) {
        for (int i : v) order.push_back(tiles[i]);
        off.push_back((int)order.size());
    }
    return nc;
}

// Tensor map over the resident table [4 m_tc_end][2N][Lt] of 2-byte halves.
int encode_table(const hpx_plan_s* P, CUtensorMap* map, int box_i, int box_rings, CUtensorMapSwizzle sw) {
    const TcPlan& T = P->tc;
    const cuuint64_t dims[3] = {(cuuint64_t)T.Lt, (cuuint64_t)P->NP, (cuuint64_t)4 * T.m_tc_end};
    const cuuint64_t strides[2] = {(cuuint64_t)T.Lt * 2, (cuuint64_t)T.Lt * 2 * P->NP};
    const cuuint32_t box[3] = {(cuuint32_t)box_i, (cuuint32_t)box_rings, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    CUresult r = ((EncodeTiledFn)T.encode)(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, T.d_table, dims, strides, box, es,
                                           CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(HPX_ERR_CUDA, "cuTensorMapEncodeTiled (table) failed: " + std::to_string((int)r));
    return HPX_OK;
}

// Deal the tensor-core tile lists onto the persistent CTAs with the given
// strategies and CTA count (0: one per SM) and upload them (synchronous).
int tc_deal(hpx_plan_s* P, int fwd_deal, int inv_deal, int ctas) {
    TcPlan& T = P->tc;
    const int nc = ctas > 0 ? std::min(ctas, T.nsm) : T.nsm;
    std::vector<int2> order;
    std::vector<int> off;
    if (!T.fwd_list.empty()) {
        T.n_fwd_ctas = schedule_tiles(T.fwd_list, T.fwd_cost, nc, fwd_deal, order, off);
        HPX_CUDA_TRY(cudaMemcpy(T.d_fwd_tiles, order.data(), sizeof(int2) * order.size(), cudaMemcpyHostToDevice));
        HPX_CUDA_TRY(cudaMemcpy(T.d_fwd_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
    }
    if (!T.inv_list.empty()) {
        T.n_inv_ctas = schedule_tiles(T.inv_list, T.inv_cost, nc, inv_deal, order, off);
        HPX_CUDA_TRY(cudaMemcpy(T.d_inv_tiles, order.data(), sizeof(int2) * order.size(), cudaMemcpyHostToDevice));
        HPX_CUDA_TRY(cudaMemcpy(T.d_inv_off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice));
    }
    T.fwd_deal = fwd_deal;
    T.inv_deal = inv_deal;
    T.ctas = ctas;
    return HPX_OK;
}

// Resident Legendre table (see HPX_FLAG_OTF_LEGENDRE): kept when it fits in
// 45% of the device memory and leaves 4 GB free; otherwise the producer warps
// generate Pbar on the fly.
int tc_table_create(hpx_plan_s* P) {
    TcPlan& T = P->tc;
    T.table = 0;
    if ((P->desc.flags & HPX_FLAG_OTF_LEGENDRE) || T.m_tc_end == 0) return HPX_OK;
    T.Lt = ((P->L + 1) / 2 + 7) & ~7;
    const size_t bytes = (size_t)4 * T.m_tc_end * P->NP * T.Lt * sizeof(uint16_t);
    size_t free_b = 0, total_b = 0;
    HPX_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    if ((double)bytes > 0.45 * (double)total_b || bytes + ((size_t)4 << 30) > free_b) return HPX_OK;
    HPX_CUDA_TRY(cudaMalloc(&T.d_table, bytes));
    HPX_CUDA_TRY(cudaMemset(T.d_table, 0, bytes));
    const int64_t n = (int64_t)T.m_tc_end * seed_blocks(P->L) * P->NP;
    const unsigned grid = (unsigned)((n + 127) / 128);
    if (P->f16())
        k_legendre_table<true><<<grid, 128>>>(T.m_tc_end, P->L, P->Lpad, P->geo, T.Lt, P->d_z, P->d_lstart,
                                              P->d_pstart, P->d_coef, P->d_seeds, T.d_table);
    else
        k_legendre_table<false><<<grid, 128>>>(T.m_tc_end, P->L, P->Lpad, P->geo, T.Lt, P->d_z, P->d_lstart,
                                               P->d_pstart, P->d_coef, P->d_seeds, T.d_table);
    HPX_CUDA_TRY(cudaGetLastError());
    HPX_CUDA_TRY(cudaDeviceSynchronize());
    int rc = encode_table(P, &T.tab_fwd, 64, kFRingS<true>, CU_TENSOR_MAP_SWIZZLE_128B);
    if (rc != HPX_OK) return rc;
    rc = encode_table(P, &T.tab_inv, kTcDegChunk / 2, kTcInvRings, CU_TENSOR_MAP_SWIZZLE_64B);
    if (rc != HPX_OK) return rc;
    T.table_bytes = bytes;
    T.table = 1;
    return HPX_OK;
}

// Tensor-core plan: tile lists, error flag, tensor-map encoder.
int tc_create(hpx_plan_s* P) {
    TcPlan& T = P->tc;
    if (P->batch_chunk != 64)
        return set_err(HPX_ERR_UNSUPPORTED, "bf16x3 plans process 64 maps per pass (batch_chunk must be 64)");
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    HPX_CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess) return set_err(HPX_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
    T.encode = fn;
    HPX_CUDA_TRY(cudaDeviceGetAttribute(&T.nsm, cudaDevAttrMultiProcessorCount, P->device));
    HPX_CUDA_TRY(cudaMalloc(&T.d_err, sizeof(int)));
    HPX_CUDA_TRY(cudaMemset(T.d_err, 0, sizeof(int)));
    T.m_tc_end = std::min(std::min(P->L, P->M), P->mtmax);
    T.Lh = (P->L + 65) / 2;
    const int rc = tc_table_create(P);
    if (rc != HPX_OK) return rc;
    // With the table: first nonzero degree of every (m, ring), so that each tile
    // starts past its all-zero chunks (tile words: fwd_tile_c0 / inv_tile_c0).
    std::vector<int> fnz;
    if (T.table) {
        int* d_fnz = nullptr;
        HPX_CUDA_TRY(cudaMalloc(&d_fnz, sizeof(int) * (size_t)T.m_tc_end * P->NP));
        k_table_first_nz<<<dim3(P->NP, T.m_tc_end), 64>>>(T.d_table, P->NP, T.Lt, d_fnz);
        fnz.resize((size_t)T.m_tc_end * P->NP);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(fnz.data(), d_fnz, sizeof(int) * fnz.size(), cudaMemcpyDeviceToHost);
        cudaFree(d_fnz);
        if (e != cudaSuccess) return set_err(HPX_ERR_CUDA, std::string("table scan: ") + cudaGetErrorString(e));
    }
    std::vector<int2> ft, it;
    std::vector<int> fch, ich;  // chunks each tile runs
    for (int m = 0; m < T.m_tc_end; ++m) {
        const int t0 = P->geo.first_ring(m);
        const int nchF = (P->NP - t0 + kFRingS<true> - 1) / kFRingS<true>;
        const int nchI = (P->L - m + kTcDegChunk - 1) / kTcDegChunk;
        const int* fz = T.table ? fnz.data() + (size_t)m * P->NP : nullptr;
        for (int j = 0; j < (P->L - m + kTcFwdDeg - 1) / kTcFwdDeg; ++j) {
            int c0 = 0;
            if (T.table) {
                while (c0 < nchF - 1) {
                    bool nz = false;
                    for (int p = t0 + c0 * kFRingS<true>; p < std::min(P->NP, t0 + (c0 + 1) * kFRingS<true>); ++p)
                        nz = nz || fz[p] < (j + 1) * kTcFwdDeg;
                    if (nz) break;
                    ++c0;
                }
                fch.push_back(nchF - c0);
            } else {
                fch.push_back((P->NP - t0 + kFRing - 1) / kFRing);
            }
            ft.push_back(make_int2(m, j | (c0 << 8)));
        }
        for (int rb = 0; rb < P->NP - t0; rb += kTcInvRings) {
            int c0 = 0;
            if (T.table) {
                int dmin = 1 << 30;
                for (int p = t0 + rb; p < std::min(P->NP, t0 + rb + kTcInvRings); ++p) dmin = std::min(dmin, fz[p]);
                c0 = std::min(dmin / kTcDegChunk, std::max(nchI - 1, 0));
            }
            ich.push_back(nchI - c0);
            it.push_back(make_int2(m, rb | (c0 << 16)));
        }
    }
    T.n_fwd_tiles = (int)ft.size();
    T.n_inv_tiles = (int)it.size();
    if (T.table) {
        // table part of a pipeline stage: 32 KB in both directions
        for (int c : fch) T.stream_fwd += (size_t)c * (kFStageBytesS<true> / 2);
        for (int c : ich) T.stream_inv += (size_t)c * (kIStageBytes / 2);
    }
    // Tile costs in pipeline chunks, plus a fixed epilogue of about seven
    // chunks per tile.  Without the resident table, a chunk whose degrees
    // start below the order's largest first significant degree takes the
    // producers' slower start-injecting recurrence (about twice the time);
    // with it every chunk costs the same, and the tiles of one order sort
    // together, run at the same time and share its data operand in L2.
    // (with the table a chunk holds 32 rings, twice the producer-fed 16: its
    // cost counts double)
    const double kSlow = T.table ? 1.0 : 2.0, kTileFixed = 7.0;
    std::vector<double> fc, ic;
    for (size_t k = 0; k < ft.size(); ++k) {
        const int2& t = ft[k];
        const double w = T.table ? 2.0 : (t.x + fwd_tile_jb(t.y) * kTcFwdDeg < P->h_lsmax[t.x] ? kSlow : 1.0);
        fc.push_back(fch[k] * w + kTileFixed);
    }
    for (size_t k = 0; k < it.size(); ++k) {
        const int2& t = it[k];
        double c = kTileFixed;
        const int nchI = (P->L - t.x + kTcDegChunk - 1) / kTcDegChunk;
        for (int ci = nchI - ich[k]; ci < nchI; ++ci) c += t.x + ci * kTcDegChunk < P->h_lsmax[t.x] ? kSlow : 1.0;
        ic.push_back(c);
    }
    T.fwd_list = ft;
    T.fwd_cost = fc;
    T.inv_list = it;
    T.inv_cost = ic;
    if (!ft.empty()) {
        HPX_CUDA_TRY(cudaMalloc(&T.d_fwd_tiles, sizeof(int2) * ft.size()));
        HPX_CUDA_TRY(cudaMalloc(&T.d_fwd_off, sizeof(int) * (T.nsm + 1)));
    }
    if (!it.empty()) {
        HPX_CUDA_TRY(cudaMalloc(&T.d_inv_tiles, sizeof(int2) * it.size()));
        HPX_CUDA_TRY(cudaMalloc(&T.d_inv_off, sizeof(int) * (T.nsm + 1)));
    }
    const int rc_deal = tc_deal(P, HPX_DEAL_ORDER_SNAKE, HPX_DEAL_ORDER_SNAKE, 0);
    if (rc_deal != HPX_OK) return rc_deal;
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_fwd_tc<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_fwd_tc<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_fwd_tc<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_fwd_tc<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFSmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_inv_tc<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kISmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_inv_tc<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kISmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_inv_tc<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kISmem));
    HPX_CUDA_TRY(cudaFuncSetAttribute(k_leg_inv_tc<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kISmem));
    T.active = 1;
    return HPX_OK;
}

// 3-D tensor map of 2-byte elements (bf16 or fp16 halves; TMA only moves bytes) over
// [outer][rows][128 cols] with a {64 cols, box_rows} box, 128B swizzle.
// spec[2M][NP][C] (FP32) for the synthesis epilogue's TMA stores: boxes of
// 16 columns x 32 rings in the 64-byte swizzle
int encode_spec_store(const hpx_plan_s* P, CUtensorMap* map, void* spec) {
    const cuuint64_t C = (cuuint64_t)P->cols();
    const cuuint64_t dims[3] = {C, (cuuint64_t)P->NP, 2ull * P->M};
    const cuuint64_t strides[2] = {C * 4, C * 4 * P->NP};
    const cuuint32_t box[3] = {16, 32, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    CUresult r = ((EncodeTiledFn)P->tc.encode)(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, spec, dims, strides, box, es,
                                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                                               CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(HPX_ERR_CUDA, "cuTensorMapEncodeTiled (spec) failed: " + std::to_string((int)r));
    return HPX_OK;
}

int encode_operand(const hpx_plan_s* P, CUtensorMap* map, void* base, uint64_t rows, uint64_t outer, int box_rows) {
    const cuuint64_t dims[3] = {(cuuint64_t)kTcCols, rows, outer};
    const cuuint64_t strides[2] = {(cuuint64_t)kTcCols * 2, (cuuint64_t)kTcCols * 2 * rows};
    const cuuint32_t box[3] = {64, (cuuint32_t)box_rows, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    CUresult r = ((EncodeTiledFn)P->tc.encode)(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, es,
                                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_err(HPX_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return HPX_OK;
}

// zero alm[b][*][m] for m in [m0, M)
__global__ void k_zero_alm_cols(float* __restrict__ alm, int nmaps, int L, int M, int m0) {
    const int64_t n = (int64_t)nmaps * L * (M - m0);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int m = m0 + (int)(i % (M - m0));
        const int64_t bl = i / (M - m0);
        *(float2*)(alm + 2 * (bl * M + m)) = make_float2(0.f, 0.f);
    }
}

// Common plan fields from the descriptor (geometry set by the caller).
void plan_init(const hpx_desc_t* d, hpx_plan_s* P) {
    P->desc = *d;
    P->desc.ring_weights = nullptr;
    P->device = d->device;
    P->nside = d->nside;
    P->L = d->lmax;
    P->M = d->mmax;
    P->prec = d->precision;
    P->f64 = d->precision == HPX_PREC_FP64;
    P->batch_chunk = d->batch_chunk > 0 ? d->batch_chunk : 64;
}

// HEALPix ring pairs (RING order, cuhpx/sht_tools.py:114-189, 319-332):
// north ring p = t and its mirror 4N-2-p; the equator pairs with itself.
void healpix_pairs(const hpx_desc_t* d, hpx_plan_s* P) {
    const int N = d->nside;
    P->NP = 2 * N;
    P->R = 4 * N - 1;
    P->npix = 12ll * N * N;
    P->geo = Geom{P->NP, P->R, P->npix, N, 0};
    P->h_pairs.resize(P->NP);
    const double four_pi_over_npix = 4.0 * M_PI / (double)P->npix;
    for (int p = 0; p < P->NP; ++p) {
        RingPair& rp = P->h_pairs[p];
        std::memset(&rp, 0, sizeof(rp));
        const int ts = 4 * N - 2 - p;
        rp.nphi = ring_nphi(p, N);
        rp.shift_n = ring_shift(p, N);
        rp.shift_s = ring_shift(ts, N);
        rp.has_south = p != 2 * N - 1;
        rp.start_n = ring_start(p, N);
        rp.start_s = ring_start(ts, N);
        rp.z = ring_z(p, N);
        rp.s2 = ring_sin2(p, N);
        // quadrature weight (cuhpx/sht_tools.py:47-59): north ring index p+1
        if (d->ring_weights) rp.w = four_pi_over_npix * (1.0 + d->ring_weights[p]);
        else rp.w = four_pi_over_npix;
    }
}

// Latitude-longitude ring pairs: nlat rings of nlon samples each, phi_k =
// 2 pi k / nlon, ring t at cos(theta_t) = z[t] with quadrature weight w[t]
// (the nodes mirror: z[nlat-1-t] = -z[t]); the ring weight carries the
// longitude factor 2 pi / nlon.
void latlon_pairs(int nlat, int nlon, const std::vector<double>& z, const std::vector<double>& s2,
                  const std::vector<double>& w, hpx_plan_s* P) {
    P->NP = (nlat + 1) / 2;
    P->R = nlat;
    P->npix = (int64_t)nlat * nlon;
    P->geo = Geom{P->NP, P->R, P->npix, 0, std::min(P->M, nlon / 2 + 1)};
    P->h_pairs.resize(P->NP);
    for (int p = 0; p < P->NP; ++p) {
        RingPair& rp = P->h_pairs[p];
        std::memset(&rp, 0, sizeof(rp));
        const int ts = nlat - 1 - p;
        rp.nphi = nlon;
        rp.has_south = ts != p;
        rp.start_n = (int64_t)p * nlon;
        rp.start_s = (int64_t)ts * nlon;
        rp.z = z[p];
        rp.s2 = s2[p];
        rp.w = w[p] * 2.0 * M_PI / (double)nlon;
    }
}

// Quadrature nodes z_j = cos(theta_j) (north to south), sin^2(theta_j) and
// weights (summing to 2) of a latitude-longitude grid, in FP64.
void latlon_quadrature(int grid, int n, std::vector<double>& z, std::vector<double>& s2, std::vector<double>& w) {
    z.assign(n, 0.0);
    s2.assign(n, 0.0);
    w.assign(n, 0.0);
    // P_k(x) and P_k'(x) by the three-term recurrence and P_j' = j P_{j-1} + x P_{j-1}'
    // (no division by 1 - x^2, so accurate next to the poles)
    auto legendre = [](int k, double x, double& pk, double& dpk) {
        double p0 = 1.0, p1 = x, d1 = 1.0;
        if (k == 0) {
            pk = 1.0;
            dpk = 0.0;
            return;
        }
        for (int j = 2; j <= k; ++j) {
            const double p2 = ((2.0 * j - 1.0) * x * p1 - (j - 1.0) * p0) / j;
            d1 = j * p1 + x * d1;
            p0 = p1;
            p1 = p2;
        }
        pk = p1;
        dpk = d1;
    };
    if (grid == HPX_GRID_EQUIANGULAR) {
        // Clenshaw-Curtis on theta_j = pi j / N, N = n - 1
        const int N = n - 1;
        for (int j = 0; j < n; ++j) {
            const double th = M_PI * j / N;
            double sum = 0.0;
            for (int k = 1; 2 * k <= N; ++k) {
                const double b = (2 * k == N) ? 1.0 : 2.0;
                sum += b / (4.0 * k * k - 1.0) * std::cos(2.0 * k * th);
            }
            const double c = (j == 0 || j == N) ? 1.0 : 2.0;
            w[j] = c / N * (1.0 - sum);
            z[j] = std::cos(th);
            const double st = std::sin(th);
            s2[j] = st * st;
        }
        z[0] = 1.0;
        z[N] = -1.0;
        s2[0] = s2[N] = 0.0;
    } else if (grid == HPX_GRID_LEGENDRE_GAUSS) {
        for (int i = 0; i < (n + 1) / 2; ++i) {
            double x = std::cos(M_PI * (i + 0.75) / (n + 0.5)), pk = 0, dpk = 0;
            for (int it = 0; it < 100; ++it) {
                legendre(n, x, pk, dpk);
                const double dx = pk / dpk;
                x -= dx;
                if (std::fabs(dx) < 1e-16) break;
            }
            legendre(n, x, pk, dpk);
            z[i] = x;
            z[n - 1 - i] = -x;
            w[i] = w[n - 1 - i] = 2.0 / ((1.0 - x * x) * dpk * dpk);
        }
        if (n & 1) z[n / 2] = 0.0;
        for (int i = 0; i < n; ++i) s2[i] = (1.0 - z[i]) * (1.0 + z[i]);
    } else {
        // Lobatto: +-1 and the roots of P'_N, N = n - 1; w = 2 / (N (N+1) P_N^2)
        const int N = n - 1;
        for (int i = 0; i < (n + 1) / 2; ++i) {
            double x = i == 0 ? 1.0 : std::cos(M_PI * i / N), pk = 0, dpk = 0;
            if (i > 0) {
                for (int it = 0; it < 100; ++it) {
                    legendre(N, x, pk, dpk);
                    // f = (1 - x^2) P_N', f' = -N (N+1) P_N
                    const double dx = ((1.0 - x * x) * dpk) / (-(double)N * (N + 1) * pk);  // f / f'
                    x -= dx;
                    if (std::fabs(dx) < 1e-16) break;
                }
            }
            legendre(N, x, pk, dpk);
            if (i == 0) pk = 1.0;
            z[i] = x;
            z[n - 1 - i] = -x;
            w[i] = w[n - 1 - i] = 2.0 / ((double)N * (N + 1) * pk * pk);
        }
        if (n & 1) z[n / 2] = 0.0;
        for (int i = 0; i < n; ++i) s2[i] = (1.0 - z[i]) * (1.0 + z[i]);
        s2[0] = s2[n - 1] = 0.0;
    }
}

// Everything after the ring-pair table: FFT sizes, spectrum offsets, Legendre
// start values, seeds and coefficient tables, work lists, FFT tables and the
// tensor-core state.
int plan_build(hpx_plan_s* P) {
    int64_t goff = 0;
    int logPmax = 1, bufP = 2, mtmax = 0, nmax = 1;
    // Bluestein length 3 * 2^10 where smaller than the power of two,
    // for HEALPix grids up to nside 1024 (every length <= 4096: the kernels'
    // shared-memory budget and the chirp precompute in shared memory)
    const bool allow_rad3 = P->nside > 0 && P->nside <= 1024;
    for (int p = 0; p < P->NP; ++p) {
        RingPair& rp = P->h_pairs[p];
        rp.h = rp.nphi / 2;
        rp.mt = std::min(P->M, rp.h + 1);
        rp.logh = ilog2_exact(rp.h);
        rp.rad3 = 0;
        if (rp.logh >= 0) {
            rp.logP = rp.logh;
            rp.gtab_off = -1;
        } else {
            rp.logP = ceil_log2(2 * rp.h - 1);
            int k3 = 0;
            while ((3 << k3) < 2 * rp.h - 1) ++k3;
            if (allow_rad3 && k3 >= kRad3MinK && k3 <= kRad3MaxK && (3 << k3) < (1 << rp.logP) &&
                fft_tpf(3 << k3) % 32 == 0 && ring_kernel_threads<2>() % fft_tpf(3 << k3) == 0) {
                rp.rad3 = 1;
                rp.logP = k3;
            }
            rp.gtab_off = goff;
            goff += ring_fft_len(rp);
        }
        const int Pf = ring_fft_len(rp);
        if (!rp.rad3) logPmax = std::max(logPmax, std::max(rp.logP, 1));
        bufP = std::max(bufP, Pf);
        // threads per FFT: ~16 points per thread, between one warp and the CTA
        rp.tpf = std::min(256, std::max(32, Pf / 16));
        mtmax = std::max(mtmax, rp.mt);
        nmax = std::max(nmax, rp.nphi);
        P->wmax = std::max(P->wmax, (float)rp.w);
    }
    // ring-major spectrum offsets: north rings 0..NP-1, then south rings
    int64_t foff = 0;
    for (int t = 0; t < P->R; ++t) {
        const bool south = t >= P->NP;
        RingPair& rp = P->h_pairs[south ? P->R - 1 - t : t];
        if (south) rp.foff_s = foff; else rp.foff_n = foff;
        foff += (rp.mt + 1) & ~1;  // even offsets: every ring's spectrum starts 16-byte aligned
    }
    P->Ftot = foff;
    P->logPmax = logPmax;
    P->bufP = bufP;
    P->mtmax = mtmax;
    P->nmax = nmax;

    HPX_CUDA_TRY(cudaMalloc(&P->d_pairs, sizeof(RingPair) * P->NP));
    HPX_CUDA_TRY(cudaMemcpy(P->d_pairs, P->h_pairs.data(), sizeof(RingPair) * P->NP, cudaMemcpyHostToDevice));
    {
        std::vector<int> pw, bl, b3;
        auto pair_of = [&](int t) -> const RingPair& { return P->h_pairs[t < P->NP ? t : P->R - 1 - t]; };
        for (int t = 0; t < P->R; ++t) {
            const RingPair& rp = pair_of(t);
            if (rp.logh >= 0) {
                pw.push_back(t);
            } else if (rp.rad3) {
                b3.push_back(t);
                P->hblue3 = std::max(P->hblue3, rp.h);
                P->pblue3 = std::max(P->pblue3, ring_fft_len(rp));
            } else {
                bl.push_back(t);
                P->hblue = std::max(P->hblue, rp.h);
                P->pblue = std::max(P->pblue, 1 << rp.logP);
            }
        }
        auto by_h = [&](int a, int b) { return pair_of(a).h > pair_of(b).h; };
        std::stable_sort(bl.begin(), bl.end(), by_h);
        std::stable_sort(b3.begin(), b3.end(), by_h);
        P->n_rings_pow2 = (int)pw.size();
        P->n_rings_blue = (int)bl.size();
        P->n_rings_blue3 = (int)b3.size();
        pw.insert(pw.end(), bl.begin(), bl.end());
        pw.insert(pw.end(), b3.begin(), b3.end());
        HPX_CUDA_TRY(cudaMalloc(&P->d_rings, sizeof(int) * pw.size()));
        HPX_CUDA_TRY(cudaMemcpy(P->d_rings, pw.data(), sizeof(int) * pw.size(), cudaMemcpyHostToDevice));
    }

    // ---- Legendre start values
    std::vector<double> logc(P->M);
    long double acc = -0.5L * std::log2(4.0L * (long double)M_PI);
    for (int m = 0; m < P->M; ++m) {
        if (m > 0) acc += 0.5L * std::log2((2.0L * m + 1.0L) / (2.0L * m));
        logc[m] = (double)acc;
    }
    double* d_logc = nullptr;
    HPX_CUDA_TRY(cudaMalloc(&d_logc, sizeof(double) * P->M));
    HPX_CUDA_TRY(cudaMemcpy(d_logc, logc.data(), sizeof(double) * P->M, cudaMemcpyHostToDevice));
    const int64_t nms = (int64_t)P->M * P->NP;
    HPX_CUDA_TRY(cudaMalloc(&P->d_lstart, sizeof(int) * nms));
    HPX_CUDA_TRY(cudaMalloc(&P->d_pstart, sizeof(double2) * nms));
    k_legendre_start<<<(unsigned)((nms + 127) / 128), 128>>>(P->M, P->L, P->geo, P->d_pairs, d_logc, P->d_lstart,
                                                           P->d_pstart);
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaDeviceSynchronize();
    cudaFree(d_logc);
    if (e != cudaSuccess || e2 != cudaSuccess)
        return set_err(HPX_ERR_CUDA, std::string("legendre start: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));

    // ---- compact ring z and per-order max start degree (fast-path test of the tensor-core producers)
    {
        std::vector<double> hz(P->NP);
        for (int p = 0; p < P->NP; ++p) hz[p] = P->h_pairs[p].z;
        HPX_CUDA_TRY(cudaMalloc(&P->d_z, sizeof(double) * P->NP));
        HPX_CUDA_TRY(cudaMemcpy(P->d_z, hz.data(), sizeof(double) * P->NP, cudaMemcpyHostToDevice));
        std::vector<int> hls((size_t)nms), hmax(P->M, 0);
        HPX_CUDA_TRY(cudaMemcpy(hls.data(), P->d_lstart, sizeof(int) * nms, cudaMemcpyDeviceToHost));
        for (int m = 0; m < P->M; ++m) {
            const int t0 = P->geo.first_ring(m);
            int mx = m;
            for (int p = t0; p < P->NP; ++p) mx = std::max(mx, hls[(size_t)m * P->NP + p]);
            hmax[m] = mx;
        }
        P->h_lsmax = hmax;
        HPX_CUDA_TRY(cudaMalloc(&P->d_lsmax, sizeof(int) * P->M));
        HPX_CUDA_TRY(cudaMemcpy(P->d_lsmax, hmax.data(), sizeof(int) * P->M, cudaMemcpyHostToDevice));
    }

    // ---- recurrence coefficients and degree-block seeds (FP64)
    P->Lpad = P->L + kCoefPad;
    HPX_CUDA_TRY(cudaMalloc(&P->d_coef, sizeof(double2) * (size_t)P->M * P->Lpad));
    {
        const int64_t n = (int64_t)P->M * P->Lpad;
        k_legendre_coef<<<(unsigned)((n + 255) / 256), 256>>>(P->M, P->L, P->Lpad, P->d_coef);
        HPX_CUDA_TRY(cudaGetLastError());
    }
    HPX_CUDA_TRY(cudaMalloc(&P->d_alphac, sizeof(AlphaC) * (size_t)P->M * P->Lpad));
    HPX_CUDA_TRY(cudaMemset(P->d_alphac, 0, sizeof(AlphaC) * (size_t)P->M * P->Lpad));
    {
        const int64_t n = (int64_t)P->M * seed_blocks(P->L);
        k_legendre_alpha<<<(unsigned)((n + 127) / 128), 128>>>(P->M, P->L, P->Lpad, P->d_coef, P->d_alphac);
        HPX_CUDA_TRY(cudaGetLastError());
    }
    const size_t nseed = (size_t)P->M * seed_blocks(P->L) * P->NP;
    HPX_CUDA_TRY(cudaMalloc(&P->d_seeds, sizeof(double2) * nseed));
    HPX_CUDA_TRY(cudaMemset(P->d_seeds, 0, sizeof(double2) * nseed));
    k_legendre_seeds<<<(unsigned)((nms + 127) / 128), 128>>>(P->M, P->L, P->Lpad, P->geo, P->d_pairs, P->d_lstart,
                                                           P->d_pstart, P->d_coef, P->d_seeds);
    e = cudaGetLastError();
    e2 = cudaDeviceSynchronize();
    if (e != cudaSuccess || e2 != cudaSuccess)
        return set_err(HPX_ERR_CUDA, std::string("legendre seeds: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
    {
        std::vector<int2> tiles;
        for (int m = 0; m < P->M; ++m) {
            const int nb = m < P->L ? (P->L - m + kSeedBlock - 1) / kSeedBlock : 1;
            for (int j = 0; j < nb; ++j) tiles.push_back(make_int2(m, j));
        }
        P->n_fwdtiles = (int)tiles.size();
        HPX_CUDA_TRY(cudaMalloc(&P->d_fwdtiles, sizeof(int2) * tiles.size()));
        HPX_CUDA_TRY(cudaMemcpy(P->d_fwdtiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice));
    }

    // ---- inverse work list: (m, ring block), heaviest first
    std::vector<int2> work;
    const int RBI = InvCfg<float>::RBI;
    for (int m = 0; m < P->M; ++m) {
        const int t0 = P->geo.first_ring(m);
        const int K = P->NP - t0;
        for (int rb = 0; rb < K; rb += RBI) work.push_back(make_int2(m, rb));
    }
    P->n_invwork = (int)work.size();
    if (P->n_invwork > 0) {
        HPX_CUDA_TRY(cudaMalloc(&P->d_invwork, sizeof(int2) * work.size()));
        HPX_CUDA_TRY(cudaMemcpy(P->d_invwork, work.data(), sizeof(int2) * work.size(), cudaMemcpyHostToDevice));
    }

    int rc = P->f64 ? create_typed<double>(P) : create_typed<float>(P);
    if (rc != HPX_OK) return rc;
    if (P->prec == HPX_PREC_TF32) return set_err(HPX_ERR_UNSUPPORTED, "tf32 contraction is not built; use f16x3 or bf16x3");
    if (P->mixed()) {
        rc = tc_create(P);
        if (rc != HPX_OK) return rc;
    }
    return HPX_OK;
}

int check_call(hpx_plan_t plan, const void* a, const void* b, int64_t batch, void* ws, size_t ws_bytes) {
    if (!plan) return set_err(HPX_ERR_INVALID_ARG, "null plan");
    if (batch < 0) return set_err(HPX_ERR_INVALID_ARG, "negative batch");
    if (batch == 0) return HPX_OK;
    if (!a || !b) return set_err(HPX_ERR_INVALID_ARG, "null data pointer");
    size_t need = 0;
    hpx_workspace_size(plan, batch, &need);
    if (!ws || ws_bytes < need)
        return set_err(HPX_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes, got " +
                                              std::to_string(ws_bytes));
    if (((uintptr_t)ws & 255) != 0) return set_err(HPX_ERR_INVALID_ARG, "workspace must be 256-byte aligned");
    return HPX_OK;
}

template <typename T>
struct Pipeline {
    const hpx_plan_s* P;
    cudaStream_t st;
    T* spec;
    T* almT;
    T* resid;
    uint16_t* tcA;  // bf16/fp16 hi/lo synthesis operand (mixed plans)
    float* ycols_alt = nullptr;  // ycols region when the ring spectra region is too small
    unsigned* fmax = nullptr;  // per-map max |F| (FP16 plans)
    unsigned* amax = nullptr;  // per-map max |a| (FP16 plans)
    float fold_wb = 0.f;       // bound on the fold factor |c| (F_t + F_t') / max|F|
    int rc = HPX_OK;

    Pipeline(const hpx_plan_s* p, void* ws, cudaStream_t s) : P(p), st(s) {
        char* c = (char*)ws;
        spec = (T*)c;
        c += (P->spec_bytes() + 255) & ~(size_t)255;
        almT = (T*)c;
        c += (P->almT_bytes() + 255) & ~(size_t)255;
        resid = (T*)c;
        c += (P->resid_bytes() + 255) & ~(size_t)255;
        tcA = (uint16_t*)c;
        c += (P->tcA_bytes() + 255) & ~(size_t)255;
        F = (T*)c;
        c += (P->F_bytes() + 255) & ~(size_t)255;
        set_scales(c);
        ycols_alt = (float*)almT;
    }
    void set_scales(char* c) {
        if (!P->f16()) return;
        fmax = (unsigned*)c;
        amax = fmax + P->batch_chunk;
    }
    // analysis-only layout: folded spectra and ring spectra at given addresses
    Pipeline(const hpx_plan_s* p, T* spec_, T* F_, char* scales, float* ycols, cudaStream_t s)
        : P(p), st(s), spec(spec_), almT(nullptr), resid(nullptr), tcA(nullptr), F(F_) {
        set_scales(scales);
        ycols_alt = ycols;
    }
    T* F;  // ring-major spectra [map][Ftot] complex
    // folded spectra as bf16 hi/lo (mixed plans), aliasing the spec region
    uint32_t* xh() const { return P->mixed() ? (uint32_t*)spec : nullptr; }
    uint32_t* xl() const {
        return P->mixed() ? (uint32_t*)((uint16_t*)spec + (size_t)2 * P->M * P->NP * kTcCols) : nullptr;
    }


    // brackets one launch with events when the plan's stats are enabled
    struct Timer {
        hpx_plan_s* P;
        cudaStream_t st;
        int stage;
        cudaEvent_t a = nullptr;
        Timer(const hpx_plan_s* p, cudaStream_t s, int stg) : P(const_cast<hpx_plan_s*>(p)), st(s), stage(stg) {
            if (!P->stats_on) return;
            std::lock_guard<std::mutex> g(P->stats_mu);
            a = P->take_event();
            cudaEventRecord(a, st);
        }
        ~Timer() {
            if (!a) return;
            std::lock_guard<std::mutex> g(P->stats_mu);
            cudaEvent_t b = P->take_event();
            cudaEventRecord(b, st);
            P->stats_recs.push_back({stage, a, b});
        }
    };

    // maps per ring CTA (default 16: amortises the CTA's table set-up -- phase
    // and twiddle tables, Bluestein chirp tables -- over twice the maps of 8,
    // 2.5% of the step; 32 measured no better); set by hpx_plan_set_schedule
    int maps_per_cta_ring() const { return P->ring_g; }

    // The power-of-two rings on the plan's auxiliary stream and the Bluestein
    // rings (2^K, then 3072 points) on st, forked and joined by events (valid
    // under stream capture), so that the launches and their tails overlap.
    template <typename Pow2, typename Blue>
    void ring_launches(Pow2 pow2, Blue blue) {
        const bool any_blue = P->n_rings_blue + P->n_rings_blue3 > 0;
        if (P->n_rings_pow2 && any_blue && P->ring_streams == 2) {
            std::lock_guard<std::mutex> lk(P->fork_mu);
            cudaError_t e = cudaEventRecord(P->ev_fork, st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(P->aux, P->ev_fork, 0);
            if (e == cudaSuccess) {
                pow2(P->aux);
                blue(st);
                e = cudaEventRecord(P->ev_join, P->aux);
            }
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, P->ev_join, 0);
            if (e != cudaSuccess) rc = set_err(HPX_ERR_CUDA, std::string("ring stream fork/join: ") + cudaGetErrorString(e));
            return;
        }
        if (P->n_rings_pow2) pow2(st);
        if (any_blue) blue(st);
    }

    // map -> ring spectra F -> folded Legendre operand (spec, or bf16 hi/lo)
    void ring_fwd(const T* map, int nb, int adjoint) {
        const int g = maps_per_cta_ring();
        {
            Timer tm(P, st, kStRingFwd);
            if (fmax) cudaMemsetAsync(fmax, 0, sizeof(unsigned) * nb, st);
            const unsigned nbk = (nb + g - 1) / g;
            const cplx<T>* gt = (const cplx<T>*)P->d_gtab;
            const cplx<T>* ch = (const cplx<T>*)P->d_chirp;
            const cplx<T>* rt = (const cplx<T>*)P->d_rtab;
            ring_launches(
                [&](cudaStream_t s) {
                    k_ring_fwd<T, 0><<<dim3(P->n_rings_pow2, nbk), 256, P->ring_smem, s>>>(
                        map, nb, g, F, P->Ftot, P->geo, P->d_pairs, P->d_rings, rt, P->rslot, gt, ch, fmax);
                },
                [&](cudaStream_t s) {
                    if (P->n_rings_blue)
                        k_ring_fwd<T, 1><<<dim3(P->n_rings_blue, nbk), 256, P->blue_smem, s>>>(
                            map, nb, g, F, P->Ftot, P->geo, P->d_pairs, P->d_rings + P->n_rings_pow2, rt, P->rslot, gt,
                            ch, fmax);
                    if (P->n_rings_blue3)
                        k_ring_fwd<T, 2><<<dim3(P->n_rings_blue3, nbk), ring_kernel_threads<2>(), P->blue3_smem, s>>>(
                            map, nb, g, F, P->Ftot, P->geo, P->d_pairs, P->d_rings + P->n_rings_pow2 + P->n_rings_blue,
                            rt, P->rslot, gt, ch, fmax);
                });
        }
        Timer tm(P, st, kStFold);
        // |c (F_t +- F_t')| <= 2 max|c| max|F|: c = w_t, or c_m <= 2 for the adjoint
        fold_wb = adjoint ? 4.f : 2.f * P->wmax;
        dim3 fg((P->mtmax + fold_mb<T>() - 1) / fold_mb<T>(), P->NP, (nb + 63) / 64);
        k_fold<T><<<fg, 256, 0, st>>>(F, P->Ftot, nb, P->geo, P->d_pairs, adjoint, spec, P->cols(), xh(), xl(),
                                      fmax, fold_wb);
    }
    // synthesis output spec (E/O) -> ring spectra F -> map (ref: residual ref - map)
    void ring_inv(T* map, int nb, int adjoint, const T* ref) {
        {
            Timer tm(P, st, kStUnfold);
            dim3 fg((P->mtmax + fold_mb<T>() - 1) / fold_mb<T>(), P->NP, (nb + 63) / 64);
            k_unfold<T><<<fg, 256, 0, st>>>(spec, P->cols(), nb, P->geo, P->d_pairs, adjoint, F, P->Ftot);
        }
        const int g = maps_per_cta_ring();
        Timer tm(P, st, kStRingInv);
        const unsigned nbk = (nb + g - 1) / g;
        const cplx<T>* gt = (const cplx<T>*)P->d_gtab;
        const cplx<T>* ch = (const cplx<T>*)P->d_chirp;
        const cplx<T>* rt = (const cplx<T>*)P->d_rtab;
        ring_launches(
            [&](cudaStream_t s) {
                k_ring_inv<T, 0><<<dim3(P->n_rings_pow2, nbk), 256, P->ring_smem, s>>>(
                    F, P->Ftot, map, nb, g, P->geo, P->d_pairs, P->d_rings, rt, P->rslot, gt, ch, ref);
            },
            [&](cudaStream_t s) {
                if (P->n_rings_blue)
                    k_ring_inv<T, 1><<<dim3(P->n_rings_blue, nbk), 256, P->blue_smem, s>>>(
                        F, P->Ftot, map, nb, g, P->geo, P->d_pairs, P->d_rings + P->n_rings_pow2, rt, P->rslot,
                        gt, ch, ref);
                if (P->n_rings_blue3)
                    k_ring_inv<T, 2><<<dim3(P->n_rings_blue3, nbk), ring_kernel_threads<2>(), P->blue3_smem, s>>>(
                        F, P->Ftot, map, nb, g, P->geo, P->d_pairs, P->d_rings + P->n_rings_pow2 + P->n_rings_blue,
                        rt, P->rslot, gt, ch, ref);
            });
    }
    void leg_fwd(T* alm, int nb, int accumulate) {
        const int C = P->cols();
        if (P->mixed()) {
            const TcPlan& TP = P->tc;
            float* yc = (float*)(P->ycols_in_F() ? (void*)F : (void*)ycols_alt);
            {
                Timer tm(P, st, kStLegFwd);
                if (!accumulate && TP.m_tc_end < P->M)
                    k_zero_alm_cols<<<1024, 256, 0, st>>>((float*)alm, nb, P->L, P->M, TP.m_tc_end);
                if (TP.n_fwd_tiles == 0) return;
                CUtensorMap mh, ml;
                const int box_rings = TP.table ? kFRingS<true> : kFRingS<false>;
                if ((rc = encode_operand(P, &mh, xh(), P->NP, 2ull * P->M, box_rings)) != HPX_OK) return;
                if ((rc = encode_operand(P, &ml, xl(), P->NP, 2ull * P->M, box_rings)) != HPX_OK) return;
                auto kern = TP.table ? (P->f16() ? k_leg_fwd_tc<true, true> : k_leg_fwd_tc<false, true>)
                                     : (P->f16() ? k_leg_fwd_tc<true, false> : k_leg_fwd_tc<false, false>);
                kern<<<TP.n_fwd_ctas, kTcThreads, kFSmem, st>>>(
                    mh, ml, TP.table ? TP.tab_fwd : mh, nb, yc, P->L, P->Lpad, P->geo, P->d_z, P->d_lstart,
                    P->d_lsmax, P->d_pstart, P->d_coef, P->d_alphac, P->d_seeds, TP.d_fwd_tiles, TP.d_fwd_off, fmax,
                    fold_wb, TP.d_err);
            }
            Timer tm(P, st, kStColsAlm);
            dim3 tg((TP.m_tc_end + 31) / 32, P->L);
            k_tc_to_alm<<<tg, dim3(32, 8), 0, st>>>(yc, nb, P->L, P->M, TP.m_tc_end, (float*)alm, accumulate);
            return;
        }
        Timer tm(P, st, kStLegFwd);
        dim3 grid(P->n_fwdtiles, (C + FwdCfg<T>::CT - 1) / FwdCfg<T>::CT);
        k_leg_fwd_simt<T><<<grid, 256, P->fwd_smem, st>>>(spec, C, nb, alm, P->L, P->M, P->geo, P->d_pairs,
                                                          P->d_lstart, P->d_pstart, P->d_coef, P->Lpad, P->d_seeds,
                                                          P->d_fwdtiles, accumulate);
    }
    void leg_inv(const T* alm, int nb) {
        const int C = P->cols();
        if (P->mixed()) {
            const TcPlan& TP = P->tc;
            uint16_t* ah = tcA;
            uint16_t* al = tcA + (size_t)2 * P->M * TP.Lh * kTcCols;
            {
                Timer tm(P, st, kStAlmCols);
                if (amax) {
                    cudaMemsetAsync(amax, 0, sizeof(unsigned) * nb, st);
                    k_alm_maxabs<<<dim3((P->L + 7) / 8, nb), 256, 0, st>>>((const float*)alm, P->L, P->M, amax);
                }
                dim3 tg((P->M + 31) / 32, P->L + 64);
                k_alm_to_tc<<<tg, dim3(32, 8), 0, st>>>((const float*)alm, nb, P->L, P->M, TP.Lh, ah, al, amax);
            }
            Timer tm(P, st, kStLegInv);
            // orders the tensor cores do not visit must read as zero in the ring stage
            if (TP.m_tc_end < P->M)
                cudaMemsetAsync(spec + (size_t)TP.m_tc_end * 2 * P->NP * C, 0,
                                (size_t)(P->M - TP.m_tc_end) * 2 * P->NP * C * sizeof(T), st);
            if (TP.n_inv_tiles == 0) return;
            CUtensorMap mh, ml;
            if ((rc = encode_operand(P, &mh, ah, TP.Lh, 2ull * P->M, 32)) != HPX_OK) return;
            if ((rc = encode_operand(P, &ml, al, TP.Lh, 2ull * P->M, 32)) != HPX_OK) return;
            CUtensorMap sm = mh;
            if (TP.table && (rc = encode_spec_store(P, &sm, spec)) != HPX_OK) return;
            auto kern = TP.table ? (P->f16() ? k_leg_inv_tc<true, true> : k_leg_inv_tc<false, true>)
                                 : (P->f16() ? k_leg_inv_tc<true, false> : k_leg_inv_tc<false, false>);
            kern<<<TP.n_inv_ctas, kTcThreads, kISmem, st>>>(
                mh, ml, TP.table ? TP.tab_inv : mh, sm, (float*)spec, C, nb, P->L, P->M, P->Lpad, P->geo, P->d_z, P->d_lstart, P->d_lsmax,
                P->d_pstart, P->d_coef, P->d_alphac, P->d_seeds, TP.d_inv_tiles, TP.d_inv_off, amax, TP.d_err);
            return;
        }
        dim3 tg((P->M + 31) / 32, P->L, (nb + 15) / 16);
        {
            Timer tm(P, st, kStAlmCols);
            k_alm_to_cols<T><<<tg, dim3(32, 8), 0, st>>>(alm, nb, P->L, P->M, almT, C);
        }
        Timer tm(P, st, kStLegInv);
        if (P->n_invwork == 0) return;
        dim3 grid(P->n_invwork, (C + InvCfg<T>::CT - 1) / InvCfg<T>::CT);
        k_leg_inv_simt<T><<<grid, 256, P->inv_smem, st>>>(almT, C, spec, P->L, P->M, P->geo, P->d_pairs,
                                                          P->d_lstart, P->d_pstart, P->d_coef, P->Lpad,
                                                          P->d_invwork);
    }
};

enum Op { kForward, kInverse, kForwardAdjoint, kInverseAdjoint, kForwardRefined };

// Bounds-checked builds: the extents (elements from each buffer's base) of one
// chunk's buffers, written before the chunk's launches on their stream.  The
// failure-detection test shrinks one of them by an element
// (HPX_TEST_SHRINK_EXTENT=<index>) so that the last access is reported (and
// skipped).  In the product build this does nothing.
void set_extents(const hpx_plan_s* P, cudaStream_t st, int64_t map_elems, int64_t alm_elems, int nb) {
#ifdef HPX_CHECK_BOUNDS
    long long v[kExtN];
    v[kExtMap] = map_elems;
    v[kExtF] = (long long)2 * nb * P->Ftot;
    v[kExtSpec] = (long long)(P->spec_bytes() / P->real_size());
    v[kExtAlm] = alm_elems;
    v[kExtYcols] = (long long)(P->ycols_bytes() / sizeof(float));
    v[kExtOperA] = P->mixed() ? (long long)2 * P->M * P->tc.Lh * kTcCols : 0;
    v[kExtOperX] = P->mixed() ? (long long)2 * P->M * P->NP * kTcCols / 2 : 0;
    if (const char* e = getenv("HPX_TEST_SHRINK_EXTENT")) {
        const int k = atoi(e);
        if (k >= 0 && k < kExtN && v[k] > 0) v[k] -= 1;
    }
    cudaMemcpyToSymbolAsync(g_hpx_ext, v, sizeof(v), 0, cudaMemcpyHostToDevice, st);
#else
    (void)P;
    (void)st;
    (void)map_elems;
    (void)alm_elems;
    (void)nb;
#endif
}

// Spin-1 transforms of a plan built with L+1 degrees and M+1 orders (see
// vector.cuh): maps [batch][2][npix] <-> coefficients [batch][2][L][M].  Each
// pass takes batch_chunk / 2 vector maps, whose 2 components run through the
// ring stages as batch_chunk scalar maps.
template <typename T>
int run_vec(hpx_plan_s* P, Op op, const void* in, void* out, int64_t batch, void* ws, cudaStream_t st, int csphase) {
    Pipeline<T> pl(P, ws, st);
    const int Lv = P->L - 1, Mv = P->M - 1;
    const int C = P->cols();
    const int64_t vc = std::max(1, P->batch_chunk / 2);
    const size_t alm_stride = (size_t)2 * Lv * Mv * 2;
    const size_t map_stride = (size_t)2 * P->npix;
    for (int64_t b0 = 0; b0 < batch; b0 += vc) {
        const int nb = (int)std::min<int64_t>(vc, batch - b0);
        set_extents(P, st, (int64_t)nb * map_stride, (int64_t)nb * alm_stride, 2 * nb);
        const bool analysis = op == kForward || op == kInverseAdjoint;
        if (analysis) {
            const T* map = (const T*)in + b0 * map_stride;
            T* alm = (T*)out + b0 * alm_stride;
            pl.ring_fwd(map, 2 * nb, op == kForward ? 0 : 1);
            typename Pipeline<T>::Timer tm(P, st, kStLegFwd);
            const int nj = (Lv + VFwdCfg<T>::LT - 1) / VFwdCfg<T>::LT;
            const dim3 grid((unsigned)(Mv * nj), (unsigned)((C + VFwdCfg<T>::CT - 1) / VFwdCfg<T>::CT));
            k_vleg_fwd<T><<<grid, 256, vfwd_smem_bytes<T>(), st>>>(
                pl.spec, C, nb, alm, Lv, Mv, P->L, P->M, P->Lpad, P->geo, P->d_pairs, P->d_lstart, P->d_pstart,
                P->d_coef, P->d_seeds, csphase, op == kForward ? 1 : 0);
        } else {
            const T* alm = (const T*)in + b0 * alm_stride;
            T* map = (T*)out + b0 * map_stride;
            {
                typename Pipeline<T>::Timer tm(P, st, kStLegInv);
                const int nr = (P->NP + VInvCfg<T>::RBI - 1) / VInvCfg<T>::RBI;
                const dim3 grid((unsigned)(P->M * nr), (unsigned)((C + VInvCfg<T>::CT - 1) / VInvCfg<T>::CT));
                k_vleg_inv<T><<<grid, 256, vinv_smem_bytes<T>(), st>>>(alm, nb, pl.spec, C, Lv, Mv, P->L, P->M,
                                                                       P->Lpad, P->geo, P->d_pairs, P->d_lstart,
                                                                       P->d_pstart, P->d_coef, csphase,
                                                                       op == kForwardAdjoint ? 1 : 0);
            }
            pl.ring_inv(map, 2 * nb, op == kInverse ? 0 : 1, nullptr);
        }
        if (pl.rc != HPX_OK) return pl.rc;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(HPX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    return HPX_OK;
}

int dispatch_vec(hpx_plan_t plan, Op op, const void* in, void* out, int64_t batch, int32_t csphase, void* ws,
                 size_t ws_bytes, void* stream) {
    int rc = check_call(plan, in, out, batch, ws, ws_bytes);
    if (rc != HPX_OK || batch == 0) return rc;
    if (plan->nside <= 0) return set_err(HPX_ERR_UNSUPPORTED, "spin-1 transforms are built for HEALPix plans");
    if (plan->mixed()) return set_err(HPX_ERR_UNSUPPORTED, "spin-1 transforms run on FP32 or FP64 plans");
    if (plan->L < 2 || plan->M < 2)
        return set_err(HPX_ERR_INVALID_ARG, "a spin-1 plan needs lmax >= 2 and mmax >= 2 (L+1 and M+1 of the transform)");
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    try {
        return plan->f64 ? run_vec<double>(plan, op, in, out, batch, ws, st, csphase ? 1 : 0)
                         : run_vec<float>(plan, op, in, out, batch, ws, st, csphase ? 1 : 0);
    } catch (const std::exception& ex) {
        return set_err(HPX_ERR_CUDA, ex.what());
    }
}

template <typename T>
int run_op(hpx_plan_s* P, Op op, const void* in, void* out, int64_t batch, void* ws, cudaStream_t st, int iters) {
    Pipeline<T> pl(P, ws, st);
    const int64_t bc = P->batch_chunk;
    const size_t alm_stride = (size_t)P->L * P->M * 2;
    for (int64_t b0 = 0; b0 < batch; b0 += bc) {
        const int nb = (int)std::min<int64_t>(bc, batch - b0);
        set_extents(P, st, (int64_t)nb * P->npix, (int64_t)nb * alm_stride, nb);
        switch (op) {
            case kForward:
            case kInverseAdjoint: {
                const T* map = (const T*)in + b0 * P->npix;
                T* alm = (T*)out + b0 * alm_stride;
                pl.ring_fwd(map, nb, op == kForward ? 0 : 1);
                pl.leg_fwd(alm, nb, 0);
                break;
            }
            case kForwardRefined: {
                // a = S f;  repeat: r = f - I a;  a += S r
                const T* map = (const T*)in + b0 * P->npix;
                T* alm = (T*)out + b0 * alm_stride;
                pl.ring_fwd(map, nb, 0);
                pl.leg_fwd(alm, nb, 0);
                for (int it = 0; it < iters; ++it) {
                    pl.leg_inv(alm, nb);
                    pl.ring_inv(pl.resid, nb, 0, map);
                    pl.ring_fwd(pl.resid, nb, 0);
                    pl.leg_fwd(alm, nb, 1);
                }
                break;
            }
            case kInverse:
            case kForwardAdjoint: {
                const T* alm = (const T*)in + b0 * alm_stride;
                T* map = (T*)out + b0 * P->npix;
                pl.leg_inv(alm, nb);
                pl.ring_inv(map, nb, op == kInverse ? 0 : 1, nullptr);
                break;
            }
        }
        if (pl.rc != HPX_OK) return pl.rc;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(HPX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    return HPX_OK;
}

int dispatch(hpx_plan_t plan, Op op, const void* in, void* out, int64_t batch, void* ws, size_t ws_bytes,
             void* stream, int iters = 0) {
    int rc = check_call(plan, in, out, batch, ws, ws_bytes);
    if (rc != HPX_OK || batch == 0) return rc;
    DeviceGuard g(plan->device);
    cudaStream_t st = (cudaStream_t)stream;
    try {
        return plan->f64 ? run_op<double>(plan, op, in, out, batch, ws, st, iters)
                         : run_op<float>(plan, op, in, out, batch, ws, st, iters);
    } catch (const std::exception& ex) {
        return set_err(HPX_ERR_CUDA, ex.what());
    }
}

// ---- analysis without allocation: one static scratch array per device
//
// Region sizes of one chunk of batch_chunk maps: folded spectra, then ring
// spectra, each 256-byte aligned.  Every scratch element a call reads was
// written earlier in the same call (ring spectra for the rings that carry an
// order, folded spectra for every column of the chunk), so nothing has to
// start at zero.
size_t noalloc_spec_offset(const hpx_plan_s* P) { return (P->spec_bytes() + 255) & ~(size_t)255; }
size_t noalloc_scale_offset(const hpx_plan_s* P) {
    return noalloc_spec_offset(P) + ((P->F_bytes() + 255) & ~(size_t)255);
}
size_t noalloc_ycols_offset(const hpx_plan_s* P) {
    return noalloc_scale_offset(P) + ((P->scale_bytes() + 255) & ~(size_t)255);
}
size_t noalloc_need(const hpx_plan_s* P) {
    return noalloc_ycols_offset(P) + (P->ycols_in_F() ? 0 : P->ycols_bytes());
}

}  // namespace

// Zero-initialised device storage of the module: no allocation call makes it,
// it exists once per device the library is loaded on, and every plan on that
// device shares it.
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
struct NoAllocSlot {
    unsigned long long ctx_id = 0;  // driver context ID the address belongs to (0: none yet)
    void* ptr = nullptr;
};
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long*);

// ID of the current context, unique for the life of the process (a context
// created after cudaDeviceReset gets a new one); 0 when it cannot be read.
unsigned long long current_ctx_id() {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrentFn)fn;
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)fn;
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur && get_id && get_cur(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS) return id;
    return 0;
}

// Address of the scratch on `device` (the caller holds a DeviceGuard for it):
// looked up with cudaGetSymbolAddress on the first call on the device, and
// again whenever the device's context is not the one the cached address
// belongs to (after cudaDeviceReset the array lives at a new address).
int noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return set_err(HPX_ERR_UNSUPPORTED, "device ordinal above 63");
    const unsigned long long id = current_ctx_id();
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    NoAllocSlot& slot = g_noalloc_slot[device];
    if (!slot.ptr || id == 0 || slot.ctx_id != id) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            slot = NoAllocSlot{};
            return set_err(HPX_ERR_CUDA, std::string("scratch symbol address: ") + cudaGetErrorString(e));
        }
        slot.ptr = p;
        slot.ctx_id = id;
    }
    *out = (unsigned char*)slot.ptr;
    return HPX_OK;
}

template <typename T>
int run_forward_noalloc(hpx_plan_s* P, const void* in, void* out, int64_t batch, unsigned char* scratch,
                        cudaStream_t st) {
    Pipeline<T> pl(P, (T*)scratch, (T*)(scratch + noalloc_spec_offset(P)), (char*)scratch + noalloc_scale_offset(P),
                   (float*)(scratch + noalloc_ycols_offset(P)), st);
    const int64_t bc = P->batch_chunk;
    const size_t alm_stride = (size_t)P->L * P->M * 2;
    for (int64_t b0 = 0; b0 < batch; b0 += bc) {
        const int nb = (int)std::min<int64_t>(bc, batch - b0);
        set_extents(P, st, (int64_t)nb * P->npix, (int64_t)nb * alm_stride, nb);
        pl.ring_fwd((const T*)in + b0 * P->npix, nb, 0);
        pl.leg_fwd((T*)out + b0 * alm_stride, nb, 0);
        if (pl.rc != HPX_OK) return pl.rc;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_err(HPX_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    }
    return HPX_OK;
}

// Opt a remap kernel into more than 48 KB of dynamic shared memory, once per
// device and kernel.
template <auto KERNEL>
int remap_smem_optin(size_t smem) {
    if (smem <= 48 * 1024) return HPX_OK;
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    HPX_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 64 && done[dev]) return HPX_OK;
    HPX_CUDA_TRY(cudaFuncSetAttribute(KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (dev < 64) done[dev] = true;
    return HPX_OK;
}

struct RemapLaunch {
    dim3 grid;
    size_t smem;
    cudaStream_t st;
    int64_t np;
    int nside, logs, log_tiles, nb, mpc, vec;
    RemapSide src, dst;
};

template <typename E, int SO, int DO>
int launch_remap_async(const E* in, E* out, const RemapLaunch& L) {
    const int rc = remap_smem_optin<k_remap_async<E, SO, DO>>(L.smem);
    if (rc != HPX_OK) return rc;
    k_remap_async<E, SO, DO><<<L.grid, kRemapThreads, L.smem, L.st>>>(in, out, L.np, L.nside, L.logs, L.log_tiles,
                                                                      L.nb, L.mpc, L.src, L.dst, L.vec);
    HPX_CUDA_TRY(cudaGetLastError());
    return HPX_OK;
}

template <typename E>
int dispatch_remap_async(const E* in, E* out, const RemapLaunch& L) {
    const int so = L.src.order, d = L.dst.order;
    if (so == kOrderRing && d == kOrderNest) return launch_remap_async<E, kOrderRing, kOrderNest>(in, out, L);
    if (so == kOrderRing && d == kOrderXY) return launch_remap_async<E, kOrderRing, kOrderXY>(in, out, L);
    if (so == kOrderNest && d == kOrderRing) return launch_remap_async<E, kOrderNest, kOrderRing>(in, out, L);
    if (so == kOrderNest && d == kOrderXY) return launch_remap_async<E, kOrderNest, kOrderXY>(in, out, L);
    if (so == kOrderXY && d == kOrderRing) return launch_remap_async<E, kOrderXY, kOrderRing>(in, out, L);
    if (so == kOrderXY && d == kOrderNest) return launch_remap_async<E, kOrderXY, kOrderNest>(in, out, L);
    if (so == kOrderXY && d == kOrderXY) return launch_remap_async<E, kOrderXY, kOrderXY>(in, out, L);
    return set_err(HPX_ERR_INVALID_ARG, "remap: equal orders are a copy");
}

// Remap launcher: squares of 64 x 64 pixels for elements of up to 4 bytes and
// 32 x 32 above, fewer for nside < 64.  Map groups of up to 16 maps a CTA
// amortise the offsets' arithmetic, while leaving at least 16 CTAs a
// multiprocessor.  Elements of 4, 8 and 16 bytes take the cp.async pipeline
// (16-byte accesses on NEST and XY sides when the tiles are at least 16 bytes
// wide and both buffers 16-byte aligned); 1- and 2-byte elements stage
// through registers.
template <typename E>
int launch_remap(const void* in, void* out, int64_t batch, int nside, RemapSide src, RemapSide dst,
                 cudaStream_t st) {
    const int logn = ilog2_exact(nside);
    const int s = std::min(nside, sizeof(E) <= 4 ? 64 : 32);
    const int logs = ilog2_exact(s);
    const int log_tiles = logn - logs;
    const int64_t tiles = 12ll << (2 * log_tiles);
    int mpc = 16;
    while (mpc > 1 && tiles * ((batch + mpc - 1) / mpc) < 148ll * 16) mpc >>= 1;
    const bool ring = src.order == kOrderRing || dst.order == kOrderRing;
    constexpr bool kAsync = sizeof(E) >= 4;
    const size_t smem = kAsync ? remap_async_smem_bytes(s, (int)sizeof(E), ring)
                               : remap_smem_bytes(s, (int)sizeof(E), ring);
    const int vec = (s * (int)sizeof(E) >= 16 && ((((uintptr_t)in) | ((uintptr_t)out)) & 15) == 0) ? 1 : 0;
    const int64_t np = 12ll * nside * nside;
    const int64_t chunk = 65535ll * mpc;
    for (int64_t b = 0; b < batch; b += chunk) {
        const int nb = (int)std::min(chunk, batch - b);
        const dim3 grid((unsigned)tiles, (unsigned)((nb + mpc - 1) / mpc));
        const E* pin = (const E*)in + b * np;
        E* pout = (E*)out + b * np;
        if constexpr (kAsync) {
            const RemapLaunch L{grid, smem, st, np, nside, logs, log_tiles, nb, mpc, vec, src, dst};
            const int rc = dispatch_remap_async<E>(pin, pout, L);
            if (rc != HPX_OK) return rc;
        } else {
            if (s == 64)
                k_remap<E, 16><<<grid, kRemapThreads, smem, st>>>(pin, pout, np, nside, logs, log_tiles, nb, mpc, src,
                                                                  dst);
            else if (s == 32)
                k_remap<E, 4><<<grid, kRemapThreads, smem, st>>>(pin, pout, np, nside, logs, log_tiles, nb, mpc, src,
                                                                 dst);
            else
                k_remap<E, 1><<<grid, kRemapThreads, smem, st>>>(pin, pout, np, nside, logs, log_tiles, nb, mpc, src,
                                                                 dst);
            HPX_CUDA_TRY(cudaGetLastError());
        }
    }
    return HPX_OK;
}

// (order, origin, clockwise) of one side -> its transform; XY faces rotate by
// the origin counter-clockwise, or by minus the origin after the flip of a
// clockwise face (src/data_remapping/hpx_remapping_cuda.cu:413-417)
int remap_side(int32_t order, int32_t origin, int32_t clockwise, RemapSide* sd, const char* which) {
    if (order < HPX_ORDER_RING || order > HPX_ORDER_XY)
        return set_err(HPX_ERR_INVALID_ARG, std::string(which) + " order must be RING, NEST or XY");
    sd->order = order;
    sd->flip = 0;
    sd->rot = 0;
    if (order == HPX_ORDER_XY) {
        if (origin < HPX_ORIGIN_S || origin > HPX_ORIGIN_W)
            return set_err(HPX_ERR_INVALID_ARG, std::string("The ") + which + " origin must be one from S, E, N, W");
        sd->flip = clockwise ? 1 : 0;
        sd->rot = (clockwise ? -origin : origin) & 3;
    }
    return HPX_OK;
}

}  // namespace

namespace {
template <typename E>
int launch_healpy(const void* in, void* out, int64_t batch, int L, int M, int cs, bool pack, cudaStream_t st) {
    const int Mk = std::min(M, L);
    const dim3 grid((unsigned)(((pack ? Mk : M) + kHpTile - 1) / kHpTile), (unsigned)((L + kHpTile - 1) / kHpTile), 1);
    const int64_t src_stride = pack ? (int64_t)L * M : healpy_size(L, M);
    const int64_t dst_stride = pack ? healpy_size(L, M) : (int64_t)L * M;
    for (int64_t b = 0; b < batch; b += 65535) {
        dim3 g = grid;
        g.z = (unsigned)std::min<int64_t>(65535, batch - b);
        const E* s = (const E*)in + b * src_stride;
        E* d = (E*)out + b * dst_stride;
        if (pack) k_healpy<E, true><<<g, dim3(kHpTile, 8), 0, st>>>(s, d, L, M, cs);
        else k_healpy<E, false><<<g, dim3(kHpTile, 8), 0, st>>>(s, d, L, M, cs);
        HPX_CUDA_TRY(cudaGetLastError());
    }
    return HPX_OK;
}

int healpy_call(const void* in, void* out, int64_t batch, int32_t lmax, int32_t mmax, int32_t elem_bytes,
                int32_t cs_phase, bool pack, void* stream) {
    if (batch < 0) return set_err(HPX_ERR_INVALID_ARG, "negative batch");
    if (lmax < 1 || mmax < 1 || lmax > 65536 || mmax > 65536)
        return set_err(HPX_ERR_INVALID_ARG, "lmax and mmax must be in [1, 65536]");
    if (elem_bytes != 8 && elem_bytes != 16)
        return set_err(HPX_ERR_INVALID_ARG, "elem_bytes must be 8 (complex float) or 16 (complex double)");
    if (batch == 0) return HPX_OK;
    if (!in || !out) return set_err(HPX_ERR_INVALID_ARG, "null pointer");
    if ((((uintptr_t)in) | ((uintptr_t)out)) % (uintptr_t)elem_bytes)
        return set_err(HPX_ERR_INVALID_ARG, "in and out must be aligned to elem_bytes");
    const uint64_t per = (uint64_t)std::max<int64_t>((int64_t)lmax * mmax, healpy_size(lmax, mmax)) * elem_bytes;
    if ((uint64_t)batch > (1ull << 62) / per) return set_err(HPX_ERR_INVALID_ARG, "batch too large");
    const uint64_t in_bytes = (uint64_t)batch * elem_bytes * (pack ? (uint64_t)lmax * mmax : (uint64_t)healpy_size(lmax, mmax));
    const uint64_t out_bytes = (uint64_t)batch * elem_bytes * (pack ? (uint64_t)healpy_size(lmax, mmax) : (uint64_t)lmax * mmax);
    const uintptr_t a = (uintptr_t)in, b = (uintptr_t)out;
    if (a < b + out_bytes && b < a + in_bytes) return set_err(HPX_ERR_INVALID_ARG, "in and out overlap");
    cudaStream_t st = (cudaStream_t)stream;
    return elem_bytes == 8 ? launch_healpy<float2>(in, out, batch, lmax, mmax, cs_phase != 0, pack, st)
                           : launch_healpy<double2>(in, out, batch, lmax, mmax, cs_phase != 0, pack, st);
}
}  // namespace

extern "C" {

int hpx_remap(const void* in, void* out, int64_t batch, int32_t nside, int32_t elem_bytes, int32_t src_order,
              int32_t src_origin, int32_t src_clockwise, int32_t dst_order, int32_t dst_origin,
              int32_t dst_clockwise, void* stream) {
    if (batch < 0) return set_err(HPX_ERR_INVALID_ARG, "negative batch");
    if (nside < 1 || nside > 8192 || ilog2_exact(nside) < 0)
        return set_err(HPX_ERR_INVALID_ARG, "nside must be a power of two in [1, 8192]");
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16)
        return set_err(HPX_ERR_INVALID_ARG, "elem_bytes must be 1, 2, 4, 8 or 16");
    RemapSide src, dst;
    int rc = remap_side(src_order, src_origin, src_clockwise, &src, "src");
    if (rc != HPX_OK) return rc;
    rc = remap_side(dst_order, dst_origin, dst_clockwise, &dst, "dest");
    if (rc != HPX_OK) return rc;
    if (batch == 0) return HPX_OK;
    if (!in || !out) return set_err(HPX_ERR_INVALID_ARG, "null pointer");
    if ((((uintptr_t)in) | ((uintptr_t)out)) % (uintptr_t)elem_bytes)
        return set_err(HPX_ERR_INVALID_ARG, "in and out must be aligned to elem_bytes");
    // bytes of one batch, bounded by 2^62 so that neither the product nor the
    // overlap test's sums (user addresses are below 2^57) can wrap
    const uint64_t per_map = 12ull * (uint64_t)nside * (uint64_t)nside * (uint64_t)elem_bytes;
    if ((uint64_t)batch > (1ull << 62) / per_map) return set_err(HPX_ERR_INVALID_ARG, "batch too large");
    const uint64_t bytes = (uint64_t)batch * per_map;
    const uintptr_t a = (uintptr_t)in, b = (uintptr_t)out;
    if (a < b + bytes && b < a + bytes) return set_err(HPX_ERR_INVALID_ARG, "in and out overlap");
    cudaStream_t st = (cudaStream_t)stream;
    if (src.order == dst.order && src.flip == dst.flip && src.rot == dst.rot) {
        HPX_CUDA_TRY(cudaMemcpyAsync(out, in, bytes, cudaMemcpyDeviceToDevice, st));
        return HPX_OK;
    }
    switch (elem_bytes) {
        case 1: return launch_remap<uint8_t>(in, out, batch, nside, src, dst, st);
        case 2: return launch_remap<uint16_t>(in, out, batch, nside, src, dst, st);
        case 4: return launch_remap<uint32_t>(in, out, batch, nside, src, dst, st);
        case 8: return launch_remap<unsigned long long>(in, out, batch, nside, src, dst, st);
        default: return launch_remap<uint4>(in, out, batch, nside, src, dst, st);
    }
}

int hpx_alm_to_healpy(const void* alm, void* packed, int64_t batch, int32_t lmax, int32_t mmax, int32_t elem_bytes,
                      int32_t cs_phase, void* stream) {
    return healpy_call(alm, packed, batch, lmax, mmax, elem_bytes, cs_phase, true, stream);
}

int hpx_healpy_to_alm(const void* packed, void* alm, int64_t batch, int32_t lmax, int32_t mmax, int32_t elem_bytes,
                      int32_t cs_phase, void* stream) {
    return healpy_call(packed, alm, batch, lmax, mmax, elem_bytes, cs_phase, false, stream);
}

int hpx_sht_forward_noalloc(hpx_plan_t plan, const void* map, void* alm, int64_t batch, void* stream) {
    if (!plan) return set_err(HPX_ERR_INVALID_ARG, "null plan");
    if (batch < 0) return set_err(HPX_ERR_INVALID_ARG, "negative batch");
    if (batch == 0) return HPX_OK;
    if (!map || !alm) return set_err(HPX_ERR_INVALID_ARG, "null data pointer");
    const size_t need = noalloc_need(plan);
    if (need > kNoAllocScratchBytes)
        return set_err(HPX_ERR_WORKSPACE, "hpx_sht_forward_noalloc: this plan needs " + std::to_string(need) +
                                              " bytes of scratch per chunk of " + std::to_string(plan->batch_chunk) +
                                              " maps, above the static scratch of " +
                                              std::to_string(kNoAllocScratchBytes) +
                                              " bytes; use hpx_sht_forward with a workspace");
    DeviceGuard g(plan->device);
    unsigned char* scratch = nullptr;
    int rc = noalloc_scratch(plan->device, &scratch);
    if (rc != HPX_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    try {
        return plan->f64 ? run_forward_noalloc<double>(plan, map, alm, batch, scratch, st)
                         : run_forward_noalloc<float>(plan, map, alm, batch, scratch, st);
    } catch (const std::exception& ex) {
        return set_err(HPX_ERR_CUDA, ex.what());
    }
}

int hpx_plan_create(const hpx_desc_t* desc, hpx_plan_t* plan) {
    if (!desc || !plan) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    *plan = nullptr;
    if (desc->nside < 1 || desc->nside > 8192) return set_err(HPX_ERR_INVALID_ARG, "nside must be in [1, 8192]");
    if (desc->lmax < 1 || desc->mmax < 1) return set_err(HPX_ERR_INVALID_ARG, "lmax and mmax must be >= 1");
    if (desc->lmax > 65536 || desc->mmax > 65536) return set_err(HPX_ERR_INVALID_ARG, "lmax/mmax too large");
    if (desc->precision < HPX_PREC_FP32 || desc->precision > HPX_PREC_F16X3)
        return set_err(HPX_ERR_INVALID_ARG, "unknown precision");
    if (desc->batch_chunk < 0 || desc->batch_chunk > 4096) return set_err(HPX_ERR_INVALID_ARG, "batch_chunk out of range");
    if (desc->refine_iters < 0 || desc->refine_iters > 64) return set_err(HPX_ERR_INVALID_ARG, "refine_iters out of range");
    if (desc->flags & ~HPX_FLAG_OTF_LEGENDRE) return set_err(HPX_ERR_INVALID_ARG, "unknown flag bits");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(HPX_ERR_CUDA, "no CUDA device");
    }
    if (desc->device < 0 || desc->device >= ndev) return set_err(HPX_ERR_INVALID_ARG, "bad device ordinal");
    hpx_plan_s* P = new (std::nothrow) hpx_plan_s();
    if (!P) return set_err(HPX_ERR_OOM, "host allocation failed");
    DeviceGuard g(desc->device);
    int rc;
    try {
        plan_init(desc, P);
        healpix_pairs(desc, P);
        rc = plan_build(P);
    } catch (const std::bad_alloc&) {
        rc = set_err(HPX_ERR_OOM, "host allocation failed");
    } catch (const std::exception& ex) {
        rc = set_err(HPX_ERR_CUDA, ex.what());
    }
    if (rc != HPX_OK) {
        delete P;
        return rc;
    }
    *plan = P;
    return HPX_OK;
}

int hpx_plan_create_latlon(const hpx_latlon_desc_t* desc, hpx_plan_t* plan) {
    if (!desc || !plan) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    *plan = nullptr;
    if (desc->nlat < 2 || desc->nlat > 16384) return set_err(HPX_ERR_INVALID_ARG, "nlat must be in [2, 16384]");
    if (desc->nlon < 2 || desc->nlon > 32768 || (desc->nlon & 1))
        return set_err(HPX_ERR_INVALID_ARG, "nlon must be even and in [2, 32768]");
    if (desc->lmax < 1 || desc->mmax < 1 || desc->lmax > 65536 || desc->mmax > 65536)
        return set_err(HPX_ERR_INVALID_ARG, "lmax and mmax must be in [1, 65536]");
    if (desc->grid < HPX_GRID_EQUIANGULAR || desc->grid > HPX_GRID_LOBATTO)
        return set_err(HPX_ERR_INVALID_ARG, "unknown grid");
    if (desc->precision < HPX_PREC_FP32 || desc->precision > HPX_PREC_F16X3)
        return set_err(HPX_ERR_INVALID_ARG, "unknown precision");
    if (desc->batch_chunk < 0 || desc->batch_chunk > 4096) return set_err(HPX_ERR_INVALID_ARG, "batch_chunk out of range");
    if ((desc->flags & ~HPX_FLAG_OTF_LEGENDRE) || desc->reserved != 0)
        return set_err(HPX_ERR_INVALID_ARG, "unknown flag bits");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_err(HPX_ERR_CUDA, "no CUDA device");
    }
    if (desc->device < 0 || desc->device >= ndev) return set_err(HPX_ERR_INVALID_ARG, "bad device ordinal");
    hpx_plan_s* P = new (std::nothrow) hpx_plan_s();
    if (!P) return set_err(HPX_ERR_OOM, "host allocation failed");
    DeviceGuard g(desc->device);
    int rc;
    try {
        hpx_desc_t d{};
        d.nside = 0;
        d.lmax = desc->lmax;
        d.mmax = desc->mmax;
        d.precision = desc->precision;
        d.batch_chunk = desc->batch_chunk;
        d.device = desc->device;
        d.flags = desc->flags;
        plan_init(&d, P);
        std::vector<double> z, s2, w;
        latlon_quadrature(desc->grid, desc->nlat, z, s2, w);
        latlon_pairs(desc->nlat, desc->nlon, z, s2, w, P);
        rc = plan_build(P);
    } catch (const std::bad_alloc&) {
        rc = set_err(HPX_ERR_OOM, "host allocation failed");
    } catch (const std::exception& ex) {
        rc = set_err(HPX_ERR_CUDA, ex.what());
    }
    if (rc != HPX_OK) {
        delete P;
        return rc;
    }
    *plan = P;
    return HPX_OK;
}

int hpx_plan_destroy(hpx_plan_t plan) {
    if (!plan) return HPX_OK;
    delete plan;
    return HPX_OK;
}

int hpx_workspace_size(hpx_plan_t plan, int64_t batch, size_t* bytes) {
    if (!plan || !bytes) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    (void)batch;  // the batch is processed in chunks of batch_chunk maps
    size_t s = ((plan->spec_bytes() + 255) & ~(size_t)255) + ((plan->almT_bytes() + 255) & ~(size_t)255) +
               ((plan->resid_bytes() + 255) & ~(size_t)255);
    s += (plan->tcA_bytes() + 255) & ~(size_t)255;
    s += (plan->F_bytes() + 255) & ~(size_t)255;
    s += plan->scale_bytes();
    *bytes = s;
    return HPX_OK;
}

// Ragged calls place the groups' workspaces one after another (256-byte
// aligned) so that the groups can run at the same time on streams of their
// own; a smaller workspace (at least the largest group's) runs them one after
// another in it.
namespace {
size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
}  // namespace

int hpx_ragged_workspace_size(const hpx_plan_t* plans, int32_t n_groups, const int64_t* batches, size_t* bytes) {
    if (!plans || !batches || !bytes || n_groups < 0) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    size_t need = 0;
    for (int g = 0; g < n_groups; ++g) {
        if (!plans[g] || batches[g] < 0) return set_err(HPX_ERR_INVALID_ARG, "invalid group " + std::to_string(g));
        size_t b = 0;
        hpx_workspace_size(plans[g], batches[g], &b);
        need += align256(b);
    }
    *bytes = need;
    return HPX_OK;
}

namespace {
// Streams and events the concurrent ragged groups fork onto, per device,
// created on the first ragged call (make it outside stream capture) and kept
// for the life of the process.
constexpr int kRaggedStreams = 8;
struct RaggedPool {
    cudaStream_t s[kRaggedStreams] = {};
    cudaEvent_t fork = nullptr, done[kRaggedStreams] = {};
    bool ready = false;
};
std::mutex g_ragged_mu;
RaggedPool g_ragged_pool[kNoAllocMaxDevices];

int ragged(Op op, const hpx_plan_t* plans, int32_t n_groups, const void* const* ins, void* const* outs,
           const int64_t* batches, void* ws, size_t ws_bytes, void* stream) {
    if (!plans || !ins || !outs || !batches || n_groups < 0) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    size_t largest = 0, total = 0;
    for (int g = 0; g < n_groups; ++g) {
        if (!plans[g] || batches[g] < 0 || (batches[g] > 0 && (!ins[g] || !outs[g])))
            return set_err(HPX_ERR_INVALID_ARG, "invalid group " + std::to_string(g));
        if (plans[g]->device != plans[0]->device) return set_err(HPX_ERR_INVALID_ARG, "plans on different devices");
        size_t b = 0;
        hpx_workspace_size(plans[g], batches[g], &b);
        largest = std::max(largest, b);
        total += align256(b);
    }
    if (n_groups == 0) return HPX_OK;
    if (!ws || ws_bytes < largest)
        return set_err(HPX_ERR_WORKSPACE, "workspace too small: need " + std::to_string(total) + " bytes (at least " +
                                              std::to_string(largest) + "), got " + std::to_string(ws_bytes));
    if (((uintptr_t)ws & 255) != 0) return set_err(HPX_ERR_INVALID_ARG, "workspace must be 256-byte aligned");
    int active = 0;
    for (int g = 0; g < n_groups; ++g) active += batches[g] > 0;
    if (ws_bytes < total || active < 2) {
        for (int g = 0; g < n_groups; ++g) {
            const int rc = dispatch(plans[g], op, ins[g], outs[g], batches[g], ws, ws_bytes, stream);
            if (rc != HPX_OK) return rc;
        }
        return HPX_OK;
    }
    const int dev = plans[0]->device;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_err(HPX_ERR_UNSUPPORTED, "device ordinal above 63");
    DeviceGuard dg(dev);
    std::lock_guard<std::mutex> lk(g_ragged_mu);
    RaggedPool& pool = g_ragged_pool[dev];
    if (!pool.ready) {
        for (int i = 0; i < kRaggedStreams; ++i) {
            HPX_CUDA_TRY(cudaStreamCreateWithFlags(&pool.s[i], cudaStreamNonBlocking));
            HPX_CUDA_TRY(cudaEventCreateWithFlags(&pool.done[i], cudaEventDisableTiming));
        }
        HPX_CUDA_TRY(cudaEventCreateWithFlags(&pool.fork, cudaEventDisableTiming));
        pool.ready = true;
    }
    cudaStream_t st = (cudaStream_t)stream;
    HPX_CUDA_TRY(cudaEventRecord(pool.fork, st));
    size_t off = 0;
    int k = 0, rc = HPX_OK;
    bool used[kRaggedStreams] = {};
    for (int g = 0; g < n_groups && rc == HPX_OK; ++g) {
        size_t b = 0;
        hpx_workspace_size(plans[g], batches[g], &b);
        if (batches[g] > 0) {
            const int i = k++ % kRaggedStreams;
            if (!used[i]) {
                const cudaError_t e = cudaStreamWaitEvent(pool.s[i], pool.fork, 0);
                if (e != cudaSuccess) {
                    rc = set_err(HPX_ERR_CUDA, std::string("ragged fork: ") + cudaGetErrorString(e));
                    break;
                }
                used[i] = true;
            }
            rc = dispatch(plans[g], op, ins[g], outs[g], batches[g], (char*)ws + off, align256(b), pool.s[i]);
        }
        off += align256(b);
    }
    // join every stream used (also after an error, so that no fork is left open)
    for (int i = 0; i < kRaggedStreams; ++i) {
        if (!used[i]) continue;
        cudaError_t e = cudaEventRecord(pool.done[i], pool.s[i]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, pool.done[i], 0);
        if (e != cudaSuccess && rc == HPX_OK) rc = set_err(HPX_ERR_CUDA, std::string("ragged join: ") + cudaGetErrorString(e));
    }
    return rc;
}
}  // namespace

int hpx_ragged_forward(const hpx_plan_t* plans, int32_t n_groups, const void* const* maps, void* const* alms,
                       const int64_t* batches, void* ws, size_t ws_bytes, void* stream) {
    return ragged(kForward, plans, n_groups, maps, alms, batches, ws, ws_bytes, stream);
}
int hpx_ragged_inverse(const hpx_plan_t* plans, int32_t n_groups, const void* const* alms, void* const* maps,
                       const int64_t* batches, void* ws, size_t ws_bytes, void* stream) {
    return ragged(kInverse, plans, n_groups, alms, maps, batches, ws, ws_bytes, stream);
}

int hpx_sht_forward(hpx_plan_t plan, const void* map, void* alm, int64_t batch, void* ws, size_t ws_bytes,
                    void* stream) {
    return dispatch(plan, kForward, map, alm, batch, ws, ws_bytes, stream);
}
int hpx_sht_inverse(hpx_plan_t plan, const void* alm, void* map, int64_t batch, void* ws, size_t ws_bytes,
                    void* stream) {
    return dispatch(plan, kInverse, alm, map, batch, ws, ws_bytes, stream);
}
int hpx_sht_forward_refined(hpx_plan_t plan, const void* map, void* alm, int64_t batch, int32_t iters, void* ws,
                            size_t ws_bytes, void* stream) {
    if (!plan) return set_err(HPX_ERR_INVALID_ARG, "null plan");
    if (iters < 0) iters = plan->desc.refine_iters;
    if (iters > 64) return set_err(HPX_ERR_INVALID_ARG, "iters out of range");
    return dispatch(plan, kForwardRefined, map, alm, batch, ws, ws_bytes, stream, iters);
}
int hpx_sht_forward_adjoint(hpx_plan_t plan, const void* alm_grad, void* map_grad, int64_t batch, void* ws,
                            size_t ws_bytes, void* stream) {
    return dispatch(plan, kForwardAdjoint, alm_grad, map_grad, batch, ws, ws_bytes, stream);
}
int hpx_sht_inverse_adjoint(hpx_plan_t plan, const void* map_grad, void* alm_grad, int64_t batch, void* ws,
                            size_t ws_bytes, void* stream) {
    return dispatch(plan, kInverseAdjoint, map_grad, alm_grad, batch, ws, ws_bytes, stream);
}

int hpx_vsht_forward(hpx_plan_t plan, const void* map, void* alm, int64_t batch, int32_t csphase, void* ws,
                     size_t ws_bytes, void* stream) {
    return dispatch_vec(plan, kForward, map, alm, batch, csphase, ws, ws_bytes, stream);
}
int hpx_vsht_inverse(hpx_plan_t plan, const void* alm, void* map, int64_t batch, int32_t csphase, void* ws,
                     size_t ws_bytes, void* stream) {
    return dispatch_vec(plan, kInverse, alm, map, batch, csphase, ws, ws_bytes, stream);
}
int hpx_vsht_forward_adjoint(hpx_plan_t plan, const void* alm_grad, void* map_grad, int64_t batch, int32_t csphase,
                             void* ws, size_t ws_bytes, void* stream) {
    return dispatch_vec(plan, kForwardAdjoint, alm_grad, map_grad, batch, csphase, ws, ws_bytes, stream);
}
int hpx_vsht_inverse_adjoint(hpx_plan_t plan, const void* map_grad, void* alm_grad, int64_t batch, int32_t csphase,
                             void* ws, size_t ws_bytes, void* stream) {
    return dispatch_vec(plan, kInverseAdjoint, map_grad, alm_grad, batch, csphase, ws, ws_bytes, stream);
}

int hpx_plan_get_schedule(hpx_plan_t plan, hpx_schedule_t* s) {
    if (!plan || !s) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    s->ring_maps_per_cta = plan->ring_g;
    s->ring_streams = plan->ring_streams;
    s->fwd_deal = plan->tc.fwd_deal;
    s->inv_deal = plan->tc.inv_deal;
    s->ctas = plan->tc.ctas;
    return HPX_OK;
}

int hpx_plan_set_schedule(hpx_plan_t plan, const hpx_schedule_t* s) {
    if (!plan || !s) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    const int g = s->ring_maps_per_cta;
    if (g != 4 && g != 8 && g != 16 && g != 32) return set_err(HPX_ERR_INVALID_ARG, "ring_maps_per_cta must be 4, 8, 16 or 32");
    for (int d : {s->fwd_deal, s->inv_deal})
        if (d < HPX_DEAL_ORDER_SNAKE || d > HPX_DEAL_CONTIGUOUS) return set_err(HPX_ERR_INVALID_ARG, "unknown deal");
    if (s->ctas < 0) return set_err(HPX_ERR_INVALID_ARG, "negative CTA count");
    if (s->ring_streams != 1 && s->ring_streams != 2) return set_err(HPX_ERR_INVALID_ARG, "ring_streams must be 1 or 2");
    DeviceGuard g_(plan->device);
    if (plan->tc.active) {
        HPX_CUDA_TRY(cudaDeviceSynchronize());  // no launch of this plan may still read the old lists
        const int rc = tc_deal(plan, s->fwd_deal, s->inv_deal, s->ctas);
        if (rc != HPX_OK) return rc;
    }
    plan->tc.fwd_deal = s->fwd_deal;  // kept (and reported) for plans without tensor-core tiles too
    plan->tc.inv_deal = s->inv_deal;
    plan->tc.ctas = s->ctas;
    plan->ring_g = g;
    plan->ring_streams = s->ring_streams;
    return HPX_OK;
}

int hpx_plan_table_bytes(hpx_plan_t plan, size_t* bytes) {
    if (!plan || !bytes) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    *bytes = plan->tc.table ? plan->tc.table_bytes : 0;
    return HPX_OK;
}

int hpx_plan_table_stream_bytes(hpx_plan_t plan, size_t* fwd, size_t* inv) {
    if (!plan || !fwd || !inv) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    *fwd = plan->tc.table ? plan->tc.stream_fwd : 0;
    *inv = plan->tc.table ? plan->tc.stream_inv : 0;
    return HPX_OK;
}

int hpx_plan_check(hpx_plan_t plan, void* stream) {
    if (!plan) return set_err(HPX_ERR_INVALID_ARG, "null plan");
    DeviceGuard dg(plan->device);
#ifdef HPX_CHECK_BOUNDS
    {
        HPX_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
        int oob = 0;
        HPX_CUDA_TRY(cudaMemcpyFromSymbol(&oob, g_hpx_oob, sizeof(int)));
        if (oob != 0) {
            const int zero = 0;
            cudaMemcpyToSymbol(g_hpx_oob, &zero, sizeof(int));
            return set_err(HPX_ERR_BOUNDS, "out-of-bounds access skipped (site code " + std::to_string(oob) + ")");
        }
    }
#endif
    if (!plan->tc.d_err) return HPX_OK;
    int h = 0;
    HPX_CUDA_TRY(cudaMemcpyAsync(&h, plan->tc.d_err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    HPX_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    if (h != 0) {
        cudaMemsetAsync(plan->tc.d_err, 0, sizeof(int), (cudaStream_t)stream);
        cudaStreamSynchronize((cudaStream_t)stream);
        return set_err(HPX_ERR_TIMEOUT, "tensor-core pipeline wait timed out (code " + std::to_string(h) + ")");
    }
    return HPX_OK;
}

int hpx_stats_enable(hpx_plan_t plan, int enable) {
    if (!plan) return set_err(HPX_ERR_INVALID_ARG, "null plan");
    std::lock_guard<std::mutex> g(plan->stats_mu);
    plan->stats_on = enable != 0;
    if (enable) {
        for (int i = 0; i < kNumStages; ++i) {
            plan->stat_launch[i] = 0;
            plan->stat_ms[i] = 0.0;
        }
    }
    return HPX_OK;
}

int hpx_stats_read(hpx_plan_t plan, hpx_stage_stat_t* out, int max_stages, int* n_stages) {
    if (!plan || (!out && max_stages > 0)) return set_err(HPX_ERR_INVALID_ARG, "null argument");
    DeviceGuard dg(plan->device);
    std::lock_guard<std::mutex> g(plan->stats_mu);
    for (auto& r : plan->stats_recs) {
        float ms = 0.f;
        if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess)
            return set_err(HPX_ERR_CUDA, "event timing failed");
        plan->stat_launch[r.stage] += 1;
        plan->stat_ms[r.stage] += ms;
        plan->ev_pool.push_back(r.a);
        plan->ev_pool.push_back(r.b);
    }
    plan->stats_recs.clear();
    const int n = std::min(max_stages, (int)kNumStages);
    for (int i = 0; i < n; ++i) {
        out[i].name = kStageNames[i];
        out[i].launches = plan->stat_launch[i];
        out[i].total_ms = plan->stat_ms[i];
    }
    for (int i = 0; i < kNumStages; ++i) {
        plan->stat_launch[i] = 0;
        plan->stat_ms[i] = 0.0;
    }
    if (n_stages) *n_stages = kNumStages;
    return HPX_OK;
}

int hpx_plan_info(hpx_plan_t plan, int32_t* nside, int32_t* lmax, int32_t* mmax, int32_t* precision) {
    if (!plan) return set_err(HPX_ERR_INVALID_ARG, "null plan");
    if (nside) *nside = plan->nside;
    if (lmax) *lmax = plan->L;
    if (mmax) *mmax = plan->M;
    if (precision) *precision = plan->prec;
    return HPX_OK;
}

const char* hpx_last_error(hpx_plan_t) { return g_last_error.c_str(); }

const char* hpx_status_string(int status) {
    switch (status) {
        case HPX_OK: return "ok";
        case HPX_ERR_INVALID_ARG: return "invalid argument";
        case HPX_ERR_OOM: return "out of memory";
        case HPX_ERR_CUDA: return "CUDA error";
        case HPX_ERR_TIMEOUT: return "timeout";
        case HPX_ERR_UNSUPPORTED: return "unsupported";
        case HPX_ERR_WORKSPACE: return "workspace too small";
        case HPX_ERR_BOUNDS: return "out-of-bounds access";
        default: return "unknown status";
    }
}

#ifdef HPX_TC_PROFILE
// Instrumented builds only: copy and clear the per-CTA role timers.
extern "C" HPX_API int hpx_tc_profile_read(unsigned long long* out) {
    cudaMemcpyFromSymbol(out, g_tc_prof, sizeof(g_tc_prof));
    static unsigned long long zero[2][296][kTcpSlots];
    cudaMemcpyToSymbol(g_tc_prof, zero, sizeof(g_tc_prof));
    return HPX_OK;
}
#endif

const char* hpx_version(void) { return "hpx_b200 0.1.0 (sm_100a)"; }

}  // extern "C"
