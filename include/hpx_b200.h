/*
 * hpx_b200 -- HEALPix real spherical-harmonic transforms on NVIDIA B200 (sm_100a).
 *
 * C ABI of the transform library (libhpx_b200.so).  Every entry point returns
 * an int status (hpx_status_t); no C++ exception crosses this boundary and the
 * library never calls exit().  Pointers are plain device pointers; streams are
 * cudaStream_t passed as void*.
 *
 * The functions replace the native layer of cuHPX's SHT path (paths relative
 * to the cuHPX repository):
 *   hpx_plan_create        cuhpx/hpx_sht.py:645-683, 696-730 (SHTCUDA/iSHTCUDA
 *                          constructors: weights, Legendre table, W) and the
 *                          HealpixFFT/HealpixIFFT plan singletons
 *                          (src/harmonic_transform/hpx_fft.h:69-255)
 *   hpx_sht_forward        cuhpx/hpx_sht.py:518-562 (SHTFunction.forward:
 *                          healpix_rfft_batch, hpx_fft.cpp:21-84, + einsum)
 *   hpx_sht_inverse        cuhpx/hpx_sht.py:589-611 (iSHTFunction.forward:
 *                          einsum + healpix_irfft_batch, hpx_fft.cpp:86-149)
 *   hpx_sht_forward_adjoint  exact adjoint of hpx_sht_forward; replaces the
 *                          approximate SHTFunction.backward (hpx_sht.py:565-583)
 *   hpx_sht_inverse_adjoint  exact adjoint of hpx_sht_inverse; replaces
 *                          iSHTFunction.backward (hpx_sht.py:614-641)
 *
 * Data layouts (row-major, batch outermost):
 *   map   [batch][12*nside^2]  real (float for FP32/mixed plans, double for FP64)
 *   alm   [batch][lmax][mmax]  complex interleaved (re, im); entries m > l are 0
 */
#ifndef HPX_B200_H
#define HPX_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HPX_API __attribute__((visibility("default")))
#else
#define HPX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    HPX_OK = 0,
    HPX_ERR_INVALID_ARG = 1,
    HPX_ERR_OOM = 2,
    HPX_ERR_CUDA = 3,
    HPX_ERR_TIMEOUT = 4,
    HPX_ERR_UNSUPPORTED = 5,
    HPX_ERR_WORKSPACE = 6,
    HPX_ERR_BOUNDS = 7   /* bounds-checked debug builds only: an access outside a buffer was skipped */
} hpx_status_t;

/* Arithmetic of the Legendre contraction.  FFT stages run in float for
 * FP32/BF16X3/F16X3/TF32 plans and in double for FP64 plans. */
typedef enum {
    HPX_PREC_FP32 = 0,   /* FP32 SIMT contraction ("plain FP32 path") */
    HPX_PREC_FP64 = 1,   /* FP64 everywhere (double I/O)              */
    HPX_PREC_BF16X3 = 2, /* tcgen05 BF16 3-term split (hi*hi + hi*lo + lo*hi),
                            FP32 accumulate; ~16-bit operands          */
    HPX_PREC_TF32 = 3,   /* tcgen05 TF32, FP32 accumulate (not built)  */
    HPX_PREC_F16X3 = 4   /* tcgen05 FP16 3-term split with a power-of-two
                            scale per map, FP32 accumulate; ~22-bit
                            operands, same speed as BF16X3             */
} hpx_precision_t;

typedef struct {
    int32_t nside;               /* HEALPix resolution, >= 1                          */
    int32_t lmax;                /* number of degrees l (l < lmax)                    */
    int32_t mmax;                /* number of orders m (m < mmax)                     */
    int32_t precision;           /* hpx_precision_t                                   */
    int32_t refine_iters;        /* default Jacobi iterations of hpx_sht_forward_refined */
    int32_t batch_chunk;         /* maps per internal pass (0 = default 64)           */
    int32_t device;              /* CUDA device ordinal the plan lives on             */
    int32_t flags;               /* HPX_FLAG_* bits, 0 by default                     */
    const double* ring_weights;  /* host array of 2*nside FITS ring-weight corrections
                                    (1 + w) factors are applied inside; NULL = uniform
                                    4*pi/npix ("none" quadrature)                     */
} hpx_desc_t;

/* Tensor-core plans (F16X3, BF16X3) keep the normalised Legendre values of
 * every (m, l, ring) resident on the device as hi/lo halves, 8 bytes per
 * (m, ring, degree pair) (34 GB at nside 1024, lmax = mmax = 2047), when that
 * fits in 45% of the device memory; the contraction then streams them with
 * TMA.  With this flag, or when the table does not fit, producer warps
 * generate them on the fly from FP64 seeds instead (slower, no table). */
#define HPX_FLAG_OTF_LEGENDRE 1

typedef struct hpx_plan_s* hpx_plan_t;

/* Build a plan: ring tables, Legendre start values (FP64 on the GPU), Bluestein
 * chirp spectra.  Immutable afterwards; usable concurrently from several streams
 * provided each call gets its own workspace. */
HPX_API int hpx_plan_create(const hpx_desc_t* desc, hpx_plan_t* plan);
HPX_API int hpx_plan_destroy(hpx_plan_t plan);

/* Bytes of device workspace a call with `batch` maps needs (same for every op). */
HPX_API int hpx_workspace_size(hpx_plan_t plan, int64_t batch, size_t* bytes);

/* Forward SHT (analysis): map -> alm. */
HPX_API int hpx_sht_forward(hpx_plan_t plan, const void* map, void* alm, int64_t batch,
                    void* workspace, size_t workspace_bytes, void* stream);
/* Inverse SHT (synthesis): alm -> map.  Imag parts of m=0 (and of the ring
 * Nyquist terms) are ignored, as an inverse real FFT does. */
HPX_API int hpx_sht_inverse(hpx_plan_t plan, const void* alm, void* map, int64_t batch,
                    void* workspace, size_t workspace_bytes, void* stream);
/* Forward SHT followed by `iters` Jacobi refinement steps
 *   alm <- alm + SHT(map - iSHT(alm))
 * (iters < 0 uses the plan's refine_iters).  Each step costs one inverse and one
 * forward transform; it removes the HEALPix quadrature error of band-limited
 * maps and the rounding error of reduced-precision contractions. */
HPX_API int hpx_sht_forward_refined(hpx_plan_t plan, const void* map, void* alm, int64_t batch, int32_t iters,
                            void* workspace, size_t workspace_bytes, void* stream);
/* Adjoint of hpx_sht_forward with respect to the real inner products
 * <x,y> = sum x*y (maps) and Re sum conj(a)*b (alm): alm-gradient -> map-gradient. */
HPX_API int hpx_sht_forward_adjoint(hpx_plan_t plan, const void* alm_grad, void* map_grad, int64_t batch,
                            void* workspace, size_t workspace_bytes, void* stream);
/* Adjoint of hpx_sht_inverse: map-gradient -> alm-gradient. */
HPX_API int hpx_sht_inverse_adjoint(hpx_plan_t plan, const void* map_grad, void* alm_grad, int64_t batch,
                            void* workspace, size_t workspace_bytes, void* stream);

/* Forward SHT (analysis) that allocates nothing and takes no workspace.  No
 * counterpart in cuHPX: it is added for callers that cannot hand the library
 * device memory, such as an FFI host with no device allocator of its own, or a
 * loop whose allocator may not be called because cudaMalloc/cudaFree
 * synchronise the device and would stall the other streams' work.
 * It runs the same kernels as hpx_sht_forward, with the ring and folded spectra
 * of one chunk of batch_chunk maps kept in one static device array of
 * 32 MiB (33554432 bytes) per device, shared by every plan and call on that
 * device.  A plan whose chunk needs more (per chunk of 64 maps: about 28 MiB at
 * nside 64, lmax = mmax = 128 for FP32/BF16X3/F16X3; FP64 twice that) is refused with
 * HPX_ERR_WORKSPACE before anything runs.  Nothing in the array has to start
 * at zero.  Calls that overlap in time -- on two streams, or from two threads --
 * race on the array and give wrong results: serialise them.  The first call on
 * a device looks up the array's address (cudaGetSymbolAddress, with the plan's
 * device current); make that first call before any stream capture.  The
 * address belongs to the device's context: after cudaDeviceReset the next call
 * looks it up again (make that call outside stream capture too). */
HPX_API int hpx_sht_forward_noalloc(hpx_plan_t plan, const void* map, void* alm, int64_t batch, void* stream);

/* Spin-1 (vector) transforms: cuHPX's VectorSHT / VectoriSHT
 * (cuhpx/hpx_sht.py:286-444, table _precompute_dlegpoly, cuhpx/sht_tools.py:267-304).
 * A vector map is [batch][2][12*nside^2] (two real components), its
 * coefficients [batch][2][L][M] complex (spheroidal, toroidal; zeros for
 * m > l and for l = 0 ... as the reference gives them).  The plan must be a
 * HEALPix FP32 or FP64 plan created with lmax = L + 1 and mmax = M + 1 (the
 * table reaches degree L and order M); workspace as hpx_workspace_size.
 * csphase != 0 negates the odd orders, as the reference's default
 * csphase=True does.  The adjoints are exact (the reference differentiates
 * its einsums by autograd). */
HPX_API int hpx_vsht_forward(hpx_plan_t plan, const void* map, void* alm, int64_t batch, int32_t csphase,
                             void* workspace, size_t workspace_bytes, void* stream);
HPX_API int hpx_vsht_inverse(hpx_plan_t plan, const void* alm, void* map, int64_t batch, int32_t csphase,
                             void* workspace, size_t workspace_bytes, void* stream);
HPX_API int hpx_vsht_forward_adjoint(hpx_plan_t plan, const void* alm_grad, void* map_grad, int64_t batch,
                                     int32_t csphase, void* workspace, size_t workspace_bytes, void* stream);
HPX_API int hpx_vsht_inverse_adjoint(hpx_plan_t plan, const void* map_grad, void* alm_grad, int64_t batch,
                                     int32_t csphase, void* workspace, size_t workspace_bytes, void* stream);

/* Ragged batches: n_groups groups of maps, group g with its own plan (for
 * instance one plan per nside) transforming batches[g] contiguous maps
 * ins[g] -> outs[g], all in one call ordered on `stream`.  With a workspace
 * of hpx_ragged_workspace_size bytes (the groups' workspaces one after
 * another) the groups run at the same time on streams of the library's own,
 * forked from `stream` and joined back to it by events (valid under stream
 * capture; the library creates those streams on its first ragged call on a
 * device, so make that call outside capture); with a smaller workspace of at
 * least the largest group's size they run one after another in it.
 * Replaces a per-map loop over SHTCUDA objects; the sequence of launches can
 * be captured once in a CUDA graph.  An invalid group (null plan or pointer,
 * negative batch) fails the call before anything runs.  The plans must live
 * on one device. */
HPX_API int hpx_ragged_workspace_size(const hpx_plan_t* plans, int32_t n_groups, const int64_t* batches,
                                      size_t* bytes);
HPX_API int hpx_ragged_forward(const hpx_plan_t* plans, int32_t n_groups, const void* const* maps,
                               void* const* alms, const int64_t* batches, void* workspace, size_t workspace_bytes,
                               void* stream);
HPX_API int hpx_ragged_inverse(const hpx_plan_t* plans, int32_t n_groups, const void* const* alms,
                               void* const* maps, const int64_t* batches, void* workspace, size_t workspace_bytes,
                               void* stream);

/* Per-kernel timing.  While enabled, every kernel the plan launches is
 * bracketed by CUDA events recorded on the launch stream; hpx_stats_read
 * synchronises on those events and returns, per stage, the number of launches
 * and their summed device time since the last read (then resets).  Leave it
 * disabled while capturing a CUDA graph. */
typedef struct {
    const char* name;
    int64_t launches;
    double total_ms;
} hpx_stage_stat_t;
HPX_API int hpx_stats_enable(hpx_plan_t plan, int enable);
HPX_API int hpx_stats_read(hpx_plan_t plan, hpx_stage_stat_t* out, int max_stages, int* n_stages);

/* Synchronise `stream` and report whether a kernel of this plan gave up on a
 * bounded pipeline wait since the last check (HPX_ERR_TIMEOUT, flag cleared).
 * Bounds-checked builds (-DHPX_CHECK_BOUNDS) also report, first, an access
 * outside the current call's buffers that a kernel skipped (HPX_ERR_BOUNDS). */
HPX_API int hpx_plan_check(hpx_plan_t plan, void* stream);

/* Latitude-longitude grids (the destination side of cuHPX's Regridding,
 * cuhpx/hpx_regrid.py:21-91, which delegates it to torch_harmonics RealSHT /
 * InverseRealSHT): nlat rings from north to south, nlon samples each at
 * phi_k = 2 pi k / nlon, maps laid out [batch][nlat][nlon].  Nodes and
 * quadrature weights (summing to 2 over cos(theta)):
 *   EQUIANGULAR     theta_j = pi j / (nlat-1), poles included, Clenshaw-Curtis
 *   LEGENDRE_GAUSS  Gauss-Legendre nodes (exact to degree 2 nlat - 1)
 *   LOBATTO         Gauss-Lobatto nodes, poles included
 * Analysis: a_lm = sum_j w_j Pbar_l^m(cos theta_j) (2 pi/nlon) sum_k f_jk
 * e^{-i m phi_k}; synthesis as for HEALPix.  The orthonormal Pbar carry no
 * Condon-Shortley phase (as the HEALPix transforms).  Plans from this entry
 * point serve hpx_sht_forward/inverse and both adjoints. */
typedef enum { HPX_GRID_EQUIANGULAR = 0, HPX_GRID_LEGENDRE_GAUSS = 1, HPX_GRID_LOBATTO = 2 } hpx_grid_t;
typedef struct {
    int32_t nlat;         /* rings, >= 2                                      */
    int32_t nlon;         /* samples per ring, even, >= 2                     */
    int32_t lmax;         /* number of degrees                                */
    int32_t mmax;         /* number of orders (orders > nlon/2 are zero)      */
    int32_t grid;         /* hpx_grid_t                                       */
    int32_t precision;    /* hpx_precision_t                                  */
    int32_t batch_chunk;  /* maps per internal pass (0 = default 64)          */
    int32_t device;
    int32_t flags;        /* HPX_FLAG_* bits                                  */
    int32_t reserved;     /* must be 0                                        */
} hpx_latlon_desc_t;
HPX_API int hpx_plan_create_latlon(const hpx_latlon_desc_t* desc, hpx_plan_t* plan);

/* Launch schedule of a plan (no counterpart in cuHPX, whose einsum and cuFFT
 * calls have none): the autotuner of this library (cuhpx_b200/autotune.py)
 * times candidates and keeps the fastest per GPU and problem.
 *   ring_maps_per_cta  maps each ring-FFT CTA transforms (4, 8, 16 or 32; 16)
 *   fwd_deal, inv_deal how the persistent tensor-core kernels' tiles are dealt
 *                      to their CTAs (the m-to-CTA schedule), HPX_DEAL_*
 *   ctas               persistent CTAs of those kernels (0: one per SM)
 *   ring_streams       2 (default) or 1, see the field
 * hpx_plan_set_schedule synchronises the device and rewrites the plan's tile
 * lists: call it while no transform of the plan is in flight and outside
 * stream capture.  Every schedule gives bit-identical results: each tile and
 * each ring transform is computed the same way whichever CTA runs it. */
typedef enum {
    HPX_DEAL_ORDER_SNAKE = 0,  /* orders by total cost, round-robin snake (default) */
    HPX_DEAL_TILE_SNAKE = 1,   /* tiles by cost, round-robin snake               */
    HPX_DEAL_GREEDY = 2,       /* longest tile first onto the least-loaded CTA    */
    HPX_DEAL_CONTIGUOUS = 3    /* order sequence cut into equal-cost ranges       */
} hpx_deal_t;
typedef struct {
    int32_t ring_maps_per_cta;
    int32_t fwd_deal;
    int32_t inv_deal;
    int32_t ctas;
    int32_t ring_streams;  /* 2: the power-of-two and Bluestein ring launches overlap on two
                              streams (default); 1: they run one after the other on the call's stream */
} hpx_schedule_t;
HPX_API int hpx_plan_get_schedule(hpx_plan_t plan, hpx_schedule_t* schedule);
HPX_API int hpx_plan_set_schedule(hpx_plan_t plan, const hpx_schedule_t* schedule);

/* Bytes of the plan's resident Legendre table (0 when it has none). */
HPX_API int hpx_plan_table_bytes(hpx_plan_t plan, size_t* bytes);

/* Table bytes one analysis (fwd) and one synthesis (inv) pass over a chunk of
 * maps streams: the table's blocks that hold a nonzero entry for some tile
 * (all-zero blocks, at polar rings below the turning point, are skipped).
 * 0 and 0 when the plan has no table.  Introspection for roofline accounting;
 * no counterpart in cuHPX. */
HPX_API int hpx_plan_table_stream_bytes(hpx_plan_t plan, size_t* fwd, size_t* inv);

/* HEALPix pixel-order remapping (no plan needed): batch maps of
 * 12*nside^2 elements of elem_bytes bytes each (1, 2, 4, 8 or 16; the bytes are
 * moved, not interpreted), read in the src layout and written in the dst
 * layout to a separate buffer.  nside is a power of two up to 8192.
 * Layouts: RING and NEST are HEALPix's; XY ("flat") is face-major with each
 * face an nside x nside row-major grid whose first pixel sits at the face's
 * origin corner (S, E, N or W) and whose rows run counter-clockwise, or
 * clockwise, from it (origin and clockwise are ignored for RING and NEST).
 * Replaces cuHPX's cuhpx_remap module: ring2nest, nest2ring, nest2xy,
 * xy2nest, ring2xy, xy2ring, xy2xy and their _batch forms
 * (src/data_remapping/hpx_remapping.cpp:21-239, 241-450; bound at :452-476;
 * Python wrappers cuhpx/hpx_remap.py:24-102).  Runs on the stream's device;
 * allocates nothing; src == dst layouts copy. */
typedef enum { HPX_ORDER_RING = 0, HPX_ORDER_NEST = 1, HPX_ORDER_XY = 2 } hpx_order_t;
typedef enum { HPX_ORIGIN_S = 0, HPX_ORIGIN_E = 1, HPX_ORIGIN_N = 2, HPX_ORIGIN_W = 3 } hpx_origin_t;
HPX_API int hpx_remap(const void* in, void* out, int64_t batch, int32_t nside, int32_t elem_bytes,
                      int32_t src_order, int32_t src_origin, int32_t src_clockwise, int32_t dst_order,
                      int32_t dst_origin, int32_t dst_clockwise, void* stream);

/* healpy a_lm packing.  This library's coefficients are dense
 * [batch][lmax][mmax] complex (zeros for m > l); healpy keeps the m <= l
 * triangle in one vector per map, order by order:
 *   packed[m (2 lmax - 1 - m) / 2 + l] = alm[l][m],  m <= l < lmax, m < min(mmax, lmax)
 * (healpy's own lmax is this lmax - 1), packed length
 * min(mmax,lmax) * lmax - min(mmax,lmax) (min(mmax,lmax) - 1) / 2.
 * cs_phase != 0 multiplies order m by (-1)^m, the Condon-Shortley factor
 * between this library's (cuHPX's) phase convention and healpy's.
 * elem_bytes: 8 (complex float) or 16 (complex double).  Unpacking writes the
 * whole dense array, zeros included.  Runs on `stream`; allocates nothing.
 * Replaces the index map cuHPX states in
 * tests/reproduce_difference_between_healpy_cuhpx.py:58-81 (hp_getidx,
 * flm_hp_to_2d). */
HPX_API int hpx_alm_to_healpy(const void* alm, void* packed, int64_t batch, int32_t lmax, int32_t mmax,
                              int32_t elem_bytes, int32_t cs_phase, void* stream);
HPX_API int hpx_healpy_to_alm(const void* packed, void* alm, int64_t batch, int32_t lmax, int32_t mmax,
                              int32_t elem_bytes, int32_t cs_phase, void* stream);

/* Plan geometry queries. */
HPX_API int hpx_plan_info(hpx_plan_t plan, int32_t* nside, int32_t* lmax, int32_t* mmax, int32_t* precision);

/* Human-readable text of the last error seen by this plan (thread-local copy),
 * and of a status code. */
HPX_API const char* hpx_last_error(hpx_plan_t plan);
HPX_API const char* hpx_status_string(int status);

/* Library version string. */
HPX_API const char* hpx_version(void);

#ifdef __cplusplus
}
#endif

#endif /* HPX_B200_H */
