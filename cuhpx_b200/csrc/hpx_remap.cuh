// HEALPix pixel-order remapping between the RING, NEST and per-face "flat"
// (XY) layouts, for a batch of maps of any element width.
//
// Replaces the cuhpx_remap extension (src/data_remapping/hpx_remapping_cuda.cu,
// hpx_remapping.cpp; Python wrappers cuhpx/hpx_remap.py:24-102).  The
// reference builds, per call, four int arrays of npix entries with cudaMalloc
// (pixel -> x, y, face -> destination pixel, hpx_remapping_cuda.cu:550-640) and
// then scatters every element to its destination one at a time
// (rearrange_data_kernel_batch, :903-918): 16 bytes of index traffic per pixel
// and a scattered access per element.  Here nothing is allocated and no index
// array exists: the maps are cut into nside-aligned squares of S x S pixels of
// one base face (S = 64 or 32), the square's pixels are read in the source
// layout's natural order (one contiguous run in NEST, S rows in XY, 2S-1
// anti-diagonal runs in RING), staged in shared memory, and written in the
// destination layout's natural order.  The offsets are computed once per CTA
// and reused for each map of the CTA's group.
//
// Canonical pixel coordinates are HEALPix's (face f, ix, iy): ix runs to the
// north-east and iy to the north-west inside a base face (Gorski et al. 2005,
// ApJ 622:759).  The three layouts, as the reference defines them:
//   NEST:  f * nside^2 + spread(ix) + 2 * spread(iy)
//          (xyf2nest_kernel, hpx_remapping_cuda.cu:307-321)
//   RING:  the ring number jr and position jp of (f, ix, iy)
//          (xyf2ring_kernel, hpx_remapping_cuda.cu:228-283)
//   XY:    f * nside^2 + fy * nside + fx with (fx, fy) = rot^k(flip(ix, iy))
//          (correct_xy_orient and xyf2flat_kernel, :55-73, :100-134; flip =
//          clockwise, k = origin for counter-clockwise faces and -origin for
//          clockwise ones, :413-417).  A flat->flat remap of the reference
//          (:400-422) equals the destination transform composed with the
//          inverse of the source transform, which is what the kernels apply.
#pragma once

#include "hpx_common.cuh"

namespace hpx {

enum { kOrderRing = 0, kOrderNest = 1, kOrderXY = 2 };

struct RemapSide {
    int order;  // kOrderRing / kOrderNest / kOrderXY
    int flip;   // XY: swap ix and iy first
    int rot;    // XY: then this many quarter turns counter-clockwise
};

// interleave the low 16 bits of v with zeros: b0 b1 b2 .. -> b0 0 b1 0 b2 ..
HPX_HD uint32_t spread_bits2(uint32_t v) {
    v &= 0xffffu;
    v = (v | (v << 8)) & 0x00ff00ffu;
    v = (v | (v << 4)) & 0x0f0f0f0fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}
// inverse of spread_bits2 on the even bits of v
HPX_HD uint32_t compress_bits2(uint32_t v) {
    v &= 0x55555555u;
    v = (v | (v >> 1)) & 0x33333333u;
    v = (v | (v >> 2)) & 0x0f0f0f0fu;
    v = (v | (v >> 4)) & 0x00ff00ffu;
    v = (v | (v >> 8)) & 0x0000ffffu;
    return v;
}

// quarter turns counter-clockwise of a face's pixel grid; ~v = -v-1, and the
// mask (nside-1) wraps the result back into [0, nside)
HPX_HD void face_rotate(int& x, int& y, int k, int mask) {
    int nx = x, ny = y;
    if (k == 1) {
        nx = ~y;
        ny = x;
    } else if (k == 2) {
        nx = ~x;
        ny = ~y;
    } else if (k == 3) {
        nx = y;
        ny = ~x;
    }
    x = nx & mask;
    y = ny & mask;
}
HPX_HD void xy_to_flat(int& x, int& y, const RemapSide& s, int mask) {
    if (s.flip) {
        const int t = x;
        x = y;
        y = t;
    }
    face_rotate(x, y, s.rot, mask);
}
HPX_HD void flat_to_xy(int& x, int& y, const RemapSide& s, int mask) {
    face_rotate(x, y, (4 - s.rot) & 3, mask);
    if (s.flip) {
        const int t = x;
        x = y;
        y = t;
    }
}

// RING index of canonical pixel (f, ix, iy).  jr: ring number counted from 1
// at the north pole; nr: pixels of that ring per base face; jp: 1-based
// position in the ring (wraps once for the equatorial face 4, whose column
// starts at phi = 0).
HPX_HD int64_t xyf_to_ring(int ix, int iy, int f, int nside) {
    const int64_t n = nside;
    const int64_t jr = (int64_t)((f >> 2) + 2) * n - ix - iy - 1;
    int64_t nr, before;
    int kshift = 0;
    if (jr < n) {  // north polar cap
        nr = jr;
        before = 2 * jr * (jr - 1);
    } else if (jr < 3 * n) {  // equatorial belt (rings alternate their shift)
        nr = n;
        before = 2 * n * (n - 1) + (jr - n) * 4 * n;
        kshift = (int)((jr - n) & 1);
    } else {  // south polar cap
        const int64_t js = 4 * n - jr;
        nr = js;
        before = 12 * n * n - 2 * js * (js + 1);
    }
    const int jpll = ((f & 3) << 1) - ((f >> 2) & 1) + 1;  // face column, in half faces
    int64_t jp = (jpll * nr + ix - iy + 1 + kshift) / 2;  // numerator is even
    if (jp < 1) jp += 4 * n;
    return before + jp - 1;
}

// ------------------------------------------------------------- square tiles
// A tile is the s x s square [x0, x0+s) x [y0, y0+s) of face f (s a power of
// two dividing nside).  Each layout enumerates the tile's pixels in its own
// natural order, position p in [0, s*s):
//   NEST: the tile is one contiguous run; p = spread(lx) + 2 spread(ly).
//   XY:   p = row * s + column in the layout's own (fx, fy) frame.
//   RING: anti-diagonals u = lx + ly (one ring each) in increasing u, and along
//         one diagonal increasing lx (= increasing RING index).
struct Tile {
    int f, x0, y0, s, logs, nside, mask;
};

// position of (lx, ly) in the diagonal order of an s x s square
HPX_HD int diag_pos(int lx, int ly, int s) {
    const int u = lx + ly;
    if (u < s) return u * (u + 1) / 2 + lx;
    const int mx = s - 1 - lx, my = s - 1 - ly;  // mirrored into the lower triangle
    const int mu = mx + my;
    return s * s - 1 - (mu * (mu + 1) / 2 + mx);
}
HPX_HD void diag_lower(int p, int& lx, int& ly) {
    int u = (int)((sqrtf(8.0f * (float)p + 1.0f) - 1.0f) * 0.5f);
    while (u * (u + 1) / 2 > p) --u;
    while ((u + 1) * (u + 2) / 2 <= p) ++u;
    lx = p - u * (u + 1) / 2;
    ly = u - lx;
}
HPX_HD void diag_coords(int p, int s, int& lx, int& ly) {
    if (p < s * (s + 1) / 2) {
        diag_lower(p, lx, ly);
    } else {
        int mx, my;
        diag_lower(s * s - 1 - p, mx, my);
        lx = s - 1 - mx;
        ly = s - 1 - my;
    }
}

// origin of the tile in an XY layout's (fx, fy) frame: the transform maps
// each axis to +-ix or +-iy, so the extremes sit on the tile's diagonal corners
HPX_HD void flat_origin(const Tile& t, const RemapSide& sd, int& fx0, int& fy0) {
    int ax = t.x0, ay = t.y0, bx = t.x0 + t.s - 1, by = t.y0 + t.s - 1;
    xy_to_flat(ax, ay, sd, t.mask);
    xy_to_flat(bx, by, sd, t.mask);
    fx0 = ax < bx ? ax : bx;
    fy0 = ay < by ? ay : by;
}

// natural position of tile pixel (lx, ly) on side sd
HPX_HD int side_pos(const Tile& t, const RemapSide& sd, int fx0, int fy0, int lx, int ly) {
    if (sd.order == kOrderNest) return (int)(spread_bits2(lx) | (spread_bits2(ly) << 1));
    if (sd.order == kOrderRing) return diag_pos(lx, ly, t.s);
    int x = t.x0 + lx, y = t.y0 + ly;
    xy_to_flat(x, y, sd, t.mask);
    return ((y - fy0) << t.logs) + (x - fx0);
}
// tile pixel at natural position p of side sd
HPX_HD void side_coords(const Tile& t, const RemapSide& sd, int fx0, int fy0, int p, int& lx, int& ly) {
    if (sd.order == kOrderNest) {
        lx = (int)compress_bits2((uint32_t)p);
        ly = (int)compress_bits2((uint32_t)p >> 1);
    } else if (sd.order == kOrderRing) {
        diag_coords(p, t.s, lx, ly);
    } else {
        int x = fx0 + (p & (t.s - 1)), y = fy0 + (p >> t.logs);
        flat_to_xy(x, y, sd, t.mask);
        lx = x - t.x0;
        ly = y - t.y0;
    }
}
// offset inside one map of tile pixel (lx, ly) on side sd
HPX_HD uint32_t side_offset(const Tile& t, const RemapSide& sd, int lx, int ly) {
    const int ix = t.x0 + lx, iy = t.y0 + ly;
    const uint32_t face = (uint32_t)t.f * (uint32_t)t.nside * (uint32_t)t.nside;
    if (sd.order == kOrderNest) return face + spread_bits2(ix) + (spread_bits2(iy) << 1);
    if (sd.order == kOrderRing) return (uint32_t)xyf_to_ring(ix, iy, t.f, t.nside);
    int x = ix, y = iy;
    xy_to_flat(x, y, sd, t.mask);
    return face + (uint32_t)y * (uint32_t)t.nside + (uint32_t)x;
}

// shared-memory slot of natural position p: one pad word per 32 elements
// keeps transposed and diagonal reads off a single bank
HPX_HD int remap_slot(int p) { return p + (p >> 5); }

constexpr int kRemapThreads = 256;

// Offset of natural position p on side sd.  NEST and XY offsets follow from p
// (a NEST tile is one run from its first pixel; an XY tile is s rows of s);
// only RING needs the table ring_tab of the tile's s*s ring offsets.
HPX_HD uint32_t natural_offset(const RemapSide& sd, uint32_t base, int p, int logs, int nside,
                               const uint32_t* ring_tab) {
    if (sd.order == kOrderRing) return ring_tab[p];
    if (sd.order == kOrderNest) return base + (uint32_t)p;
    return base + (uint32_t)(p >> logs) * (uint32_t)nside + (uint32_t)(p & ((1 << logs) - 1));
}
HPX_HD uint32_t natural_base(const Tile& t, const RemapSide& sd, int fx0, int fy0) {
    const uint32_t face = (uint32_t)t.f * (uint32_t)t.nside * (uint32_t)t.nside;
    if (sd.order == kOrderNest) return face + spread_bits2(t.x0) + (spread_bits2(t.y0) << 1);
    if (sd.order == kOrderXY) return face + (uint32_t)fy0 * (uint32_t)t.nside + (uint32_t)fx0;
    return 0;
}

// Shared memory of one CTA: the staged tile(s), the tile slot that each
// destination-order pixel reads (u16), and the ring offsets (u32) of the side
// in RING order, if any (RING -> RING is a copy and never launches).
HPX_HD size_t remap_tile_bytes(int s, int elem) { return ((size_t)remap_slot(s * s) * (size_t)elem + 15) & ~(size_t)15; }
HPX_HD size_t remap_slot_bytes(int s) { return ((size_t)s * s * 2 + 15) & ~(size_t)15; }
HPX_HD size_t remap_smem_bytes(int s, int elem, bool ring) {
    return remap_tile_bytes(s, elem) + remap_slot_bytes(s) + (ring ? (size_t)s * s * 4 : 0);
}

// The tile of block b: face by face, and inside a face in NEST (Morton)
// order of the tiles' corners.  Fills the shared tables (ring offsets of the
// RING side, source slot of each destination-order pixel) and returns the
// natural bases of both sides.
__device__ __forceinline__ void remap_setup(Tile& t, int nside, int logs, int log_tiles, const RemapSide& src,
                                            const RemapSide& dst, uint16_t* sslot, uint32_t* ring_tab,
                                            uint32_t& sbase, uint32_t& dbase) {
    t.s = 1 << logs;
    t.logs = logs;
    t.nside = nside;
    t.mask = nside - 1;
    t.f = (int)(blockIdx.x >> (2 * log_tiles));
    const uint32_t ti = blockIdx.x & ((1u << (2 * log_tiles)) - 1u);
    t.x0 = (int)compress_bits2(ti) << logs;
    t.y0 = (int)compress_bits2(ti >> 1) << logs;
    const int ss = t.s * t.s;
    int sfx = 0, sfy = 0, dfx = 0, dfy = 0;
    if (src.order == kOrderXY) flat_origin(t, src, sfx, sfy);
    if (dst.order == kOrderXY) flat_origin(t, dst, dfx, dfy);
    sbase = natural_base(t, src, sfx, sfy);
    dbase = natural_base(t, dst, dfx, dfy);
    for (int p = threadIdx.x; p < ss; p += kRemapThreads) {
        int lx, ly;
        if (src.order == kOrderRing) {  // p-th pixel in source order
            side_coords(t, src, sfx, sfy, p, lx, ly);
            ring_tab[p] = side_offset(t, src, lx, ly);
        }
        side_coords(t, dst, dfx, dfy, p, lx, ly);  // p-th pixel in destination order
        if (dst.order == kOrderRing) ring_tab[p] = side_offset(t, dst, lx, ly);
        sslot[p] = (uint16_t)remap_slot(side_pos(t, src, sfx, sfy, lx, ly));
    }
}

// Elements of 1 or 2 bytes: one CTA per (tile, group of maps), R = ceil(s*s /
// 256) pixels per thread staged through registers; the next map's loads are
// issued before this map's stores.
template <typename E, int R>
__global__ void __launch_bounds__(kRemapThreads, 5) k_remap(const E* __restrict__ in, E* __restrict__ out,
                                                            int64_t npix, int nside, int logs, int log_tiles,
                                                            int nmaps, int maps_per_cta, RemapSide src,
                                                            RemapSide dst) {
    extern __shared__ __align__(16) unsigned char remap_smem[];
    const int s = 1 << logs, ss = s * s;
    E* tile = reinterpret_cast<E*>(remap_smem);
    uint16_t* sslot = reinterpret_cast<uint16_t*>(remap_smem + remap_tile_bytes(s, (int)sizeof(E)));
    uint32_t* ring_tab = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(sslot) + remap_slot_bytes(s));
    Tile t;
    uint32_t sbase, dbase;
    remap_setup(t, nside, logs, log_tiles, src, dst, sslot, ring_tab, sbase, dbase);
    __syncthreads();

    const int b0 = blockIdx.y * maps_per_cta;
    const int b1 = min(nmaps, b0 + maps_per_cta);
    E v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int p = threadIdx.x + r * kRemapThreads;
        if (p < ss) v[r] = in[(int64_t)b0 * npix + natural_offset(src, sbase, p, logs, nside, ring_tab)];
    }
    for (int b = b0; b < b1; ++b) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = threadIdx.x + r * kRemapThreads;
            if (p < ss) tile[remap_slot(p)] = v[r];
        }
        __syncthreads();
        if (b + 1 < b1) {
            const E* nb = in + (int64_t)(b + 1) * npix;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int p = threadIdx.x + r * kRemapThreads;
                if (p < ss) v[r] = nb[natural_offset(src, sbase, p, logs, nside, ring_tab)];
            }
        }
        E* ob = out + (int64_t)b * npix;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int p = threadIdx.x + r * kRemapThreads;
            if (p < ss) ob[natural_offset(dst, dbase, p, logs, nside, ring_tab)] = tile[sslot[p]];
        }
        __syncthreads();
    }
}

// Elements of 4, 8 or 16 bytes: the same tiles, compiled per (source order,
// destination order) so that no order test runs per element, with the loads
// issued as cp.async straight into a ring of kRemapStages staged tiles (each
// CTA keeps the next kRemapStages-1 maps' loads in flight, and no registers
// hold them) and one barrier per map ordering the ring.  NEST and XY sides
// move V = 16 / sizeof(E) consecutive pixels per access (one 16-byte cp.async
// or store: a NEST tile is one run, an XY tile s rows of s >= V); a RING side
// moves single elements along its diagonal runs, whose offsets come from the
// tile's table.  Shared-memory tiles are unpadded: the V-element vectors of
// each 32-element row are XOR-swizzled by the row number, which keeps every
// vector 16-byte aligned while spreading transposed and diagonal reads over
// the banks.  64 x 64 float tiles: 72 KB per CTA, three CTAs and six maps of
// loads (96 KB) in flight per SM.
constexpr int kRemapStages = 3;

template <int V>
HPX_HD int remap_swz(int p) {
    return p ^ (((p >> 5) & (32 / V - 1)) * V);
}
HPX_HD size_t remap_async_smem_bytes(int s, int elem, bool ring) {
    return kRemapStages * (((size_t)s * s * elem + 15) & ~(size_t)15) + remap_slot_bytes(s) +
           (ring ? (size_t)s * s * 4 : 0);
}

template <int BYTES>
__device__ __forceinline__ void cp_async_elem(void* smem, const void* gmem) {
    if constexpr (BYTES == 4)
        cp_async4(smem, gmem);
    else if constexpr (BYTES == 8)
        cp_async8(smem, gmem);
    else
        cp_async16(smem, gmem);
}

// offset of natural position p on a NEST or XY side (compile-time order)
template <int ORDER>
__device__ __forceinline__ uint32_t nat_offset(uint32_t base, int p, int logs, int nside) {
    if constexpr (ORDER == kOrderNest) return base + (uint32_t)p;
    return base + (uint32_t)(p >> logs) * (uint32_t)nside + (uint32_t)(p & ((1 << logs) - 1));
}

template <typename E, int SO, int DO>
__global__ void __launch_bounds__(kRemapThreads) k_remap_async(const E* __restrict__ in, E* __restrict__ out,
                                                               int64_t npix, int nside, int logs, int log_tiles,
                                                               int nmaps, int maps_per_cta, RemapSide src,
                                                               RemapSide dst, int vec) {
    static_assert(sizeof(E) == 4 || sizeof(E) == 8 || sizeof(E) == 16, "cp.async moves 4, 8 or 16 bytes");
    static_assert(SO != DO || SO == kOrderXY, "equal orders are a copy");
    constexpr int V = 16 / (int)sizeof(E);
    extern __shared__ __align__(16) unsigned char remap_smem[];
    const int s = 1 << logs, ss = s * s;
    const size_t tb = ((size_t)ss * sizeof(E) + 15) & ~(size_t)15;
    uint16_t* sslot = reinterpret_cast<uint16_t*>(remap_smem + kRemapStages * tb);
    uint32_t* ring_tab = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(sslot) + remap_slot_bytes(s));

    // tile, bases and tables (the slot table holds swizzled source positions)
    Tile t;
    t.s = s;
    t.logs = logs;
    t.nside = nside;
    t.mask = nside - 1;
    t.f = (int)(blockIdx.x >> (2 * log_tiles));
    const uint32_t ti = blockIdx.x & ((1u << (2 * log_tiles)) - 1u);
    t.x0 = (int)compress_bits2(ti) << logs;
    t.y0 = (int)compress_bits2(ti >> 1) << logs;
    int sfx = 0, sfy = 0, dfx = 0, dfy = 0;
    if constexpr (SO == kOrderXY) flat_origin(t, src, sfx, sfy);
    if constexpr (DO == kOrderXY) flat_origin(t, dst, dfx, dfy);
    const uint32_t sbase = natural_base(t, src, sfx, sfy);
    const uint32_t dbase = natural_base(t, dst, dfx, dfy);
    for (int p = threadIdx.x; p < ss; p += kRemapThreads) {
        int lx, ly;
        if constexpr (SO == kOrderRing) {
            side_coords(t, src, sfx, sfy, p, lx, ly);
            ring_tab[p] = side_offset(t, src, lx, ly);
        }
        side_coords(t, dst, dfx, dfy, p, lx, ly);
        if constexpr (DO == kOrderRing) ring_tab[p] = side_offset(t, dst, lx, ly);
        sslot[p] = (uint16_t)remap_swz<V>(side_pos(t, src, sfx, sfy, lx, ly));
    }
    __syncthreads();

    const int b0 = blockIdx.y * maps_per_cta;
    const int b1 = min(nmaps, b0 + maps_per_cta);
    auto issue = [&](int b) {  // map b -> stage (b - b0) % kRemapStages
        E* tl = reinterpret_cast<E*>(remap_smem + ((b - b0) % kRemapStages) * tb);
        const E* ib = in + (int64_t)b * npix;
        if constexpr (SO == kOrderRing) {
            for (int p = threadIdx.x; p < ss; p += kRemapThreads)
                cp_async_elem<sizeof(E)>(tl + remap_swz<V>(p), ib + ring_tab[p]);
        } else if (vec) {
            for (int p = threadIdx.x * V; p < ss; p += kRemapThreads * V)
                cp_async16(tl + remap_swz<V>(p), ib + nat_offset<SO>(sbase, p, logs, nside));
        } else {
            for (int p = threadIdx.x; p < ss; p += kRemapThreads)
                cp_async_elem<sizeof(E)>(tl + remap_swz<V>(p), ib + nat_offset<SO>(sbase, p, logs, nside));
        }
    };
#pragma unroll
    for (int k = 0; k < kRemapStages - 1; ++k) {
        if (b0 + k < b1) issue(b0 + k);
        cp_async_commit();
    }
    for (int b = b0; b < b1; ++b) {
        // groups committed so far: maps b0 .. b+kRemapStages-2; all but the
        // newest kRemapStages-2 are complete, so map b is in shared memory
        cp_async_wait<kRemapStages - 2>();
        __syncthreads();  // every thread's copies of map b landed; stage of map b-1 is free
        if (b + kRemapStages - 1 < b1) issue(b + kRemapStages - 1);
        cp_async_commit();
        const E* tl = reinterpret_cast<const E*>(remap_smem + ((b - b0) % kRemapStages) * tb);
        E* ob = out + (int64_t)b * npix;
        if constexpr (DO == kOrderRing) {
            for (int p = threadIdx.x; p < ss; p += kRemapThreads) ob[ring_tab[p]] = tl[sslot[p]];
        } else if (vec) {
            for (int p = threadIdx.x * V; p < ss; p += kRemapThreads * V) {
                union {
                    E e[V];
                    uint4 w;
                } u;
#pragma unroll
                for (int i = 0; i < V; ++i) u.e[i] = tl[sslot[p + i]];
                *reinterpret_cast<uint4*>(ob + nat_offset<DO>(dbase, p, logs, nside)) = u.w;
            }
        } else {
            for (int p = threadIdx.x; p < ss; p += kRemapThreads)
                ob[nat_offset<DO>(dbase, p, logs, nside)] = tl[sslot[p]];
        }
    }
    cp_async_wait<0>();
}

}  // namespace hpx
