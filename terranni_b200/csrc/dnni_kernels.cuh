// dnni_kernels.cuh -- sm_100a kernels of the discrete natural-neighbour
// interpolation hot path, for a batch of work packages ("tiles") at once.
//
// Replaces, per work package:
//   nni.cpp:722-790 renderInputPoints / nni.cpp:171-230 drawPlane (the GL
//     depth-tested site planes that leave each pixel's nearest site in the
//     colour buffer)                       -> k_bin_* + k_near_dense/far
//   nni.cpp:794-820 performNNIQueries / nni.cpp:483-534 makeBlocks and
//     cuda_nni.cu:407-488 calcNNI (query planes OR-blended into bit masks,
//     then per-pixel int32 atomics)        -> k_scatter_window + k_rows_final stencil
//   cuda_nni.cu:491-503 divide, cuda_nni.cu:399-402 zeroValues
//                                          -> k_rows_final
//
// Every kernel covers all tiles of a batch in one launch: its blocks (or
// warps, or threads) are numbered across the tiles and an exclusive prefix
// array per kind of work (point chunks, scan blocks, raster tiles, ...) maps
// a block back to its tile.  A single work package is a batch of one.
// Nothing here waits on the host, so a batch's whole launch sequence can be
// captured in one CUDA graph.
//
// Data layout in HBM (per tile, at the offsets in TileParams):
//   sorted points  int4 {x-ox, y-oy, z, gid}, grouped by search bin;
//   bin starts     int32 [nbins+1], bins ordered superblock (64x64 bins) ->
//                  block (8x8 bins) -> bin, so any bin, block or superblock is
//                  one contiguous point range;
//   occupancy      one 64-bit mask per block (its bins) and per superblock
//                  (its blocks); a nearest non-empty block per block;
//   pixel records  int2 {z of nearest site, R2 = floor(d^2/cell^2)} per
//                  raster pixel (R2 = -1: no site);
//   span words     one 64-bit word per grid cell holding (Zrel << K) + C, or
//                  int64 Z plus int32 C when the packed form cannot hold the
//                  largest possible per-cell sums.
#pragma once

#include <cuda_pipeline_primitives.h>

#include "dnni_search.cuh"

namespace dnni {

constexpr int kChunk = 2048;     // points per block in the point passes
constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;   // counts per scan block

// Prefix arrays of one batch (each of length ntiles + 1, first entry 0).
struct BatchTables {
    const TileParams* tiles;
    int ntiles;
    const int* chunk_base;       // point chunks of kChunk points
    const int* scan_base;        // scan blocks of kScanTile counts (and block-sum slots)
    const int64_t* blk_base;     // blocks (== TileParams::blk_off)
    const int64_t* sup_base;     // superblocks (== TileParams::sup_off)
    const int* row1_base;        // rows of the block grid
    const int* rt_base;          // 32 x kTileY raster tiles
    const int* ct_base;          // 32 x 16 cell tiles
    const int* grow_base;        // grid rows
    const int* band_base;        // bands of 16 grid rows
};

struct BatchCounters {
    int nfar;                    // far worklist slots used
    int err;                     // kErrRange when a point was out of range
    int far_next;                // next far group to hand out
    int pad;
};

template <typename B>
__device__ __forceinline__ int find_tile(const B* __restrict__ base, int ntiles, long long k) {
    int lo = 0, hi = ntiles - 1;   // last tile with base[t] <= k
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((long long)__ldg(&base[mid]) <= k) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// point passes
// ---------------------------------------------------------------------------

__global__ void k_init_scalars(BatchTables bt, Scalars* sc, BatchCounters* ctr) {
    const int t = blockIdx.x, l = threadIdx.x;
    Scalars* s = sc + t;
    if (l == 0) {
        s->bbox[0] = INT_MAX; s->bbox[1] = INT_MIN;
        s->bbox[2] = INT_MAX; s->bbox[3] = INT_MIN;
        s->bbox[4] = INT_MAX; s->bbox[5] = INT_MIN;
        s->err = 0; s->packed = 0; s->kbits = 0; s->zbase = 0;
        if (t == 0) { ctr->nfar = 0; ctr->err = 0; ctr->far_next = 0; }
    }
    if (l < kStatSlots) {
        s->max_r2[l] = -1; s->big_pixels[l] = 0; s->spans[l] = 0; s->nodata[l] = 0;
        s->evals_dense[l] = 0; s->evals_far[l] = 0;
    }
    if (l < kSpanHistBuckets) s->span_hist[l] = 0;
}

// Bounding box of each tile's points relative to its origin, with range checks
// (the coordinate range, and the declared extent where the caller gave one):
// bbox_point per point, bbox_flush once per warp.
struct BBoxAcc {
    int mnx = INT_MAX, mxx = INT_MIN, mny = INT_MAX, mxy = INT_MIN, mnz = INT_MAX, mxz = INT_MIN;
    unsigned bad = 0;
};

__device__ __forceinline__ void bbox_point(const TileParams& T, int xr, int yr, int zr, BBoxAcc& acc) {
    const long long x = (long long)xr - T.ox, y = (long long)yr - T.oy, z = zr;
    if (x <= -kCoordLimit || x >= kCoordLimit || y <= -kCoordLimit || y >= kCoordLimit || z <= -kCoordLimit ||
        z >= kCoordLimit || (T.has_ext && (x < T.ex0 || x > T.ex1 || y < T.ey0 || y > T.ey1))) {
        acc.bad = 1;
        return;
    }
    acc.mnx = min(acc.mnx, (int)x); acc.mxx = max(acc.mxx, (int)x);
    acc.mny = min(acc.mny, (int)y); acc.mxy = max(acc.mxy, (int)y);
    acc.mnz = min(acc.mnz, (int)z); acc.mxz = max(acc.mxz, (int)z);
}

__device__ __forceinline__ void bbox_flush(BBoxAcc& acc, Scalars* s, BatchCounters* ctr) {
    acc.mnx = __reduce_min_sync(0xffffffffu, acc.mnx); acc.mxx = __reduce_max_sync(0xffffffffu, acc.mxx);
    acc.mny = __reduce_min_sync(0xffffffffu, acc.mny); acc.mxy = __reduce_max_sync(0xffffffffu, acc.mxy);
    acc.mnz = __reduce_min_sync(0xffffffffu, acc.mnz); acc.mxz = __reduce_max_sync(0xffffffffu, acc.mxz);
    acc.bad = __reduce_or_sync(0xffffffffu, acc.bad);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&s->bbox[0], acc.mnx); atomicMax(&s->bbox[1], acc.mxx);
        atomicMin(&s->bbox[2], acc.mny); atomicMax(&s->bbox[3], acc.mxy);
        atomicMin(&s->bbox[4], acc.mnz); atomicMax(&s->bbox[5], acc.mxz);
        if (acc.bad) { atomicOr(&s->err, kErrRange); atomicOr(&ctr->err, kErrRange); }
    }
}

__global__ void __launch_bounds__(256) k_bbox(BatchTables bt, const int32_t* __restrict__ xyz, Scalars* sc,
                                              BatchCounters* ctr) {
    const int t = find_tile(bt.chunk_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int64_t c0 = (int64_t)(blockIdx.x - __ldg(&bt.chunk_base[t])) * kChunk;
    const int64_t c1 = c0 + kChunk < T.npts ? c0 + kChunk : T.npts;
    const int32_t* p = xyz + 3 * T.pt_off;
    BBoxAcc acc;
    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) bbox_point(T, p[3 * i], p[3 * i + 1], p[3 * i + 2], acc);
    bbox_flush(acc, sc + t, ctr);
}

// A tile's points outside its bin grid (possible only when the caller's
// declared point extent was wrong) are counted as a range error and binned
// at the grid's edge, so that no access leaves the tile's arrays.
__device__ __forceinline__ int64_t point_bin_checked(const BinGrid& g, int xr, int yr, unsigned& bad) {
    const long long ux = (long long)xr - g.gx0, uy = (long long)yr - g.gy0;
    if (ux < 0 || uy < 0 || ux >= (long long)g.nbx * g.bs || uy >= (long long)g.nby * g.bs) bad = 1;
    int bx = ux < 0 ? 0 : (ux >= (1LL << 32) ? g.nbx - 1 : udiv32(ux, g.bs));
    int by = uy < 0 ? 0 : (uy >= (1LL << 32) ? g.nby - 1 : udiv32(uy, g.bs));
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    return bin_id(g, bx, by);
}

// Counting-sort pass 1: per-bin counts, with reductions whose result is not
// returned (no round trip per point).  with_bbox: also the bounding box and
// range checks of k_bbox (batches, whose bin grids are planned before any
// point is seen, skip k_bbox).
__global__ void __launch_bounds__(256) k_bin_count(BatchTables bt, const int32_t* __restrict__ xyz,
                                                   int* __restrict__ cnt, Scalars* sc, BatchCounters* ctr,
                                                   int with_bbox) {
    const int t = find_tile(bt.chunk_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int64_t c0 = (int64_t)(blockIdx.x - __ldg(&bt.chunk_base[t])) * kChunk;
    const int64_t c1 = c0 + kChunk < T.npts ? c0 + kChunk : T.npts;
    const int32_t* p = xyz + 3 * T.pt_off;
    int* c = cnt + T.bin_off;
    unsigned bad = 0;
    BBoxAcc acc;
    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
        const int xr = p[3 * i], yr = p[3 * i + 1];
        if (with_bbox) bbox_point(T, xr, yr, p[3 * i + 2], acc);
        const int64_t id = point_bin_checked(T.bg, rel_coord(xr, T.ox), rel_coord(yr, T.oy), bad);
        atomicAdd(&c[id], 1);
    }
    if (with_bbox) bbox_flush(acc, sc + t, ctr);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&ctr->err, kErrRange);
}

// Counting-sort pass 3: each point takes a slot of its bin by counting the
// bin's count down (cnt ends at zero), at start[bin] + the count taken - 1.
// The order of the points inside a bin is therefore arbitrary, which no
// result depends on: every comparison of sites orders them by (distance,
// gid, z), never by position.
__global__ void __launch_bounds__(256) k_bin_scatter(BatchTables bt, const int32_t* __restrict__ xyz,
                                                     const uint32_t* __restrict__ gid, const int* __restrict__ start,
                                                     int* __restrict__ cnt, int4* __restrict__ sorted) {
    const int t = find_tile(bt.chunk_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int64_t c0 = (int64_t)(blockIdx.x - __ldg(&bt.chunk_base[t])) * kChunk;
    const int64_t c1 = c0 + kChunk < T.npts ? c0 + kChunk : T.npts;
    const int32_t* p = xyz + 3 * T.pt_off;
    const int* st = start + T.bin_off;
    int* c = cnt + T.bin_off;
    int4* out = sorted + T.srt_off;
    unsigned bad = 0;
    for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) {
        const int xr = rel_coord(p[3 * i], T.ox), yr = rel_coord(p[3 * i + 1], T.oy);
        const int64_t id = point_bin_checked(T.bg, xr, yr, bad);
        const int pos = st[id] + atomicSub(&c[id], 1) - 1;
        const uint32_t g = gid ? gid[T.pt_off + i] : (uint32_t)i;
        out[pos] = make_int4(xr, yr, p[3 * i + 2], (int)g);
    }
}

// ---- exclusive scan of each tile's bin counts (three passes, 4096 per block) ----

template <typename V>
__device__ __forceinline__ V block_exclusive_sum(V v, V* wsum, V& total, int tid) {
    // 256 threads (8 warps); tid is the linear thread index in the block
    const int lane = tid & 31, warp = tid >> 5;
    V x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        V y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        V w = lane < 8 ? wsum[lane] : V(0);
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            V y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) wsum[lane] = w;
    }
    __syncthreads();
    total = wsum[7];
    const V excl = x - v + (warp ? wsum[warp - 1] : V(0));
    __syncthreads();
    return excl;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_partial(BatchTables bt, const int* __restrict__ cnt,
                                                               int* __restrict__ bsum) {
    __shared__ int wsum[8];
    const int t = find_tile(bt.scan_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int64_t m = T.bg.nbins + 1;
    const int64_t base = (int64_t)(blockIdx.x - __ldg(&bt.scan_base[t])) * kScanTile;
    const int* c = cnt + T.bin_off;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t idx = base + k * kScanThreads + threadIdx.x;
        if (idx < m) s += c[idx];
    }
    int total;
    block_exclusive_sum(s, wsum, total, (int)threadIdx.x);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// One block per tile: exclusive scan of the tile's block sums, in place.
__global__ void __launch_bounds__(1024) k_scan_bsum(BatchTables bt, int* __restrict__ bsum) {
    __shared__ int wsum[32];
    const int t = blockIdx.x;
    const int b0g = __ldg(&bt.scan_base[t]), nb = __ldg(&bt.scan_base[t + 1]) - b0g;
    int* bs = bsum + b0g;
    const int per = (nb + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    int s = 0;
    for (int k = 0; k < per; ++k) if (b0 + k < nb) s += bs[b0 + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = s;
    for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) { int y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
        wsum[lane] = w;
    }
    __syncthreads();
    int run = x - s + (warp ? wsum[warp - 1] : 0);
    for (int k = 0; k < per; ++k)
        if (b0 + k < nb) { const int v = bs[b0 + k]; bs[b0 + k] = run; run += v; }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_final(BatchTables bt, const int* __restrict__ cnt,
                                                             const int* __restrict__ bsum, int* __restrict__ start) {
    __shared__ int tile[kScanTile];
    __shared__ int wsum[8];
    const int t = find_tile(bt.scan_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int64_t m = T.bg.nbins + 1;
    const int64_t base = (int64_t)(blockIdx.x - __ldg(&bt.scan_base[t])) * kScanTile;
    const int* c = cnt + T.bin_off;
    int* st = start + T.bin_off;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int li = k * kScanThreads + threadIdx.x;
        const int64_t idx = base + li;
        tile[li] = idx < m ? c[idx] : 0;
    }
    __syncthreads();
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) { v[k] = tile[threadIdx.x * kScanItems + k]; s += v[k]; }
    int total;
    int run = block_exclusive_sum(s, wsum, total, (int)threadIdx.x) + bsum[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) { tile[threadIdx.x * kScanItems + k] = run; run += v[k]; }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int li = k * kScanThreads + threadIdx.x;
        const int64_t idx = base + li;
        if (idx < m) st[idx] = tile[li];
    }
}

// ---------------------------------------------------------------------------
// occupancy masks and the nearest non-empty block map
// ---------------------------------------------------------------------------

// One warp per block (bit l = bin l of the block is non-empty).
__global__ void __launch_bounds__(256) k_block_masks(BatchTables bt, const int* __restrict__ start,
                                                     uint64_t* __restrict__ bmask) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= __ldg(&bt.blk_base[bt.ntiles])) return;
    const int t = find_tile(bt.blk_base, bt.ntiles, w);
    const TileParams& T = bt.tiles[t];
    const int64_t k = w - T.blk_off;
    const int* s = start + T.bin_off + (k << 6);
    const bool lo = s[lane + 1] != s[lane];
    const bool hi = s[lane + 33] != s[lane + 32];
    const unsigned mlo = __ballot_sync(0xffffffffu, lo), mhi = __ballot_sync(0xffffffffu, hi);
    if (lane == 0) bmask[w] = (uint64_t)mlo | ((uint64_t)mhi << 32);
}

// One warp per superblock (bit m = block m of the superblock is non-empty).
__global__ void __launch_bounds__(256) k_super_masks(BatchTables bt, const uint64_t* __restrict__ bmask,
                                                     uint64_t* __restrict__ smask) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= __ldg(&bt.sup_base[bt.ntiles])) return;
    const int t = find_tile(bt.sup_base, bt.ntiles, w);
    const TileParams& T = bt.tiles[t];
    const uint64_t* b = bmask + T.blk_off + ((w - T.sup_off) << 6);
    const unsigned mlo = __ballot_sync(0xffffffffu, b[lane] != 0), mhi = __ballot_sync(0xffffffffu, b[lane + 32] != 0);
    if (lane == 0) smask[w] = (uint64_t)mlo | ((uint64_t)mhi << 32);
}

// Nearest non-empty block map, exact in block-centre distance: per block
// row the nearest non-empty column (forward and backward sweep), then per
// block the best row found by walking rows outward until the row offset
// alone exceeds the best distance.  near = bmask index of the chosen block
// within the tile, -1 when the tile has no points.
__global__ void k_block_rows(BatchTables bt, const uint64_t* __restrict__ bmask, int* __restrict__ rownear) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= __ldg(&bt.row1_base[bt.ntiles])) return;
    const int t = find_tile(bt.row1_base, bt.ntiles, r);
    const TileParams& T = bt.tiles[t];
    const BinGrid g = T.bg;
    const int n1x = g.nbx >> 3;
    const int cy = r - __ldg(&bt.row1_base[t]);
    const uint64_t* bm = bmask + T.blk_off;
    int* row = rownear + T.blk_off + (int64_t)cy * n1x;
    int last = -1;
    for (int cx = 0; cx < n1x; ++cx) {
        if (bm[block_index(g, cx, cy)]) last = cx;
        row[cx] = last;
    }
    last = -1;
    for (int cx = n1x - 1; cx >= 0; --cx) {
        if (bm[block_index(g, cx, cy)]) last = cx;
        const int l = row[cx];
        if (last >= 0 && (l < 0 || last - cx < cx - l)) row[cx] = last;
    }
}

__global__ void k_block_near(BatchTables bt, const int* __restrict__ rownear, int64_t* __restrict__ near) {
    const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (w >= __ldg(&bt.blk_base[bt.ntiles])) return;
    const int t = find_tile(bt.blk_base, bt.ntiles, w);
    const TileParams& T = bt.tiles[t];
    if (T.npts == 0) {   // no row sweep ran for a tile without points
        near[w] = -1;
        return;
    }
    const int n1x = T.bg.nbx >> 3, n1y = T.bg.nby >> 3;
    const int64_t k = w - T.blk_off;
    const int cx = (int)(k % n1x), cy = (int)(k / n1x);
    const int* rn = rownear + T.blk_off;
    long long best = LLONG_MAX;
    int bxn = -1, byn = -1;
    for (int d = 0; d < n1y; ++d) {
        if ((long long)d * d > best) break;
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            if (d == 0 && sgn > 0) continue;
            const int y = cy + sgn * d;
            if (y < 0 || y >= n1y) continue;
            const int x = rn[(int64_t)y * n1x + cx];
            if (x < 0) continue;
            const long long v = (long long)(x - cx) * (x - cx) + (long long)d * d;
            if (v < best) { best = v; bxn = x; byn = y; }
        }
    }
    near[w] = bxn >= 0 ? block_index(T.bg, bxn, byn) : -1;
}

// ---------------------------------------------------------------------------
// nearest site per raster pixel
// ---------------------------------------------------------------------------

// Records a settled pixel: its record and (optionally) its site; returns
// its R2.
__device__ __forceinline__ int settle_pixel(const TileParams& T, int i, int j, const Best& b, int2* __restrict__ pix,
                                            uint32_t* __restrict__ site) {
    const int R2 = r2_of(b.d2, (long long)T.cs * T.cs, T.r2cap);
    const int64_t o = (int64_t)j * T.rw + i;
    pix[T.pix_off + o] = make_int2(b.z, R2);
    if (site && T.site_off >= 0) site[T.site_off + o] = b.gid;
    return R2;
}

// Statistics of settled pixels, accumulated per thread and flushed once per
// warp: span-path pixels and their spans, the largest R2, and the candidate
// distance evaluations made (counted into evals_dense or evals_far).
struct StatAcc {
    unsigned big = 0, spans = 0, nev = 0;
    int mx = -1;
    __device__ __forceinline__ void add(const TileParams& T, int R2, int n) {
        if (R2 > T.rs * T.rs) {
            big += 1u;
            spans += 2u * (unsigned)isqrt_i32(R2) + 1u;
        }
        mx = R2 > mx ? R2 : mx;
        nev += (unsigned)n;
    }
    __device__ __forceinline__ void flush(Scalars* __restrict__ s, int slot, bool far_pass) {
        const unsigned nbig = __reduce_add_sync(0xffffffffu, big);
        const unsigned nsp = __reduce_add_sync(0xffffffffu, spans);
        const unsigned nv = __reduce_add_sync(0xffffffffu, nev);
        const int m = __reduce_max_sync(0xffffffffu, mx);
        if ((threadIdx.x & 31) == 0) {
            slot &= kStatSlots - 1;
            if (nbig) {
                atomicAdd(&s->big_pixels[slot], (unsigned long long)nbig);
                atomicAdd(&s->spans[slot], (unsigned long long)nsp);
            }
            if (nv) atomicAdd(far_pass ? &s->evals_far[slot] : &s->evals_dense[slot], (unsigned long long)nv);
            if (m >= 0) atomicMax(&s->max_r2[slot], m);
        }
    }
};

// Far worklist slot: tile, raster pixel index within the tile (-1 = empty
// slot), sorted-array position of the best site so far (-1 = none).
struct FarSlot {
    int tile, pix, idx, pad;
};

// R2 of a pixel record that the ring search left unsettled (the far pass
// overwrites it); real records hold R2 >= -1.
constexpr int kPixFar = -2;
constexpr int kFarBlocksDefault = 1;   // far groups of 8 x 4 pixels

// Dense pass.  One CTA per 32 x kTileY raster tile of a work package
// (blockDim 32 x 8; warp w takes pixel rows w, w + 8, ... of the tile): the
// tile's bin window (bin rings
// of every pixel) is staged in shared memory and the rings are searched
// there; windows too large for shared memory use the global arrays.  A warp
// with pixels the rings do not settle appends its whole row as one group of
// 32 slots to the far worklist.  With no points every pixel is settled as
// "no site".
__global__ void __launch_bounds__(256, 4) k_near_dense(BatchTables bt, const int4* __restrict__ pts_all,
                                                       const int* __restrict__ start_all, int2* __restrict__ pix,
                                                       uint32_t* __restrict__ site, FarSlot* __restrict__ far,
                                                       Scalars* __restrict__ sc, BatchCounters* __restrict__ ctr,
                                                       int far_blocks, int band0) {
    extern __shared__ int4 smem[];
    int4* s_pts = smem;
    int* s_lstart = (int*)(smem + kWinMaxPts);
    int* s_gstart = s_lstart + kWinMaxBins + 1;
    __shared__ int s_rowbase[kWinMaxRows];
    __shared__ int s_total;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int t = find_tile(bt.rt_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const BinGrid g = T.bg;
    const int4* pts = pts_all + T.srt_off;
    const int* start = start_all + T.bin_off;
    const int lt = blockIdx.x - __ldg(&bt.rt_base[t]);
    const int ntx = (T.rw + kTileX - 1) / kTileX;
    const int i0 = (lt % ntx) * kTileX, j0 = (lt / ntx) * kTileY;
    const int i = i0 + threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    // the tile's rows go in bands, each with its own staged window: band0
    // rows (8, 16, 32 or 64: the shape of the pixel block that shares one
    // window, a tuning choice) when that window fits shared memory, else
    // halves, down to 8 rows
    StatAcc acc;
    int band = band0;
    for (int jb = 0; jb < kTileY && j0 + jb < T.rh; jb += band) {
    int wx0 = 0, wy0 = 0, wnx = 0, wny = 0;
    bool staged = false;
    while (T.npts > 0) {
        tile_window(T, i0, j0 + jb, band, wx0, wy0, wnx, wny);
        const int nwb = wnx * wny;
        if (nwb > kWinMaxBins || wny > kWinMaxRows) {
            if (band > 8) { band >>= 1; continue; }
            break;
        }
        {
            // each window bin's global start and end, copied asynchronously
            // (all of a band's copies in flight at once; a thread later reads
            // only the entries it copied itself): warp w takes window rows w,
            // w+8, ...; lanes take columns
            for (int r = warp; r < wny; r += 8)
                for (int c = lane; c < wnx; c += 32) {
                    const int64_t id = bin_id(g, wx0 + c, wy0 + r);
                    __pipeline_memcpy_async(&s_gstart[r * wnx + c], &start[id], sizeof(int));
                    __pipeline_memcpy_async(&s_lstart[r * wnx + c], &start[id + 1], sizeof(int));
                }
            __pipeline_commit();
            __pipeline_wait_prior(0);
            // per-bin counts -> local starts, with a warp scan along the row
            for (int r = warp; r < wny; r += 8) {
                int rowsum = 0;
                for (int c0 = 0; c0 < wnx; c0 += 32) {
                    const int c = c0 + lane;
                    int cnt = 0;
                    if (c < wnx) cnt = s_lstart[r * wnx + c] - s_gstart[r * wnx + c];
                    int x = cnt;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (c < wnx) s_lstart[r * wnx + c] = rowsum + x - cnt;
                    rowsum += __shfl_sync(0xffffffffu, x, 31);
                }
                if (lane == 0) s_rowbase[r] = rowsum;
            }
            __syncthreads();
            if (warp == 0) {
                int run = 0;
                for (int r0 = 0; r0 < wny; r0 += 32) {
                    const int r = r0 + lane;
                    const int v = r < wny ? s_rowbase[r] : 0;
                    int x = v;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (r < wny) s_rowbase[r] = run + x - v;
                    run += __shfl_sync(0xffffffffu, x, 31);
                }
                if (lane == 0) { s_lstart[nwb] = run; s_total = run; }
            }
            __syncthreads();
            for (int r = warp; r < wny; r += 8)
                for (int c = lane; c < wnx; c += 32) s_lstart[r * wnx + c] += s_rowbase[r];
            __syncthreads();
            if (s_total > kWinMaxPts && band > 8) {   // too many points: a shorter band
                band >>= 1;
                __syncthreads();
                continue;
            }
            staged = s_total <= kWinMaxPts;
            if (staged) {
                // copy the window's points run by run (asynchronous 16-byte
                // copies, all in flight before one wait): the bins of one
                // window row inside one block are consecutive in both layouts;
                // one warp per run, lanes striding over its points
                const int cb0 = wx0 >> 3, cb1 = (wx0 + wnx - 1) >> 3;
                const int nseg = cb1 - cb0 + 1, nrun = nseg * wny;
                for (int run = warp; run < nrun; run += 8) {
                    const int r = run / nseg, sg = run - r * nseg;
                    const int xa = (cb0 + sg) * 8 > wx0 ? (cb0 + sg) * 8 : wx0;
                    const int xb = (cb0 + sg) * 8 + 7 < wx0 + wnx - 1 ? (cb0 + sg) * 8 + 7 : wx0 + wnx - 1;
                    const int lk0 = r * wnx + (xa - wx0), lk1 = r * wnx + (xb - wx0);
                    const int l0 = s_lstart[lk0], cntp = s_lstart[lk1 + 1] - l0, g0 = s_gstart[lk0];
                    for (int q = lane; q < cntp; q += 32) __pipeline_memcpy_async(&s_pts[l0 + q], &pts[g0 + q], sizeof(int4));
                }
                __pipeline_commit();
                __pipeline_wait_prior(0);
            }
            __syncthreads();
        }
        break;
    }
#pragma unroll 1
    for (int sub = 0; sub < band / 8; ++sub) {
    const int j = j0 + jb + threadIdx.y + 8 * sub;
    const bool valid = i < T.rw && j < T.rh;
    int R2 = -1;
    bool far_pixel = false;
    Best b{LLONG_MAX, 0xFFFFFFFFu, INT_MAX, -1, 0};
    if (valid) {
        if (T.npts > 0) {
            const int px = (T.rx0 + i) * T.cs, py = (T.ry0 + j) * T.cs;
            bool done;
            if (staged) {
                const BinWindow w{wx0, wy0, wnx, wny, s_lstart, s_gstart, s_pts};
                done = window_fits32(g, w) ? search_window_fast32(g, w, px, py, b) : search_window_fast(g, w, px, py, b);
                if (!done) b.idx = window_global_index(w, b.idx);
            } else {
                done = search_bins(g, pts, start, px, py, b);
            }
            if (done) {
                R2 = settle_pixel(T, i, j, b, pix, site);
            } else {
                far_pixel = true;
            }
        } else {
            const int64_t o = (int64_t)j * T.rw + i;
            pix[T.pix_off + o] = make_int2(0, -1);
            if (site && T.site_off >= 0) site[T.site_off + o] = 0xFFFFFFFFu;
        }
    }
    if (far_blocks) {
        // marked for the block pass below: the record holds the best site
        // found so far (-1: none) and kPixFar
        if (far_pixel) pix[T.pix_off + (int64_t)j * T.rw + i] = make_int2(b.idx, kPixFar);
    } else {
        // worklist: a warp with any unsettled pixel appends its whole row of
        // 32 slots as one group (settled or absent pixels as empty slots), so
        // that a far warp later takes 32 neighbouring pixels of one tile
        const unsigned mfar = __ballot_sync(0xffffffffu, far_pixel);
        if (mfar) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&ctr->nfar, 32);
            base = __shfl_sync(0xffffffffu, base, 0);
            far[base + lane] = far_pixel ? FarSlot{t, j * T.rw + i, b.idx, 0} : FarSlot{t, -1, -1, 0};
        }
    }
    acc.add(T, R2, b.nev);
    }
    __syncthreads();     // the next band restages the window
    }
    acc.flush(sc + t, blockIdx.x + threadIdx.y, false);
    if (far_blocks) {
        // worklist in 8 x 4 pixel blocks: a block with any unsettled pixel
        // appends its 32 pixels as one group (lane = 8 * row + column), so
        // that a far warp takes a compact patch whose discs overlap most;
        // the records written above are visible after the barrier
        __syncthreads();
        for (int blk = warp; blk < (kTileX / 8) * (kTileY / 4); blk += 8) {
            const int ii = i0 + (blk % (kTileX / 8)) * 8 + (lane & 7);
            const int jj = j0 + (blk / (kTileX / 8)) * 4 + (lane >> 3);
            bool fp = false;
            int idx = -1;
            if (ii < T.rw && jj < T.rh) {
                const int2 r = pix[T.pix_off + (int64_t)jj * T.rw + ii];
                fp = r.y == kPixFar;
                idx = r.x;
            }
            if (__ballot_sync(0xffffffffu, fp)) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&ctr->nfar, 32);
                base = __shfl_sync(0xffffffffu, base, 0);
                far[base + lane] = fp ? FarSlot{t, jj * T.rw + ii, idx, 0} : FarSlot{t, -1, -1, 0};
            }
        }
    }
}

__device__ __forceinline__ long long warp_min64(long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) { const long long w = __shfl_xor_sync(0xffffffffu, v, o); v = w < v ? w : v; }
    return v;
}
__device__ __forceinline__ long long warp_max64(long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) { const long long w = __shfl_xor_sync(0xffffffffu, v, o); v = w > v ? w : v; }
    return v;
}

__device__ __forceinline__ uint64_t warp_or64(uint64_t v) {
    const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)v), hi = __reduce_or_sync(0xffffffffu, (unsigned)(v >> 32));
    return ((uint64_t)hi << 32) | lo;
}

// 8 x 8 cell mask of the cells [a0,a1] x [b0,b1] (x = bit & 7, y = bit >> 3);
// 0 when the range is empty.
__device__ __forceinline__ uint64_t box_mask8(int a0, int a1, int b0, int b1) {
    a0 = a0 < 0 ? 0 : a0;
    b0 = b0 < 0 ? 0 : b0;
    a1 = a1 > 7 ? 7 : a1;
    b1 = b1 > 7 ? 7 : b1;
    if (a0 > a1 || b0 > b1) return 0;
    const uint64_t row = (uint64_t)((0xFFu << a0) & (0xFFu >> (7 - a1)) & 0xFFu);
    uint64_t m = 0;
    for (int y = b0; y <= b1; ++y) m |= row << (8 * y);
    return m;
}

// Cells (u wide, 8 per side, origin o) that the box [c - r, c + r] may touch,
// widened by one cell on each side so float rounding can only add cells.
__device__ __forceinline__ void cell_span8(long long c, long long r, long long o, float inv_u, int& lo, int& hi) {
    const float a = (float)(c - r - o) * inv_u, b = (float)(c + r - o) * inv_u;
    lo = a < -2.0f ? -2 : (a > 9.0f ? 9 : (int)floorf(a)) - 1;
    hi = b < -2.0f ? -2 : (b > 9.0f ? 9 : (int)floorf(b)) + 1;
}

// Squared box bound in 32-bit arithmetic, for gaps below 46341 (larger
// gaps are clamped there, which still exceeds any bound below 2^31).
__device__ __forceinline__ unsigned box_lb32(int rx, int ry, int x0, int x1, int y0, int y1) {
    int dx = rx < x0 ? x0 - rx : (rx > x1 ? rx - x1 : 0);
    int dy = ry < y0 ? y0 - ry : (ry > y1 ? ry - y1 : 0);
    dx = dx < 46340 ? dx : 46340;
    dy = dy < 46340 ? dy : 46340;
    return (unsigned)(dx * dx) + (unsigned)(dy * dy);
}

// 8 x 8 mask of the cells (u wide, origin (X0, Y0)) that the union of the
// active lanes' discs may touch, row by row: in cell row r the lanes' disc
// chords, widened by one unit, are merged into their hull across the warp.
// A superset of the cells within some lane's bound, so the search stays
// exact; the lanes of a group are neighbouring pixels of one row, whose
// chords overlap, so the hull adds little.  Warp-uniform result.
__device__ __forceinline__ uint64_t chord_mask8(bool act, long long px, long long py, long long d2, long long X0,
                                                long long Y0, long long u, bool small) {
    uint64_t m = 0;
#pragma unroll 1
    for (int r = 0; r < 8; ++r) {
        int a = 8, e = -1;
        if (act) {
            const long long gy = axis_gap(py, Y0 + r * u, Y0 + (r + 1) * u - 1);
            if (gy * gy <= d2) {
                const long long v = d2 - gy * gy;
                const long long w = (small ? (long long)sqrtf((float)v) : (long long)sqrt((double)v)) + 1;
                const long long lo = px - w - X0, hi = px + w - X0;
                if (hi >= 0 && lo < 8 * u) {
                    a = lo <= 0 ? 0 : udiv32(lo, u);
                    e = hi >= 8 * u ? 7 : udiv32(hi, u);
                }
            }
        }
        a = __reduce_min_sync(0xffffffffu, a);
        e = __reduce_max_sync(0xffffffffu, e);
        if (a <= e) m |= (uint64_t)((0xFFu >> (7 - e)) & (0xFFu << a) & 0xFFu) << (8 * r);
    }
    return m;
}

// chord_mask8 for a warp whose every active lane has a bound below 2^31 (a
// real site found), in 32-bit arithmetic relative to the mask's origin: rx,
// ry = pixel - origin (|rx|, |ry| < 2^30), u = cell width (8u <= 2^30).  The
// row gap beyond 46340 units already exceeds any such bound.  The chord's
// cell range is the same as chord_mask8's: floor(x / u) for 0 < x < 8u from
// a float product with 1/u (within one of the quotient there), corrected
// with exact integer products.
__device__ __forceinline__ int floor_div8(int x, int u, float inv_u) {
    int q = (int)((float)x * inv_u);
    q -= q * u > x ? 1 : 0;
    q += (q + 1) * u <= x ? 1 : 0;
    return q;
}

__device__ __forceinline__ uint64_t chord_mask8_32(bool act, int rx, int ry, unsigned d2, int u, float inv_u) {
    uint64_t m = 0;
#pragma unroll 1
    for (int r = 0; r < 8; ++r) {
        int a = 8, e = -1;
        if (act) {
            const int y0 = r * u, y1 = y0 + u - 1;
            const int gy = ry < y0 ? y0 - ry : (ry > y1 ? ry - y1 : 0);
            if (gy <= 46340 && (unsigned)(gy * gy) <= d2) {
                const int w = (int)sqrt_est((float)(d2 - (unsigned)(gy * gy))) + 1;
                const int lo = rx - w, hi = rx + w;
                if (hi >= 0 && lo < 8 * u) {
                    a = lo <= 0 ? 0 : floor_div8(lo, u, inv_u);
                    e = hi >= 8 * u ? 7 : floor_div8(hi, u, inv_u);
                }
            }
        }
        a = __reduce_min_sync(0xffffffffu, a);
        e = __reduce_max_sync(0xffffffffu, e);
        if (a <= e) m |= (uint64_t)((0xFFu >> (7 - e)) & (0xFFu << a) & 0xFFu) << (8 * r);
    }
    return m;
}

// A candidate block with at most this many points is scanned whole, which
// costs less than its bin mask.
constexpr int kFarWholeBlock = 24;

// Warp-cooperative exact search for the 32 pixels of one worklist group
// (neighbouring pixels of one tile row; inactive lanes have act = false).
// The warp walks the superblocks of the union of the lanes' bound boxes
// (rows outward from the group's centre); inside a superblock the candidate
// blocks are the non-empty ones under the chord hull of the lanes' discs
// (chord_mask8), inside a candidate block the candidate bins likewise, and
// every point of a candidate bin is considered by every active lane (the
// comparison is exact, so extra candidates cost time, never correctness).
// All control flow is uniform across the warp.  Complete for each active
// lane whose b holds a real site on entry, by the same argument as
// search_disc.
__device__ void search_disc_warp(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                                 const uint64_t* __restrict__ bmask, const uint64_t* __restrict__ smask, bool act,
                                 int px, int py, Best& b) {
    const unsigned full = 0xffffffffu;
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    const long long u1 = bs * kBinsPerBlockEdge, u2 = bs * kBinsPerSuperEdge;
    const float inv_u1 = 1.0f / (float)u1, inv_bs = 1.0f / (float)bs;
    const long long reach = act ? reach_of(b.d2) : 0;
    const long long xlo = warp_min64(act ? px - reach : LLONG_MAX), xhi = warp_max64(act ? px + reach : LLONG_MIN);
    const long long ylo = warp_min64(act ? py - reach : LLONG_MAX), yhi = warp_max64(act ? py + reach : LLONG_MIN);
    if (xlo > xhi) return;   // no active lane
    int sx0, sx1, sy0, sy1;
    cell_range((xlo + xhi) / 2, (xhi - xlo) / 2 + 1, gx0, u2, g.n2x, sx0, sx1);
    cell_range((ylo + yhi) / 2, (yhi - ylo) / 2 + 1, gy0, u2, g.n2y, sy0, sy1);
    if (sx0 > sx1 || sy0 > sy1) return;
    const long long cyy = warp_min64(act ? py : LLONG_MAX);
    int csy = udiv32((cyy < gy0 ? gy0 : cyy) - gy0, u2);
    csy = csy < sy0 ? sy0 : (csy > sy1 ? sy1 : csy);
    const int span = (csy - sy0) > (sy1 - csy) ? (csy - sy0) : (sy1 - csy);
    for (int r = 0; r <= 2 * span; ++r) {
        const int sy = csy + ((r & 1) ? -((r + 1) >> 1) : (r >> 1));
        if (sy < sy0 || sy > sy1) continue;
        const long long SY0 = gy0 + (long long)sy * u2;
        for (int sx = sx0; sx <= sx1; ++sx) {
            const int sidx = sy * g.n2x + sx;
            const uint64_t sm = __ldg(&smask[sidx]);
            if (!sm) continue;
            const long long SX0 = gx0 + (long long)sx * u2;
            const bool need_s = act && box_lb(px, py, SX0, SX0 + u2 - 1, SY0, SY0 + u2 - 1) <= b.d2;
            if (!__any_sync(full, need_s)) continue;
            // 32-bit arithmetic while every bound is below 2^31 and every
            // active lane lies within 2^29 units of the superblock's origin
            // (then within 2^30 of each of its blocks' origins)
            const long long ox = px - SX0, oy = py - SY0;
            const bool near = !act || (ox > -(1LL << 29) && ox < (1LL << 29) && oy > -(1LL << 29) && oy < (1LL << 29));
            bool small = __all_sync(full, !act || (b.d2 < (1LL << 31) && near));
            uint64_t cand = sm & (small ? chord_mask8_32(act, (int)(px - SX0), (int)(py - SY0), (unsigned)b.d2,
                                                         (int)u1, inv_u1)
                                        : chord_mask8(act, px, py, b.d2, SX0, SY0, u1, false));
            while (cand) {
                const int m = ffs64(cand);
                cand &= cand - 1;
                const long long BX0 = SX0 + (long long)(m & 7) * u1, BY0 = SY0 + (long long)(m >> 3) * u1;
                const int64_t blk = ((int64_t)sidx << 6) + m;
                const int bp0 = __ldg(&start[blk << 6]), bp1 = __ldg(&start[(blk + 1) << 6]);
                if (bp1 - bp0 <= kFarWholeBlock) {
                    // few points: the block's range whole (its bins are consecutive)
                    if (act) b.nev += bp1 - bp0;
                    for (int q = bp0; q < bp1; ++q) {
                        const int4 p = __ldg(&pts[q]);
                        if (act) consider(b, p, q, px, py);
                    }
                    continue;
                }
                const uint64_t bm = __ldg(&bmask[blk]);
                small = __all_sync(full, !act || (b.d2 < (1LL << 31) && near));
                uint64_t qc = bm & (small ? chord_mask8_32(act, (int)(px - BX0), (int)(py - BY0), (unsigned)b.d2,
                                                           (int)bs, inv_bs)
                                          : chord_mask8(act, px, py, b.d2, BX0, BY0, bs, false));
                while (qc) {
                    const int l = ffs64(qc);
                    qc &= qc - 1;
                    const int64_t id = (blk << 6) + l;
                    const int s0 = __ldg(&start[id]), e0 = __ldg(&start[id + 1]);
                    if (act) b.nev += e0 - s0;
                    if (small) {
                        for (int q = s0; q < e0; ++q) {
                            const int4 p = __ldg(&pts[q]);
                            if (act) consider_below31(b, p, q, px, py);
                        }
                    } else {
                        for (int q = s0; q < e0; ++q) {
                            const int4 p = __ldg(&pts[q]);
                            if (act) consider(b, p, q, px, py);
                        }
                    }
                }
            }
        }
    }
}

// Far pass over the worklist: one warp per group of 32 slots (handed out by a counter;
// all slots of a group belong to one tile).  Each lane seeds its bound (its
// best site so far, else the nearest non-empty block's closest bin, else the
// nearest non-empty superblock) and the warp searches the union of the bound
// discs cooperatively.
__global__ void __launch_bounds__(256, 4) k_near_far(BatchTables bt, const int4* __restrict__ pts_all,
                                                     const int* __restrict__ start_all,
                                                     const uint64_t* __restrict__ bmask_all,
                                                     const uint64_t* __restrict__ smask_all,
                                                     const int64_t* __restrict__ near_all,
                                                     const FarSlot* __restrict__ far, int2* __restrict__ pix,
                                                     uint32_t* __restrict__ site, Scalars* __restrict__ sc,
                                                     BatchCounters* __restrict__ ctr) {
    const int count = ctr->nfar;
    const int lane = threadIdx.x & 31;
    // groups differ in cost by orders of magnitude (a lake's centre against
    // its shore), so each warp takes the next group from a counter instead of
    // a fixed stride
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&ctr->far_next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= count) break;
        const FarSlot item = far[base + lane];
        const int t = __shfl_sync(0xffffffffu, item.tile, 0);
        const TileParams& T = bt.tiles[t];
        const BinGrid g = T.bg;
        const int4* pts = pts_all + T.srt_off;
        const int* start = start_all + T.bin_off;
        const uint64_t* bmask = bmask_all + T.blk_off;
        const uint64_t* smask = smask_all + T.sup_off;
        const bool act = item.pix >= 0;
        int i = 0, j = 0, px = 0, py = 0;
        Best b{LLONG_MAX, 0xFFFFFFFFu, INT_MAX, -1, 0};
        if (act) {
            i = item.pix % T.rw;
            j = item.pix / T.rw;
            px = (T.rx0 + i) * T.cs;
            py = (T.ry0 + j) * T.cs;
            if (item.idx >= 0) {
                consider(b, __ldg(&pts[item.idx]), item.idx, px, py);
                b.nev += 1;
            }
            int bx = udiv32((long long)px - g.gx0, g.bs), by = udiv32((long long)py - g.gy0, g.bs);
            bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
            by = by < g.nby - 1 ? by : g.nby - 1;
            const int64_t nb = __ldg(&near_all[T.blk_off + (int64_t)(by >> 3) * (g.nbx >> 3) + (bx >> 3)]);
            if (nb >= 0) seed_from_block(g, pts, start, bmask, nb, px, py, b);
            if (b.d2 == LLONG_MAX) seed_from_superblocks(g, pts, start, bmask, smask, px, py, b);
        }
        // the seeds of the group's corner lanes are candidates for every
        // pixel of the group: a lane whose own seed came from a distant
        // block starts the disc search with a tighter bound
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int src = (k & 1 ? 7 : 0) + (k & 2 ? 24 : 0);
            const int q = __shfl_sync(0xffffffffu, b.idx, src);
            if (act && q >= 0) {
                consider(b, __ldg(&pts[q]), q, px, py);
                b.nev += 1;
            }
        }
        search_disc_warp(g, pts, start, bmask, smask, act, px, py, b);
        int R2 = -1;
        if (act) R2 = settle_pixel(T, i, j, b, pix, site);
        StatAcc acc;
        acc.add(T, R2, b.nev);
        acc.flush(sc + t, blockIdx.x * 3 + (threadIdx.x >> 5), true);
    }
}

// ---------------------------------------------------------------------------
// scatter-accumulate and finalize
// ---------------------------------------------------------------------------

// Per tile: the accumulator form of the span path (see decide_packing).
__global__ void k_decide(BatchTables bt, Scalars* sc) {
    const int t = blockIdx.x, l = threadIdx.x;
    const TileParams& T = bt.tiles[t];
    Scalars* s = sc + t;
    int mx = s->max_r2[l];
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (l == 0) {
        int packed, K;
        long long zbase;
        decide_packing(mx, (long long)T.rw * T.rh, s->bbox[4], s->bbox[5], packed, K, zbase);
        s->packed = packed;
        s->kbits = K;
        s->zbase = zbase;
    }
}

__device__ __forceinline__ void emit_span(int row, int a, int b, int ncols, int nrows, bool packed,
                                          unsigned long long v, long long z,
                                          unsigned long long* __restrict__ D, int* __restrict__ Dc) {
    if (row < 0 || row >= nrows) return;
    a = a > 0 ? a : 0;
    b = b < ncols - 1 ? b : ncols - 1;
    if (a > b) return;
    const int64_t base = (int64_t)row * ncols;
    if (packed) {
        atomicAdd(&D[base + a], v);
        if (b + 1 < ncols) atomicAdd(&D[base + b + 1], (unsigned long long)(-(long long)v));
    } else {
        atomicAdd(&D[base + a], (unsigned long long)z);
        atomicAdd(&Dc[base + a], 1);
        if (b + 1 < ncols) {
            atomicAdd(&D[base + b + 1], (unsigned long long)(-z));
            atomicAdd(&Dc[base + b + 1], -1);
        }
    }
}

// Span path: every pixel with R2 > rs^2 adds its disc as row spans (+v at
// the first cell, -v after the last, into the per-row difference words).
// One CTA (32 x 8 threads) per 32 x kTileY raster tile.  The tile's discs
// cover a window of grid cells a little larger than the tile by the largest
// radius; the window is processed in chunks of whole rows that fit
// `win_words` 8-byte cells of shared memory.  For each chunk every disc of
// the tile adds its row spans' markers (z - zbase and 1 at the first cell,
// their negatives after the last) to two int32 arrays with native
// shared-memory atomics,
// and each touched cell is then added to the grid's difference array as one
// packed word, (sum << K) + count, with one coalesced global atomic.  The
// markers of a tile's discs fall on far fewer distinct cells than there are
// markers (neighbouring pixels' discs share rows and end near each other),
// so the grid sees a fraction of the global atomics of the direct path, and
// those it sees are contiguous.  The sum is the same: the words add modulo
// 2^64 in any order and the packed form is linear.  Tiles with the unpacked
// accumulators (separate int64 Z and int32 C), with a z range the int32
// window sums could overflow, or with windows wider than one chunk row,
// take the direct path.
constexpr int kSpanWindowWords = 4096;      // default: 32 KB per CTA (two int32 arrays)
constexpr int kSpanWindowMaxWords = 26624;  // 208 KB, the most one CTA may take

// Minimum (or maximum) of v over a 32 x 8 CTA; red: 8 ints of shared memory.
template <bool kMax>
__device__ __forceinline__ int block_reduce_int(int v, int* red) {
    v = kMax ? __reduce_max_sync(0xffffffffu, v) : __reduce_min_sync(0xffffffffu, v);
    if (threadIdx.x == 0) red[threadIdx.y] = v;
    __syncthreads();
    int r = red[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) r = kMax ? max(r, red[k]) : min(r, red[k]);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) k_scatter_window(BatchTables bt, const int2* __restrict__ pix,
                                                        const Scalars* __restrict__ sc,
                                                        unsigned long long* __restrict__ D_all,
                                                        int* __restrict__ Dc_all, int win_words) {
    extern __shared__ int swin[];              // 2 x win_words: z - zbase sums, then counts
    __shared__ int red[8];
    const int t = find_tile(bt.rt_base, bt.ntiles, blockIdx.x);
    const TileParams T = bt.tiles[t];          // by value: the loops below keep what they use in registers
    const int lt = blockIdx.x - __ldg(&bt.rt_base[t]);
    const int ntx = (T.rw + kTileX - 1) / kTileX;
    const int i = (lt % ntx) * kTileX + threadIdx.x;
    const int jt = (lt / ntx) * kTileY + threadIdx.y;
    const int rs2 = T.rs * T.rs;
    const int px = T.rx0 + i;
    int R2v[kDenseSub], zv[kDenseSub], rv[kDenseSub];
    int xlo = INT_MAX, xhi = INT_MIN, ylo = INT_MAX, yhi = INT_MIN;
#pragma unroll
    for (int sub = 0; sub < kDenseSub; ++sub) {
        const int j = jt + 8 * sub;
        int R2 = -1, z = 0;
        if (i < T.rw && j < T.rh) {
            const int2 r = pix[T.pix_off + (int64_t)j * T.rw + i];
            z = r.x;
            R2 = r.y;
        }
        const int r = R2 > rs2 ? isqrt_i32(R2) : -1;
        R2v[sub] = R2;
        zv[sub] = z;
        rv[sub] = r;
        if (r >= 0) {
            const int py = T.ry0 + j;
            xlo = min(xlo, px - r);
            xhi = max(xhi, px + r + 1);
            ylo = min(ylo, py - r);
            yhi = max(yhi, py + r);
        }
    }
    xlo = block_reduce_int<false>(xlo, red);
    if (xlo == INT_MAX) return;                 // no disc in this tile takes the span path
    xhi = block_reduce_int<true>(xhi, red);
    ylo = block_reduce_int<false>(ylo, red);
    yhi = block_reduce_int<true>(yhi, red);
    const int c0 = max(xlo, 0), c1 = min(xhi, T.ncols - 1);
    const int r0 = max(ylo, 0), r1 = min(yhi, T.nrows - 1);
    if (c0 > c1 || r0 > r1) return;             // every disc lies outside the grid
    const Scalars& s = sc[t];
    const bool packed = s.packed != 0;
    unsigned long long* D = D_all + T.cell_off;
    int* Dc = Dc_all + T.cell_off;
    const int W = c1 - c0 + 1;
    const int CH = (win_words & ~3) / W;
    // the window sums z relative to zbase and the counts in two int32 arrays
    // (native shared-memory atomics); a window cell receives at most one
    // marker per pixel of the tile, so |sum| <= kTileX * kTileY * zabs must
    // stay below 2^31
    const long long zabs = max((long long)s.bbox[5] - s.zbase, s.zbase - (long long)s.bbox[4]);
    const bool fits32 = zabs < (1LL << 31) / (kTileX * kTileY);
    if (!packed || CH < 1 || !fits32) {
        // direct path: every span's markers straight to the grid
#pragma unroll 1
        for (int sub = 0; sub < kDenseSub; ++sub) {
            const int r = rv[sub];
            if (r < 0) continue;
            const int R2 = R2v[sub], z = zv[sub];
            const int py = T.ry0 + jt + 8 * sub;
            const unsigned long long v = span_word(z, s.zbase, s.kbits);
            int w = r;
            for (int dy = 0; dy <= r; ++dy) {
                const long long t2 = (long long)R2 - (long long)dy * dy;
                while ((long long)w * w > t2) --w;
                emit_span(py + dy, px - w, px + w, T.ncols, T.nrows, packed, v, z, D, Dc);
                if (dy) emit_span(py - dy, px - w, px + w, T.ncols, T.nrows, packed, v, z, D, Dc);
            }
        }
        return;
    }
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int ncols = T.ncols;
    const int ww4 = win_words & ~3;           // whole int4s: the chunk is zeroed 16 bytes at a time
    int* sz = swin;                           // z - zbase sums
    int* scn = swin + ww4;                    // counts
#pragma unroll 1
    for (int y0 = r0; y0 <= r1; y0 += CH) {
        const int y1 = min(y0 + CH - 1, r1);
        const int nw = (y1 - y0 + 1) * W;
        for (int e = tid; e < (nw + 3) >> 2; e += 256) {
            reinterpret_cast<int4*>(sz)[e] = make_int4(0, 0, 0, 0);
            reinterpret_cast<int4*>(scn)[e] = make_int4(0, 0, 0, 0);
        }
        __syncthreads();
#pragma unroll 1
        for (int sub = 0; sub < kDenseSub; ++sub) {
            const int r = rv[sub];
            if (r < 0) continue;
            const int py = T.ry0 + jt + 8 * sub;
            const int ya = max(py - r, y0), yb = min(py + r, y1);
            if (ya > yb) continue;
            const unsigned R2 = (unsigned)R2v[sub];
            const int zr = (int)((long long)zv[sub] - s.zbase);
            // the lanes of a warp are 32 neighbouring pixels of one row, whose
            // markers on a common row often fall on one cell (same-address
            // atomics serialise); each lane starts its rows at its own offset
            // so that the warp's markers spread over the chunk's rows.  The
            // half-width floor(sqrt(t2)) comes from the hardware square-root
            // estimate, within one of it for t2 < 2^31, and one exact step
            // each way.
            const int nrow = yb - ya + 1;
            int y = ya + (int)(threadIdx.x % (unsigned)nrow);
            for (int k = 0; k < nrow; ++k, y = (y == yb) ? ya : y + 1) {
                const int dy = y - py;
                const unsigned t2 = R2 - (unsigned)(dy * dy);
                unsigned w = (unsigned)sqrt_est((float)t2);
                w -= (w * w > t2) ? 1u : 0u;
                w += ((w + 1) * (w + 1) <= t2) ? 1u : 0u;
                const int a = max(px - (int)w, 0), b = px + (int)w + 1;
                if (a >= ncols || b <= 0) continue;       // this row's span misses the grid
                const int row = (y - y0) * W - c0;     // a and b lie in [c0, c1]
                atomicAdd(&sz[row + a], zr);
                atomicAdd(&scn[row + a], 1);
                if (b < ncols) {
                    atomicAdd(&sz[row + b], -zr);
                    atomicAdd(&scn[row + b], -1);
                }
            }
        }
        __syncthreads();
        // one packed word per touched cell: (sum zrel << K) + count, modulo 2^64
        for (int rr = threadIdx.y; rr <= y1 - y0; rr += 8) {
            unsigned long long* dst = D + (int64_t)(y0 + rr) * ncols + c0;
            for (int c = threadIdx.x; c < W; c += 32) {
                const int zs = sz[rr * W + c], cn = scn[rr * W + c];
                if (zs | cn)
                    atomicAdd(&dst[c], ((unsigned long long)(long long)zs << s.kbits) +
                                           (unsigned long long)(long long)cn);
            }
        }
        __syncthreads();
    }
}

// Statistics only (not part of the launch sequence): spans per radius
// bucket of the span-path pixels (r = floor(sqrt(R2)), bucket = bit length
// of r), one CTA per 32 x kTileY raster tile.
__global__ void __launch_bounds__(256) k_span_hist(BatchTables bt, const int2* __restrict__ pix, Scalars* sc) {
    __shared__ unsigned hist[kSpanHistBuckets];
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if (tid < kSpanHistBuckets) hist[tid] = 0;
    __syncthreads();
    const int t = find_tile(bt.rt_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int lt = blockIdx.x - __ldg(&bt.rt_base[t]);
    const int ntx = (T.rw + kTileX - 1) / kTileX;
    const int i = (lt % ntx) * kTileX + threadIdx.x;
    const int rs2 = T.rs * T.rs;
    for (int sub = 0; sub < kDenseSub; ++sub) {
        const int j = (lt / ntx) * kTileY + threadIdx.y + 8 * sub;
        if (i >= T.rw || j >= T.rh) continue;
        const int R2 = pix[T.pix_off + (int64_t)j * T.rw + i].y;
        if (R2 <= rs2) continue;
        const int r = isqrt_i32(R2);
        const int k = min(32 - __clz(r), kSpanHistBuckets - 1);
        atomicAdd(&hist[k], 2u * (unsigned)r + 1u);
    }
    __syncthreads();
    if (tid < kSpanHistBuckets && hist[tid]) atomicAdd(&sc[t].span_hist[tid], (unsigned long long)hist[tid]);
}

// In-place inclusive prefix of one grid row (256 threads, 4 values each per step).
template <typename V>
__device__ __forceinline__ void row_prefix(V* __restrict__ row, int ncols, V* wsum) {
    V carry = 0;
    for (int base = 0; base < ncols; base += kScanThreads * 4) {
        const int idx = base + threadIdx.x * 4;
        V v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = (idx + k < ncols) ? row[idx + k] : V(0);
        v[1] += v[0]; v[2] += v[1]; v[3] += v[2];
        V total;
        const V excl = block_exclusive_sum(v[3], wsum, total, (int)threadIdx.x) + carry;
#pragma unroll
        for (int k = 0; k < 4; ++k) if (idx + k < ncols) row[idx + k] = v[k] + excl;
        carry += total;
    }
}

// One block per grid row: prefix of the span words, and of the int32 counts
// when the tile's accumulators are not packed.
__global__ void __launch_bounds__(kScanThreads) k_rowscan(BatchTables bt, unsigned long long* __restrict__ D_all,
                                                          int* __restrict__ Dc_all, const Scalars* __restrict__ sc) {
    __shared__ unsigned long long wsum[8];
    __shared__ int wsumc[8];
    const int t = find_tile(bt.grow_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int64_t off = T.cell_off + (int64_t)(blockIdx.x - __ldg(&bt.grow_base[t])) * T.ncols;
    row_prefix(D_all + off, T.ncols, wsum);
    if (!sc[t].packed) row_prefix(Dc_all + off, T.ncols, wsumc);
}

__device__ __forceinline__ float finalize_height(long long Z, long long C, double zs, double zo, float nodata) {
    if (C <= 0) return nodata;
    const double q = __ddiv_rn(__ll2double_rn(Z), __ll2double_rn(C));
    return __double2float_rn(__dadd_rn(__dmul_rn(q, zs), zo));
}

// Row scan, stencil and finalize in one pass: one CTA (32 x 16 threads) per
// band of 16 grid rows of a work package, walking the band's columns in
// chunks of 32.  Each warp owns one row: it prefix-sums the row's span words
// (the per-row difference form of the span path) chunk by chunk, carrying
// the running sum in a register, so the prefix is never written back; each
// cell then gathers the small discs (R2 <= H^2) of the pixels within H from
// the chunk's pixel records in shared memory, adds its prefix, and divides.
template <int H>
__global__ void __launch_bounds__(512) k_rows_final(BatchTables bt, const int2* __restrict__ pix,
                                                    Scalars* __restrict__ sc,
                                                    const unsigned long long* __restrict__ S_all,
                                                    const int* __restrict__ Sc_all, float* __restrict__ h_all) {
    constexpr int TX = 32, TY = 16, SW = TX + 2 * H, SH = TY + 2 * H;
    constexpr int NL = (SW * SH + TX * TY - 1) / (TX * TY);   // pixel records each thread loads per chunk
    __shared__ int2 tile[2][SH][SW];                          // double buffer: this chunk and the next
    const int t = find_tile(bt.band_base, bt.ntiles, blockIdx.x);
    const TileParams T = bt.tiles[t];
    const int cy0 = (blockIdx.x - __ldg(&bt.band_base[t])) * TY;
    const int2* P = pix + T.pix_off;
    Scalars* s = sc + t;
    const bool packed = s->packed != 0;
    const int K = s->kbits;
    const long long zbase = s->zbase;
    const int lane = threadIdx.x, tid = threadIdx.y * TX + threadIdx.x;
    const int qy = cy0 + threadIdx.y;
    const bool row_in = qy < T.nrows;
    // the chunk starting at column cx: this thread's pixel records (into
    // registers) and its cell's span words
    int2 rec[NL];
    auto load_tile = [&](int cx) {
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            const int idx = tid + k * TX * TY;
            int2 v = make_int2(0, -1);
            if (idx < SW * SH) {
                const int ly = idx / SW, lx = idx - ly * SW;
                const int rxi = cx - H + lx - T.rx0, ryi = cy0 - H + ly - T.ry0;
                if (rxi >= 0 && rxi < T.rw && ryi >= 0 && ryi < T.rh) v = P[(int64_t)ryi * T.rw + rxi];
            }
            rec[k] = v;
        }
    };
    auto store_tile = [&](int b) {
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            const int idx = tid + k * TX * TY;
            if (idx < SW * SH) tile[b][idx / SW][idx % SW] = rec[k];
        }
    };
    auto load_words = [&](int cx, unsigned long long& w, int& wc) {
        const int qx = cx + lane;
        const bool in = row_in && qx < T.ncols;
        const int64_t q = (int64_t)qy * T.ncols + qx;
        w = in ? S_all[T.cell_off + q] : 0ull;
        wc = (in && !packed) ? Sc_all[T.cell_off + q] : 0;
    };
    unsigned long long carry = 0;   // running prefix of the row's span words (Z when unpacked)
    int carry_c = 0;                // running prefix of the counts (unpacked)
    unsigned nod = 0;
    unsigned long long w;
    int wc;
    load_tile(0);
    store_tile(0);
    load_words(0, w, wc);
    __syncthreads();
    int b = 0;
#pragma unroll 1
    for (int cx0 = 0; cx0 < T.ncols; cx0 += TX, b ^= 1) {
        // the next chunk's loads are in flight while this one computes
        const bool more = cx0 + TX < T.ncols;
        unsigned long long w_next = 0;
        int wc_next = 0;
        if (more) {
            load_tile(cx0 + TX);
            load_words(cx0 + TX, w_next, wc_next);
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
            const int yc = __shfl_up_sync(0xffffffffu, wc, o);
            if (lane >= o) {
                w += y;
                wc += yc;
            }
        }
        w += carry;
        wc += carry_c;
        carry = __shfl_sync(0xffffffffu, w, 31);
        carry_c = __shfl_sync(0xffffffffu, wc, 31);
        long long Z = 0, C = 0;
#pragma unroll
        for (int dy = -H; dy <= H; ++dy)
#pragma unroll
            for (int dx = -H; dx <= H; ++dx) {
                if (dx * dx + dy * dy > H * H) continue;
                const int2 p = tile[b][threadIdx.y + H + dy][lane + H + dx];
                if (p.y >= dx * dx + dy * dy && p.y <= H * H) { Z += p.x; C += 1; }
            }
        const int qx = cx0 + lane;
        if (row_in && qx < T.ncols) {
            if (packed) {
                long long zb, cb;
                decode_span_word(w, K, zbase, zb, cb);
                Z += zb;
                C += cb;
            } else {
                Z += (long long)w;
                C += wc;
            }
            h_all[T.out_off + (int64_t)qy * T.ncols + qx] = finalize_height(Z, C, T.z_scale, T.z_offset, T.nodata);
            nod += C <= 0 ? 1u : 0u;
        }
        if (more) {
            // the other buffer's last readers (the chunk before this one)
            // finished before the barrier that ended that chunk
            store_tile(b ^ 1);
            w = w_next;
            wc = wc_next;
        }
        __syncthreads();
    }
    nod = __reduce_add_sync(0xffffffffu, nod);
    if (lane == 0 && nod) {
        const int slot = (blockIdx.x + threadIdx.y) & (kStatSlots - 1);
        atomicAdd(&s->nodata[slot], (unsigned long long)nod);
    }
}

}  // namespace dnni
