// dnni_search.cuh -- data layout and the exact nearest-site search of the
// discrete natural-neighbour interpolation engine, as __host__ __device__
// code shared by the sm_100a kernels (dnni_kernels.cuh) and a host build
// that the test suite checks against the oracle.
//
// Replaces, per work package:
//   nni.cpp:722-790 renderInputPoints / nni.cpp:171-230 drawPlane (the GL
//     depth-tested site planes that leave each pixel's nearest site in the
//     colour buffer)                       -> k_bin_* + k_nearest
//   nni.cpp:794-820 performNNIQueries / nni.cpp:483-534 makeBlocks and
//     cuda_nni.cu:407-488 calcNNI (query planes OR-blended into bit masks,
//     then per-pixel int32 atomics)        -> k_scatter_window + k_rows_final stencil
//   cuda_nni.cu:491-503 divide, cuda_nni.cu:399-402 zeroValues
//                                          -> k_rows_final
//
// Data layout in HBM (per call):
//   sorted points  int4 {x-ox, y-oy, z, gid}, grouped by search bin;
//   bin starts     int32 [nbins+1], bins ordered superblock (64x64 bins) ->
//                  block (8x8 bins) -> bin, so any bin, block or superblock is
//                  one contiguous point range;
//   pixel records  int2 {z of nearest site, R2 = floor(d^2/cell^2)} per
//                  raster pixel (R2 = -1: no site);
//   span sums      one 64-bit word per grid cell holding (Zrel << K) + C, or
//                  int64 Z plus int32 C when the packed form cannot hold the
//                  largest possible per-cell sums.
#pragma once

#include <climits>
#include <cstdint>
#include <cstdlib>
#include <cmath>
#include <cuda_runtime.h>

// Helpers below are __host__ __device__ so that a host build of the same code
// can be checked against the CPU oracle without a GPU.
#ifdef __CUDA_ARCH__
#define DNNI_LDG(p) __ldg(p)
#else
#define DNNI_LDG(p) (*(p))
#endif
#define DNNI_HD __host__ __device__ __forceinline__

namespace dnni {

constexpr int kBinsPerBlockEdge = 8;      // bins per block edge
constexpr int kBinsPerSuperEdge = 64;     // bins per superblock edge
constexpr int kBinsPerBlock = 64;
constexpr int kBinsPerSuper = 4096;
constexpr int kRingsBins = 2;             // bin rings searched before blocks
constexpr int kRingsBlocks = 1;           // block rings searched before superblocks
constexpr int kMaxSmallRadius = 6;
constexpr int kStatSlots = 32;
constexpr long long kCoordLimit = 1LL << 30;
constexpr long long kDistCap = (1LL << 31) - 1;

enum ErrBits { kErrRange = 1 };

struct BinGrid {
    int32_t gx0, gy0;    // bin grid origin, LAS units relative to the WP origin
    int32_t bs;          // bin edge, LAS units
    int32_t nbx, nby;    // bins per axis, multiples of 64
    int32_t n2x, n2y;    // superblocks per axis
    int32_t pad;
    int64_t nbins;
};

struct TileParams {
    int32_t ncols, nrows, cs;
    int32_t ox, oy;              // absolute LAS origin of cell (0,0)
    int32_t rx0, ry0, rw, rh;    // raster origin (cell index) and size
    int32_t r2cap;               // no pixel/cell pair is farther apart (cell units^2)
    int32_t rs;                  // small-disc radius of the stencil path
    int32_t has_gid;
    int64_t npts;
    double z_scale, z_offset;
    float nodata;
    int32_t tile_id;             // position in the caller's tile list
    int32_t has_ext;             // the caller declared the points' extent:
    int32_t ex0, ex1, ey0, ey1;  // every point must lie in it (relative, inclusive)
    BinGrid bg;
    // where this tile's parts live in the batch's arrays
    int64_t pt_off;              // input points (xyz rows, gids)
    int64_t srt_off;             // sorted points and bin ranks (tiles may share input rows)
    int64_t bin_off;             // bin counts / starts (nbins + 1 entries)
    int64_t blk_off;             // block masks, block nearest map (nbins / 64)
    int64_t sup_off;             // superblock masks (nbins / 4096)
    int64_t pix_off;             // raster pixel records
    int64_t cell_off;            // span words (grid cells)
    int64_t out_off;             // heights in the caller's output array
    int64_t site_off;            // site map in the caller's array, -1 = none
};

constexpr int kSpanHistBuckets = 16;   // span radius r in [2^(k-1), 2^k), k = 0: r = 0

struct Scalars {
    int32_t bbox[6];             // min/max of x-ox, y-oy, z
    int32_t err;
    int32_t packed;              // decided after the nearest-site pass
    int32_t kbits;
    int32_t pad;
    long long zbase;
    int32_t max_r2[kStatSlots];
    unsigned long long big_pixels[kStatSlots];
    unsigned long long spans[kStatSlots];
    unsigned long long nodata[kStatSlots];
    unsigned long long evals_dense[kStatSlots];   // candidate evaluations of the ring search
    unsigned long long evals_far[kStatSlots];     // and of the far pass (seeds and disc search)
    unsigned long long span_hist[kSpanHistBuckets];   // spans per radius bucket (statistics runs)
};

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------

#ifdef __CUDACC__
// Square-root estimate of a non-negative float from the hardware
// approximation (PTX sqrt.approx.ftz.f32; relative error a few units of
// 2^-23), for callers that correct the result with exact integer products or
// need it only within a fraction of one unit (below 2^31 the absolute error
// stays under 0.05).
__device__ __forceinline__ float sqrt_est(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
#endif

DNNI_HD int isqrt_i32(int v) {
    // floor(sqrt(v)) for 0 <= v < 2^31: float estimate, exact integer fix-up
#ifdef __CUDA_ARCH__
    int s = (int)sqrt_est((float)v);
#else
    int s = (int)sqrtf((float)v);
#endif
    while ((long long)s * s > v) --s;
    while ((long long)(s + 1) * (s + 1) <= v) ++s;
    return s;
}

// a / b for 0 <= a < 2^32, 0 < b < 2^32 (32-bit unsigned divide; a 64-bit
// divide costs several times more on the GPU)
DNNI_HD int udiv32(long long a, long long b) { return (int)((uint32_t)a / (uint32_t)b); }

// min(floor(d2 / cs2), cap) exactly: the quotient estimate from doubles is
// within one of the truth for quotients below 2^31, and is then corrected
// with exact products.
DNNI_HD int r2_of(long long d2, long long cs2, int cap) {
    if (d2 >= ((long long)cap + 1) * cs2) return cap;
    if (d2 < (1LL << 32) && cs2 < (1LL << 32)) return (int)((uint32_t)d2 / (uint32_t)cs2);
    long long q = (long long)((double)d2 / (double)cs2);
    while (q > 0 && q * cs2 > d2) --q;
    while ((q + 1) * cs2 <= d2) ++q;
    return (int)(q < cap ? q : cap);
}

DNNI_HD int64_t bin_id(const BinGrid& g, int bx, int by) {
    const int sx = bx >> 6, sy = by >> 6;
    const int bkx = (bx >> 3) & 7, bky = (by >> 3) & 7;
    const int lx = bx & 7, ly = by & 7;
    return ((int64_t)(sy * g.n2x + sx) << 12) | (int64_t)(((bky << 3) | bkx) << 6) | (int64_t)((ly << 3) | lx);
}

DNNI_HD int rel_coord(int32_t a, int32_t o) {
    // a - o, exact when the true difference fits in int32 (checked by k_bbox)
    return (int)((uint32_t)a - (uint32_t)o);
}

struct Best {
    long long d2;
    uint32_t gid;
    int z;
    int idx;      // position of the site in the sorted point array
    int nev;      // candidate distance evaluations made for this pixel
};

// Most candidates are farther than the best so far; one comparison of the
// distance rejects them, and only the rest go through the full (d2, gid, z)
// order (written as a branch expected not taken: on the far pass's wide
// candidate sets this beat the flat three-key comparison).
DNNI_HD void consider(Best& b, const int4 p, int q, int px, int py) {
    const int dx = p.x - px, dy = p.y - py;      // |p.x|, |px| < 2^30
    const long long d2 = (long long)dx * dx + (long long)dy * dy;
    if (__builtin_expect(d2 <= b.d2, 0)) {
        const uint32_t g = (uint32_t)p.w;
        if (d2 < b.d2 || g < b.gid || (g == b.gid && p.z < b.z)) {
            b.d2 = d2;
            b.gid = g;
            b.z = p.z;
            b.idx = q;
        }
    }
}

// consider() for a pixel whose bound is below 2^31 (a real site found): a
// candidate with |dx| or |dy| above 46340 lies beyond the bound, so the
// distance and its comparison stay in 32-bit arithmetic.  Same result.
DNNI_HD void consider_below31(Best& b, const int4 p, int q, int px, int py) {
    const int dx = p.x - px, dy = p.y - py;      // |p.x|, |px| < 2^30
    const unsigned ax = (unsigned)(dx < 0 ? -dx : dx), ay = (unsigned)(dy < 0 ? -dy : dy);
    if (ax > 46340u || ay > 46340u) return;
    const unsigned d2 = ax * ax + ay * ay, bd = (unsigned)b.d2;
    if (__builtin_expect(d2 <= bd, 0)) {
        const uint32_t g = (uint32_t)p.w;
        if (d2 < bd || g < b.gid || (g == b.gid && p.z < b.z)) {
            b.d2 = d2;
            b.gid = g;
            b.z = p.z;
            b.idx = q;
        }
    }
}

DNNI_HD long long axis_gap(long long p, long long lo, long long hi) {
    long long d = p < lo ? lo - p : (p > hi ? p - hi : 0);
    return d < kDistCap ? d : kDistCap;
}

// squared distance lower bound from (px,py) to the box [x0,x1] x [y0,y1]
DNNI_HD long long box_lb(long long px, long long py, long long x0, long long x1,
                                            long long y0, long long y1) {
    const long long dx = axis_gap(px, x0, x1), dy = axis_gap(py, y0, y1);
    return dx * dx + dy * dy;
}

// Cell e (0 <= e < ring_size(k)) of the Chebyshev ring k around (cx,cy):
// bottom row, top row, then the left/right columns in between.
DNNI_HD int ring_size(int k) { return k ? 8 * k : 1; }

DNNI_HD void ring_cell(int cx, int cy, int k, int e, int& x, int& y) {
    const int side = 2 * k + 1;
    if (e < side) {
        x = cx - k + e;
        y = cy - k;
    } else if (e < 2 * side) {
        x = cx - k + (e - side);
        y = cy + k;
    } else {
        const int f = e - 2 * side;
        x = (f & 1) ? cx + k : cx - k;
        y = cy - k + 1 + (f >> 1);
    }
}

// After visiting every cell of the (unclipped) box [x0,x1]x[y0,y1] of a level
// whose cells are u LAS units wide, every unvisited point lies at distance
// >= m from (px,py); the search may stop once best < m^2.  Sides at the grid
// border are closed (nothing lies beyond them).
DNNI_HD bool ring_done(long long best, long long px, long long py, long long gx0,
                                          long long gy0, long long u, int x0, int x1, int y0, int y1,
                                          int nx, int ny) {
    long long m = LLONG_MAX;
    bool open = false;
    if (x0 > 0) { long long v = px - (gx0 + (long long)x0 * u) + 1; m = v < m ? v : m; open = true; }
    if (x1 < nx - 1) { long long v = gx0 + (long long)(x1 + 1) * u - px; m = v < m ? v : m; open = true; }
    if (y0 > 0) { long long v = py - (gy0 + (long long)y0 * u) + 1; m = v < m ? v : m; open = true; }
    if (y1 < ny - 1) { long long v = gy0 + (long long)(y1 + 1) * u - py; m = v < m ? v : m; open = true; }
    if (!open) return true;
    if (m > kDistCap) m = kDistCap;
    return best < m * m;
}

DNNI_HD void scan_points(Best& b, const int4* __restrict__ pts, int s, int e, int px, int py) {
    b.nev += e - s;
    for (int q = s; q < e; ++q) consider(b, DNNI_LDG(&pts[q]), q, px, py);
}

// Conservative bound on the distance reach of a squared bound v >= 0:
// floor(sqrt(v)) + 1 (the double square root is correctly rounded; the +1
// absorbs its rounding, so no cell within the disc is ever left out).
DNNI_HD long long reach_of(long long v) { return (long long)sqrt((double)v) + 1; }

// Range [lo,hi] of cell indices (cells u wide from origin o, n of them)
// that the interval [c-w, c+w] touches; empty when lo > hi.
DNNI_HD void cell_range(long long c, long long w, long long o, long long u, int n, int& lo, int& hi) {
    long long a = c - w, b = c + w;
    const long long end = o + (long long)n * u - 1;
    if (b < o || a > end) { lo = 1; hi = 0; return; }
    if (a < o) a = o;
    if (b > end) b = end;
    lo = udiv32(a - o, u);
    hi = udiv32(b - o, u);
}

// Level 0 of the search: bin rings 0..kRingsBins around the pixel's bin.
// Returns true when the nearest site is certain.
DNNI_HD bool search_bins(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                         int px, int py, Best& b) {
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    int bx = udiv32((long long)px - gx0, bs);
    int by = udiv32((long long)py - gy0, bs);
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    for (int k = 0; k <= kRingsBins; ++k) {
        const int ne = ring_size(k);
        for (int e = 0; e < ne; ++e) {
            int x, y;
            ring_cell(bx, by, k, e, x, y);
            if (x < 0 || y < 0 || x >= g.nbx || y >= g.nby) continue;
            const long long X0 = gx0 + (long long)x * bs, Y0 = gy0 + (long long)y * bs;
            if (k > 0 && box_lb(px, py, X0, X0 + bs - 1, Y0, Y0 + bs - 1) > b.d2) continue;
            const int64_t id = bin_id(g, x, y);
            scan_points(b, pts, DNNI_LDG(&start[id]), DNNI_LDG(&start[id + 1]), px, py);
        }
        if (ring_done(b.d2, px, py, gx0, gy0, bs, bx - k, bx + k, by - k, by + k, g.nbx, g.nby)) return true;
    }
    return false;
}

// A tile's staged bin window: the bins [wx0, wx0+wnx) x [wy0, wy0+wny) with
// their points copied (to shared memory) in window row-major bin order.
struct BinWindow {
    int wx0, wy0, wnx, wny;
    const int* lstart;   // wnx*wny+1 starts into lpts
    const int* gstart;   // sorted-array position of each window bin's first point
    const int4* lpts;
};

// search_bins on a staged window; identical results.  Every bin within
// kRingsBins rings of the pixel's bin (inside the grid) must lie in the window.
DNNI_HD bool search_bins_window(const BinGrid& g, const BinWindow& w, int px, int py, Best& b) {
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    int bx = udiv32((long long)px - gx0, bs);
    int by = udiv32((long long)py - gy0, bs);
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    for (int k = 0; k <= kRingsBins; ++k) {
        const int ne = ring_size(k);
        for (int e = 0; e < ne; ++e) {
            int x, y;
            ring_cell(bx, by, k, e, x, y);
            if (x < 0 || y < 0 || x >= g.nbx || y >= g.nby) continue;
            const long long X0 = gx0 + (long long)x * bs, Y0 = gy0 + (long long)y * bs;
            if (k > 0 && box_lb(px, py, X0, X0 + bs - 1, Y0, Y0 + bs - 1) > b.d2) continue;
            const int lk = (y - w.wy0) * w.wnx + (x - w.wx0);
            const int s0 = w.lstart[lk], e0 = w.lstart[lk + 1], g0 = w.gstart[lk];
            b.nev += e0 - s0;
            for (int q = s0; q < e0; ++q) consider(b, w.lpts[q], g0 + (q - s0), px, py);
        }
        if (ring_done(b.d2, px, py, gx0, gy0, bs, bx - k, bx + k, by - k, by + k, g.nbx, g.nby)) return true;
    }
    return false;
}

// The bin rings of search_bins_window with contiguous ranges: in the staged
// window's row-major order each row of a pixel's 3 x 3 (then 5 x 5) bin
// neighbourhood is one run of points, so rings 0-1 are three loops and ring 2
// is two rows plus two columns.  b.idx holds a window-local point index on
// return (window_global_index converts it).  Same result as search_bins.
DNNI_HD void scan_local(Best& b, const int4* lpts, int s, int e, int px, int py) {
    b.nev += e - s;
    for (int q = s; q < e; ++q) consider(b, lpts[q], q, px, py);
}

DNNI_HD bool search_window_fast(const BinGrid& g, const BinWindow& w, int px, int py, Best& b) {
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    int bx = udiv32((long long)px - gx0, bs);
    int by = udiv32((long long)py - gy0, bs);
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    const int lx = bx - w.wx0, ly = by - w.wy0;
    {
        const int x0 = lx - 1 > 0 ? lx - 1 : 0, x1 = lx + 1 < w.wnx - 1 ? lx + 1 : w.wnx - 1;
        const int y0 = ly - 1 > 0 ? ly - 1 : 0, y1 = ly + 1 < w.wny - 1 ? ly + 1 : w.wny - 1;
        for (int r = y0; r <= y1; ++r) scan_local(b, w.lpts, w.lstart[r * w.wnx + x0], w.lstart[r * w.wnx + x1 + 1], px, py);
    }
    if (ring_done(b.d2, px, py, gx0, gy0, bs, bx - 1, bx + 1, by - 1, by + 1, g.nbx, g.nby)) return true;
    {
        const int x0 = lx - 2 > 0 ? lx - 2 : 0, x1 = lx + 2 < w.wnx - 1 ? lx + 2 : w.wnx - 1;
        const long long X0 = gx0 + (long long)(w.wx0 + x0) * bs, X1 = gx0 + (long long)(w.wx0 + x1 + 1) * bs - 1;
        for (int d = -2; d <= 2; d += 4) {
            const int r = ly + d;
            if (r < 0 || r >= w.wny) continue;
            const long long Y0 = gy0 + (long long)(w.wy0 + r) * bs;
            if (box_lb(px, py, X0, X1, Y0, Y0 + bs - 1) > b.d2) continue;
            scan_local(b, w.lpts, w.lstart[r * w.wnx + x0], w.lstart[r * w.wnx + x1 + 1], px, py);
        }
        const int ya = ly - 1 > 0 ? ly - 1 : 0, yb = ly + 1 < w.wny - 1 ? ly + 1 : w.wny - 1;
        const long long Y0 = gy0 + (long long)(w.wy0 + ya) * bs, Y1 = gy0 + (long long)(w.wy0 + yb + 1) * bs - 1;
        for (int d = -2; d <= 2; d += 4) {
            const int c = lx + d;
            if (c < 0 || c >= w.wnx) continue;
            const long long CX0 = gx0 + (long long)(w.wx0 + c) * bs;
            if (box_lb(px, py, CX0, CX0 + bs - 1, Y0, Y1) > b.d2) continue;
            for (int r = ya; r <= yb; ++r)
                scan_local(b, w.lpts, w.lstart[r * w.wnx + c], w.lstart[r * w.wnx + c + 1], px, py);
        }
    }
    return ring_done(b.d2, px, py, gx0, gy0, bs, bx - 2, bx + 2, by - 2, by + 2, g.nbx, g.nby);
}

// The same search with 32-bit distances, for windows that span less than
// 2^15 LAS units in each direction (squared distances then fit in 31 bits).
// The (d^2, gid) part of the (d^2, gid, z) order is one 64-bit key.
struct Best32 {
    unsigned long long key;   // d2 << 32 | gid; ~0 = none
    int z;
    int idx;
    int nev;                  // candidate distance evaluations
};

DNNI_HD void consider32(Best32& b, const int4 p, int q, int px, int py) {
    const int dx = p.x - px, dy = p.y - py;
    const unsigned d2 = (unsigned)(dx * dx) + (unsigned)(dy * dy);
    const unsigned long long key = ((unsigned long long)d2 << 32) | (unsigned)p.w;
    if (key < b.key || (key == b.key && p.z < b.z)) {
        b.key = key;
        b.z = p.z;
        b.idx = q;
    }
}

DNNI_HD long long best32_d2(const Best32& b) { return b.key == ~0ull ? LLONG_MAX : (long long)(b.key >> 32); }

DNNI_HD void scan_local32(Best32& b, const int4* lpts, int s, int e, int px, int py) {
    b.nev += e - s;
#pragma unroll 2
    for (int q = s; q < e; ++q) consider32(b, lpts[q], q, px, py);
}

DNNI_HD bool window_fits32(const BinGrid& g, const BinWindow& w) {
    const long long ax = g.gx0 < 0 ? -(long long)g.gx0 : g.gx0, ay = g.gy0 < 0 ? -(long long)g.gy0 : g.gy0;
    return (long long)(w.wnx + 1) * g.bs < 32768 && (long long)(w.wny + 1) * g.bs < 32768 &&
           ax + (long long)(g.nbx + 1) * g.bs < (1LL << 31) && ay + (long long)(g.nby + 1) * g.bs < (1LL << 31);
}

// ring_done for the 32-bit window path: every coordinate involved lies
// within the window (less than 2^15 LAS units from the pixel), so the margins
// and their squares fit in 32 bits; a missing best (none found) never stops.
DNNI_HD bool ring_done32(long long best, int px, int py, const BinGrid& g, int x0, int x1, int y0, int y1) {
    if (best == LLONG_MAX) return false;
    int m = INT_MAX;
    bool open = false;
    const int gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    if (x0 > 0) { const int v = px - (gx0 + x0 * bs) + 1; m = v < m ? v : m; open = true; }
    if (x1 < g.nbx - 1) { const int v = gx0 + (x1 + 1) * bs - px; m = v < m ? v : m; open = true; }
    if (y0 > 0) { const int v = py - (gy0 + y0 * bs) + 1; m = v < m ? v : m; open = true; }
    if (y1 < g.nby - 1) { const int v = gy0 + (y1 + 1) * bs - py; m = v < m ? v : m; open = true; }
    if (!open) return true;
    return best < (long long)m * m;
}

DNNI_HD bool search_window_fast32(const BinGrid& g, const BinWindow& w, int px, int py, Best& out) {
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    int bx = udiv32((long long)px - gx0, bs);
    int by = udiv32((long long)py - gy0, bs);
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    const int lx = bx - w.wx0, ly = by - w.wy0;
    Best32 b{~0ull, INT_MAX, -1, 0};
    bool done;
    {
        const int x0 = lx - 1 > 0 ? lx - 1 : 0, x1 = lx + 1 < w.wnx - 1 ? lx + 1 : w.wnx - 1;
        const int y0 = ly - 1 > 0 ? ly - 1 : 0, y1 = ly + 1 < w.wny - 1 ? ly + 1 : w.wny - 1;
        for (int r = y0; r <= y1; ++r)
            scan_local32(b, w.lpts, w.lstart[r * w.wnx + x0], w.lstart[r * w.wnx + x1 + 1], px, py);
    }
    done = ring_done32(best32_d2(b), px, py, g, bx - 1, bx + 1, by - 1, by + 1);
    if (!done) {
        const int x0 = lx - 2 > 0 ? lx - 2 : 0, x1 = lx + 2 < w.wnx - 1 ? lx + 2 : w.wnx - 1;
        const long long X0 = gx0 + (long long)(w.wx0 + x0) * bs, X1 = gx0 + (long long)(w.wx0 + x1 + 1) * bs - 1;
        for (int d = -2; d <= 2; d += 4) {
            const int r = ly + d;
            if (r < 0 || r >= w.wny) continue;
            const long long Y0 = gy0 + (long long)(w.wy0 + r) * bs;
            if (box_lb(px, py, X0, X1, Y0, Y0 + bs - 1) > best32_d2(b)) continue;
            scan_local32(b, w.lpts, w.lstart[r * w.wnx + x0], w.lstart[r * w.wnx + x1 + 1], px, py);
        }
        const int ya = ly - 1 > 0 ? ly - 1 : 0, yb = ly + 1 < w.wny - 1 ? ly + 1 : w.wny - 1;
        const long long Y0 = gy0 + (long long)(w.wy0 + ya) * bs, Y1 = gy0 + (long long)(w.wy0 + yb + 1) * bs - 1;
        for (int d = -2; d <= 2; d += 4) {
            const int c = lx + d;
            if (c < 0 || c >= w.wnx) continue;
            const long long CX0 = gx0 + (long long)(w.wx0 + c) * bs;
            if (box_lb(px, py, CX0, CX0 + bs - 1, Y0, Y1) > best32_d2(b)) continue;
            for (int r = ya; r <= yb; ++r)
                scan_local32(b, w.lpts, w.lstart[r * w.wnx + c], w.lstart[r * w.wnx + c + 1], px, py);
        }
        done = ring_done32(best32_d2(b), px, py, g, bx - 2, bx + 2, by - 2, by + 2);
    }
    out.d2 = best32_d2(b);
    out.gid = b.key == ~0ull ? 0xFFFFFFFFu : (uint32_t)(b.key & 0xFFFFFFFFull);
    out.z = b.z;
    out.idx = b.idx;
    out.nev += b.nev;
    return done;
}

// Sorted-array position of window-local point q (-1 stays -1).
DNNI_HD int window_global_index(const BinWindow& w, int q) {
    if (q < 0) return -1;
    int lo = 0, hi = w.wnx * w.wny - 1;     // last bin with lstart <= q
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (w.lstart[mid] <= q) lo = mid; else hi = mid - 1;
    }
    return w.gstart[lo] + (q - w.lstart[lo]);
}

// Window of the 32 x rows pixel band whose first pixel is raster (i0, j0).
// Raster tiles are 32 x kTileY pixels, one CTA of 32 x 8 threads each; a
// thread takes kDenseSub pixels of its column, so that one staged bin window
// serves kTileY rows.
constexpr int kDenseSub = 8;
constexpr int kTileX = 32, kTileY = 8 * kDenseSub;
DNNI_HD void tile_window(const TileParams& t, int i0, int j0, int rows, int& wx0, int& wy0, int& wnx, int& wny) {
    const BinGrid& g = t.bg;
    const int i1 = (i0 + kTileX - 1 < t.rw - 1) ? i0 + kTileX - 1 : t.rw - 1;
    const int j1 = (j0 + rows - 1 < t.rh - 1) ? j0 + rows - 1 : t.rh - 1;
    long long bxa = udiv32((long long)(t.rx0 + i0) * t.cs - g.gx0, g.bs), bxb = udiv32((long long)(t.rx0 + i1) * t.cs - g.gx0, g.bs);
    long long bya = udiv32((long long)(t.ry0 + j0) * t.cs - g.gy0, g.bs), byb = udiv32((long long)(t.ry0 + j1) * t.cs - g.gy0, g.bs);
    bxa = bxa < g.nbx - 1 ? bxa : g.nbx - 1;
    bxb = bxb < g.nbx - 1 ? bxb : g.nbx - 1;
    bya = bya < g.nby - 1 ? bya : g.nby - 1;
    byb = byb < g.nby - 1 ? byb : g.nby - 1;
    const long long x0 = bxa - kRingsBins > 0 ? bxa - kRingsBins : 0, x1 = bxb + kRingsBins < g.nbx - 1 ? bxb + kRingsBins : g.nbx - 1;
    const long long y0 = bya - kRingsBins > 0 ? bya - kRingsBins : 0, y1 = byb + kRingsBins < g.nby - 1 ? byb + kRingsBins : g.nby - 1;
    wx0 = (int)x0;
    wy0 = (int)y0;
    wnx = (int)(x1 - x0 + 1);
    wny = (int)(y1 - y0 + 1);
}

// Occupancy masks: bit l of bmask[block] is set when bin l of that block
// (row-major 8x8) holds points; bit m of smask[superblock] when block m of it
// does.  They let the search skip empty cells without touching their ranges.
DNNI_HD int ffs64(uint64_t v) {
#ifdef __CUDA_ARCH__
    return __ffsll((long long)v) - 1;
#else
    return __builtin_ctzll(v);
#endif
}

// A first bound for a pixel whose bound is still infinite: the nearest
// non-empty superblock ring is found, and in each of its non-empty
// superblocks the closest non-empty block and, in it, the closest non-empty
// bin contribute their points.  Needs n > 0.
DNNI_HD void seed_from_superblocks(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                                   const uint64_t* __restrict__ bmask, const uint64_t* __restrict__ smask,
                                   int px, int py, Best& b) {
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    const long long u1 = bs * kBinsPerBlockEdge, u2 = bs * kBinsPerSuperEdge;
    int cx = udiv32((long long)px - gx0, u2), cy = udiv32((long long)py - gy0, u2);
    cx = cx < g.n2x - 1 ? cx : g.n2x - 1;
    cy = cy < g.n2y - 1 ? cy : g.n2y - 1;
    const int kmax = (g.n2x > g.n2y ? g.n2x : g.n2y);
    for (int k = 0; k <= kmax; ++k) {
        bool found = false;
        const int ne = ring_size(k);
        for (int e = 0; e < ne; ++e) {
            int x, y;
            ring_cell(cx, cy, k, e, x, y);
            if (x < 0 || y < 0 || x >= g.n2x || y >= g.n2y) continue;
            const int sidx = y * g.n2x + x;
            uint64_t sm = DNNI_LDG(&smask[sidx]);
            if (!sm) continue;
            found = true;
            const long long SX0 = gx0 + (long long)x * u2, SY0 = gy0 + (long long)y * u2;
            long long blb = LLONG_MAX;
            int bm_idx = 0;
            while (sm) {
                const int m = ffs64(sm);
                sm &= sm - 1;
                const long long BX0 = SX0 + (long long)(m & 7) * u1, BY0 = SY0 + (long long)(m >> 3) * u1;
                const long long lb = box_lb(px, py, BX0, BX0 + u1 - 1, BY0, BY0 + u1 - 1);
                if (lb < blb) { blb = lb; bm_idx = m; }
            }
            const int64_t blk = ((int64_t)sidx << 6) + bm_idx;
            uint64_t bm = DNNI_LDG(&bmask[blk]);
            const long long BX0 = SX0 + (long long)(bm_idx & 7) * u1, BY0 = SY0 + (long long)(bm_idx >> 3) * u1;
            long long qlb = LLONG_MAX;
            int q_idx = 0;
            while (bm) {
                const int l = ffs64(bm);
                bm &= bm - 1;
                const long long QX0 = BX0 + (long long)(l & 7) * bs, QY0 = BY0 + (long long)(l >> 3) * bs;
                const long long lb = box_lb(px, py, QX0, QX0 + bs - 1, QY0, QY0 + bs - 1);
                if (lb < qlb) { qlb = lb; q_idx = l; }
            }
            const int64_t id = (blk << 6) + q_idx;
            scan_points(b, pts, DNNI_LDG(&start[id]), DNNI_LDG(&start[id + 1]), px, py);
        }
        if (found) return;
    }
}

// Exact search inside the disc of the current bound: every non-empty
// superblock, block and bin the disc touches is visited (superblock rows in
// order of distance from the pixel, columns narrowed per row to the disc's
// chord, empty cells skipped through the occupancy masks), and nothing else.
// The bound only shrinks, so a cell left out when its row was reached can
// never hold a closer site.  Complete whenever b holds a real site on entry.
DNNI_HD void search_disc(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                         const uint64_t* __restrict__ bmask, const uint64_t* __restrict__ smask,
                         int px, int py, Best& b) {
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    const long long u1 = bs * kBinsPerBlockEdge, u2 = bs * kBinsPerSuperEdge;
    int sy0, sy1;
    cell_range(py, reach_of(b.d2), gy0, u2, g.n2y, sy0, sy1);
    if (sy0 > sy1) return;
    int csy = udiv32((long long)py - gy0, u2);
    csy = csy < sy0 ? sy0 : (csy > sy1 ? sy1 : csy);
    const int span = (csy - sy0) > (sy1 - csy) ? (csy - sy0) : (sy1 - csy);
    for (int r = 0; r <= 2 * span; ++r) {
        // superblock rows outward from the pixel's own row: csy, csy-1, csy+1, ...
        const int sy = csy + ((r & 1) ? -((r + 1) >> 1) : (r >> 1));
        if (sy < sy0 || sy > sy1) continue;
        const long long SY0 = gy0 + (long long)sy * u2;
        const long long gy = axis_gap(py, SY0, SY0 + u2 - 1);
        if (gy * gy > b.d2) continue;
        int sx0, sx1;
        cell_range(px, reach_of(b.d2 - gy * gy), gx0, u2, g.n2x, sx0, sx1);
        for (int sx = sx0; sx <= sx1; ++sx) {
            const int sidx = sy * g.n2x + sx;
            const uint64_t sm = DNNI_LDG(&smask[sidx]);
            if (!sm) continue;
            const long long SX0 = gx0 + (long long)sx * u2;
            if (box_lb(px, py, SX0, SX0 + u2 - 1, SY0, SY0 + u2 - 1) > b.d2) continue;
            // non-empty blocks of this superblock within the bound
            for (int ly = 0; ly < kBinsPerBlockEdge; ++ly) {
                unsigned row = (unsigned)(sm >> (ly * 8)) & 0xFFu;
                if (!row) continue;
                const long long BY0 = SY0 + (long long)ly * u1;
                const long long gyb = axis_gap(py, BY0, BY0 + u1 - 1);
                const long long gyb2 = gyb * gyb;
                if (gyb2 > b.d2) continue;
                while (row) {
                    const int lx = ffs64(row);
                    row &= row - 1;
                    const long long BX0 = SX0 + (long long)lx * u1;
                    const long long gxb = axis_gap(px, BX0, BX0 + u1 - 1);
                    if (gxb * gxb + gyb2 > b.d2) continue;
                    const int64_t blk = ((int64_t)sidx << 6) + ly * 8 + lx;
                    const uint64_t bm = DNNI_LDG(&bmask[blk]);
                    // non-empty bins of this block within the bound
                    for (int qy = 0; qy < kBinsPerBlockEdge; ++qy) {
                        unsigned qrow = (unsigned)(bm >> (qy * 8)) & 0xFFu;
                        if (!qrow) continue;
                        const long long QY0 = BY0 + (long long)qy * bs;
                        const long long gq = axis_gap(py, QY0, QY0 + bs - 1);
                        const long long gq2 = gq * gq;
                        if (gq2 > b.d2) continue;
                        const int64_t id0 = (blk << 6) + qy * 8;
                        while (qrow) {
                            const int qx = ffs64(qrow);
                            qrow &= qrow - 1;
                            const long long QX0 = BX0 + (long long)qx * bs;
                            const long long gx = axis_gap(px, QX0, QX0 + bs - 1);
                            if (gx * gx + gq2 > b.d2) continue;
                            scan_points(b, pts, DNNI_LDG(&start[id0 + qx]), DNNI_LDG(&start[id0 + qx + 1]), px, py);
                        }
                    }
                }
            }
        }
    }
}

// Block index (in bmask order) of block (cx, cy) of the block grid.
DNNI_HD int64_t block_index(const BinGrid& g, int cx, int cy) {
    return ((int64_t)((cy >> 3) * g.n2x + (cx >> 3)) << 6) + (((cy & 7) << 3) | (cx & 7));
}

// 8 x 8 mask of the cells [a0,a1] x [b0,b1] of a block (x = bit & 7,
// y = bit >> 3), clipped to the block; 0 when the range is empty.
DNNI_HD uint64_t cell_box_mask8(int a0, int a1, int b0, int b1) {
    a0 = a0 > 0 ? a0 : 0;
    b0 = b0 > 0 ? b0 : 0;
    a1 = a1 < 7 ? a1 : 7;
    b1 = b1 < 7 ? b1 : 7;
    if (a0 > a1 || b0 > b1) return 0;
    const uint64_t row = (0xFFull >> (7 - a1 + a0)) << a0;
    return (row * 0x0101010101010101ull) & (~0ull >> (8 * (7 - b1))) & (~0ull << (8 * b0));
}

// A first bound from the nearest non-empty block map: the points of a
// non-empty bin of block `nb` (in bmask order) close to the pixel.  The
// pixel's cell in the block (clamped to the block) is the centre of square
// rings of bins; the first ring that holds a non-empty bin gives the
// candidates, and the one whose box is closest to the pixel is scanned.  Any
// non-empty bin gives a real site, so the search stays exact; a near one
// keeps the disc that the search then walks small.
DNNI_HD void seed_from_block(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                             const uint64_t* __restrict__ bmask, int64_t nb, int px, int py, Best& b) {
    const long long bs = g.bs, u1 = bs * kBinsPerBlockEdge, u2 = bs * kBinsPerSuperEdge;
    const int64_t sidx = nb >> 6;
    const int m = (int)(nb & 63);
    const long long BX0 = g.gx0 + (long long)(sidx % g.n2x) * u2 + (long long)(m & 7) * u1;
    const long long BY0 = g.gy0 + (long long)(sidx / g.n2x) * u2 + (long long)(m >> 3) * u1;
    const uint64_t bm = DNNI_LDG(&bmask[nb]);
    const long long dx = (long long)px - BX0, dy = (long long)py - BY0;
    const int cx = dx < 0 ? 0 : (dx >= u1 ? 7 : udiv32(dx, bs));
    const int cy = dy < 0 ? 0 : (dy >= u1 ? 7 : udiv32(dy, bs));
    uint64_t hit = 0;
    for (int r = 0; r < 8 && !hit; ++r) hit = bm & cell_box_mask8(cx - r, cx + r, cy - r, cy + r);
    long long qlb = LLONG_MAX;
    int q_idx = 0;
    while (hit) {
        const int l = ffs64(hit);
        hit &= hit - 1;
        const long long QX0 = BX0 + (long long)(l & 7) * bs, QY0 = BY0 + (long long)(l >> 3) * bs;
        const long long lb = box_lb(px, py, QX0, QX0 + bs - 1, QY0, QY0 + bs - 1);
        if (lb < qlb) { qlb = lb; q_idx = l; }
    }
    const int64_t id = (nb << 6) + q_idx;
    scan_points(b, pts, DNNI_LDG(&start[id]), DNNI_LDG(&start[id + 1]), px, py);
}

// Completes the search of a pixel that the bin rings did not settle: the
// bound so far (b) or else the nearest non-empty superblock gives a real
// site, and the disc of that bound is searched exhaustively.
DNNI_HD void finish_search(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                           const uint64_t* __restrict__ bmask, const uint64_t* __restrict__ smask,
                           int px, int py, Best& b, const int64_t* __restrict__ near = nullptr) {
    if (near) {
        // the nearest non-empty block of the pixel's block
        const int n1x = g.nbx >> 3;
        int bx = udiv32((long long)px - g.gx0, g.bs), by = udiv32((long long)py - g.gy0, g.bs);
        bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
        by = by < g.nby - 1 ? by : g.nby - 1;
        const int64_t nb = DNNI_LDG(&near[(int64_t)(by >> 3) * n1x + (bx >> 3)]);
        if (nb >= 0) seed_from_block(g, pts, start, bmask, nb, px, py, b);
    }
    if (b.d2 == LLONG_MAX) seed_from_superblocks(g, pts, start, bmask, smask, px, py, b);
    search_disc(g, pts, start, bmask, smask, px, py, b);
}

// Exact nearest site of the pixel at (px,py) (LAS units relative to the WP
// origin), all levels in one call.
DNNI_HD void nearest_search(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                            const uint64_t* __restrict__ bmask, const uint64_t* __restrict__ smask,
                            int px, int py, Best& b) {
    if (search_bins(g, pts, start, px, py, b)) return;
    finish_search(g, pts, start, bmask, smask, px, py, b);
}

DNNI_HD int64_t point_bin(const BinGrid& g, int xr, int yr) {
    int bx = (int)((uint32_t)(xr - g.gx0) / (uint32_t)g.bs);
    int by = (int)((uint32_t)(yr - g.gy0) / (uint32_t)g.bs);
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    return bin_id(g, bx, by);
}

// Picks the accumulator form for the span path.  The per-cell count from big
// discs is at most the lattice points of a disc of radius^2 max_r2, (2r+1)^2,
// and at most the raster size; z enters relative to zbase (the mid-range),
// so |Zrel| <= C * zabs.  Packed: word = (Zrel << K) + C with C < 2^K and
// |Zrel| < 2^(62-K); otherwise separate int64 Z and int32 C.
DNNI_HD void decide_packing(int max_r2, long long npix, long long zmin, long long zmax, int& packed, int& K,
                            long long& zbase, int layers = 1) {
    long long cb = 0;
    if (max_r2 >= 0) {
        const long long r = isqrt_i32(max_r2);
        cb = (2 * r + 1) * (2 * r + 1);
        if (cb > npix) cb = npix;
        cb *= layers;          // stacked rasters (space-time slices) add up per cell
    }
    K = 1;
    while (K < 62 && (1LL << K) <= cb) ++K;
    zbase = 0;
    long long zabs = 0;
    if (zmin <= zmax) {
        zbase = (zmin + zmax) >> 1;
        zabs = (zmax - zbase) > (zbase - zmin) ? (zmax - zbase) : (zbase - zmin);
    }
    packed = (K <= 40 && cb * zabs < (1LL << (62 - K))) ? 1 : 0;
}

DNNI_HD unsigned long long span_word(int z, long long zbase, int K) {
    return ((unsigned long long)((long long)z - zbase) << K) + 1ull;
}

DNNI_HD void decode_span_word(unsigned long long w, int K, long long zbase, long long& Z, long long& C) {
    const long long cb = (long long)(w & ((1ull << K) - 1ull));
    const long long zrel = ((long long)(w - (unsigned long long)cb)) >> K;
    Z = zrel + cb * zbase;
    C = cb;
}

constexpr int kWinMaxBins = 1536;
constexpr int kWinMaxRows = 256;
constexpr int kWinMaxPts = 2560;
constexpr size_t kDenseSmem = sizeof(int4) * kWinMaxPts + sizeof(int) * (2 * kWinMaxBins + 1);


}  // namespace dnni
