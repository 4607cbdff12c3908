// dnni_kernels.cuh -- sm_100a kernels of the discrete natural-neighbour
// interpolation hot path (one work package per launch sequence).
//
// Replaces, per work package:
//   nni.cpp:722-790 renderInputPoints / nni.cpp:171-230 drawPlane (the GL
//     depth-tested site planes that leave each pixel's nearest site in the
//     colour buffer)                       -> k_bin_* + k_nearest
//   nni.cpp:794-820 performNNIQueries / nni.cpp:483-534 makeBlocks and
//     cuda_nni.cu:407-488 calcNNI (query planes OR-blended into bit masks,
//     then per-pixel int32 atomics)        -> k_scatter_spans + k_final stencil
//   cuda_nni.cu:491-503 divide, cuda_nni.cu:399-402 zeroValues
//                                          -> k_rowscan + k_final
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
    int32_t pad;
    BinGrid bg;
};

struct Scalars {
    int32_t bbox[6];             // min/max of x-ox, y-oy, z
    int32_t err;
    int32_t packed;              // decided after the nearest-site pass
    int32_t kbits;
    int32_t nfar;                // far worklist length
    int32_t pad2;
    int32_t pad;
    long long zbase;
    int32_t max_r2[kStatSlots];
    unsigned long long big_pixels[kStatSlots];
    unsigned long long spans[kStatSlots];
    unsigned long long nodata[kStatSlots];
};

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------

DNNI_HD int isqrt_i32(int v) {
    // floor(sqrt(v)) for 0 <= v < 2^31: float estimate, exact integer fix-up
    int s = (int)sqrtf((float)v);
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
};

DNNI_HD void consider(Best& b, const int4 p, int q, int px, int py) {
    const int dx = p.x - px, dy = p.y - py;      // |p.x|, |px| < 2^30
    const long long d2 = (long long)dx * dx + (long long)dy * dy;
    const uint32_t g = (uint32_t)p.w;
    if (d2 < b.d2 || (d2 == b.d2 && (g < b.gid || (g == b.gid && p.z < b.z)))) {
        b.d2 = d2;
        b.gid = g;
        b.z = p.z;
        b.idx = q;
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
    Best32 b{~0ull, INT_MAX, -1};
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

// Window of the 32 x 8 pixel tile whose first pixel is raster (i0, j0).
constexpr int kTileX = 32, kTileY = 8;
DNNI_HD void tile_window(const TileParams& t, int i0, int j0, int& wx0, int& wy0, int& wnx, int& wny) {
    const BinGrid& g = t.bg;
    const int i1 = (i0 + kTileX - 1 < t.rw - 1) ? i0 + kTileX - 1 : t.rw - 1;
    const int j1 = (j0 + kTileY - 1 < t.rh - 1) ? j0 + kTileY - 1 : t.rh - 1;
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

// A first bound from the nearest non-empty block map: the points of the bin
// of block `nb` (in bmask order) whose box is closest to the pixel.
DNNI_HD void seed_from_block(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                             const uint64_t* __restrict__ bmask, int64_t nb, int px, int py, Best& b) {
    const long long bs = g.bs, u1 = bs * kBinsPerBlockEdge, u2 = bs * kBinsPerSuperEdge;
    const int64_t sidx = nb >> 6;
    const int m = (int)(nb & 63);
    const long long BX0 = g.gx0 + (long long)(sidx % g.n2x) * u2 + (long long)(m & 7) * u1;
    const long long BY0 = g.gy0 + (long long)(sidx / g.n2x) * u2 + (long long)(m >> 3) * u1;
    uint64_t bm = DNNI_LDG(&bmask[nb]);
    long long qlb = LLONG_MAX;
    int q_idx = 0;
    while (bm) {
        const int l = ffs64(bm);
        bm &= bm - 1;
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

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

__global__ void k_init_scalars(Scalars* sc) {
    const int l = threadIdx.x;
    if (l == 0) {
        sc->bbox[0] = INT_MAX; sc->bbox[1] = INT_MIN;
        sc->bbox[2] = INT_MAX; sc->bbox[3] = INT_MIN;
        sc->bbox[4] = INT_MAX; sc->bbox[5] = INT_MIN;
        sc->err = 0; sc->packed = 0; sc->kbits = 0; sc->zbase = 0;
        sc->nfar = 0;
    }
    if (l < kStatSlots) {
        sc->max_r2[l] = -1; sc->big_pixels[l] = 0; sc->spans[l] = 0; sc->nodata[l] = 0;
    }
}

// Bounding box of the points relative to the WP origin, with range checks.
__global__ void k_bbox(const int32_t* __restrict__ xyz, int64_t n, int32_t ox, int32_t oy, Scalars* sc) {
    int mnx = INT_MAX, mxx = INT_MIN, mny = INT_MAX, mxy = INT_MIN, mnz = INT_MAX, mxz = INT_MIN;
    unsigned bad = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const long long x = (long long)xyz[3 * i] - ox, y = (long long)xyz[3 * i + 1] - oy;
        const long long z = xyz[3 * i + 2];
        if (x <= -kCoordLimit || x >= kCoordLimit || y <= -kCoordLimit || y >= kCoordLimit ||
            z <= -kCoordLimit || z >= kCoordLimit) {
            bad = 1;
            continue;
        }
        mnx = min(mnx, (int)x); mxx = max(mxx, (int)x);
        mny = min(mny, (int)y); mxy = max(mxy, (int)y);
        mnz = min(mnz, (int)z); mxz = max(mxz, (int)z);
    }
    mnx = __reduce_min_sync(0xffffffffu, mnx); mxx = __reduce_max_sync(0xffffffffu, mxx);
    mny = __reduce_min_sync(0xffffffffu, mny); mxy = __reduce_max_sync(0xffffffffu, mxy);
    mnz = __reduce_min_sync(0xffffffffu, mnz); mxz = __reduce_max_sync(0xffffffffu, mxz);
    bad = __reduce_or_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&sc->bbox[0], mnx); atomicMax(&sc->bbox[1], mxx);
        atomicMin(&sc->bbox[2], mny); atomicMax(&sc->bbox[3], mxy);
        atomicMin(&sc->bbox[4], mnz); atomicMax(&sc->bbox[5], mxz);
        if (bad) atomicOr(&sc->err, kErrRange);
    }
}

DNNI_HD int64_t point_bin(const BinGrid& g, int xr, int yr) {
    int bx = (int)((uint32_t)(xr - g.gx0) / (uint32_t)g.bs);
    int by = (int)((uint32_t)(yr - g.gy0) / (uint32_t)g.bs);
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    return bin_id(g, bx, by);
}

// Counting-sort pass 1: per-bin counts; each point keeps its rank in its bin.
__global__ void k_bin_count(const int32_t* __restrict__ xyz, int64_t n, int32_t ox, int32_t oy, BinGrid g,
                            int* __restrict__ cnt, int* __restrict__ rank) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int xr = rel_coord(xyz[3 * i], ox), yr = rel_coord(xyz[3 * i + 1], oy);
        rank[i] = atomicAdd(&cnt[point_bin(g, xr, yr)], 1);
    }
}

// Counting-sort pass 3: place every point at start[bin] + rank.
__global__ void k_bin_scatter(const int32_t* __restrict__ xyz, const uint32_t* __restrict__ gid, int64_t n,
                              int32_t ox, int32_t oy, BinGrid g, const int* __restrict__ start,
                              const int* __restrict__ rank, int4* __restrict__ sorted) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int xr = rel_coord(xyz[3 * i], ox), yr = rel_coord(xyz[3 * i + 1], oy);
        const int pos = start[point_bin(g, xr, yr)] + rank[i];
        sorted[pos] = make_int4(xr, yr, xyz[3 * i + 2], (int)(gid ? gid[i] : (uint32_t)i));
    }
}

// Occupancy masks from the bin starts: one warp per block (bit l = bin l of
// the block is non-empty), then one warp per superblock (bit m = block m is).
__global__ void __launch_bounds__(256) k_block_masks(const int* __restrict__ start, int64_t nblocks,
                                                     uint64_t* __restrict__ bmask) {
    const int64_t blk = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (blk >= nblocks) return;
    const int* s = start + (blk << 6);
    const bool lo = s[lane + 1] != s[lane];
    const bool hi = s[lane + 33] != s[lane + 32];
    const unsigned mlo = __ballot_sync(0xffffffffu, lo), mhi = __ballot_sync(0xffffffffu, hi);
    if (lane == 0) bmask[blk] = (uint64_t)mlo | ((uint64_t)mhi << 32);
}

__global__ void __launch_bounds__(256) k_super_masks(const uint64_t* __restrict__ bmask, int64_t nsuper,
                                                     uint64_t* __restrict__ smask) {
    const int64_t sidx = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (sidx >= nsuper) return;
    const uint64_t* b = bmask + (sidx << 6);
    const unsigned mlo = __ballot_sync(0xffffffffu, b[lane] != 0), mhi = __ballot_sync(0xffffffffu, b[lane + 32] != 0);
    if (lane == 0) smask[sidx] = (uint64_t)mlo | ((uint64_t)mhi << 32);
}

// Nearest non-empty block map, exact in block-centre distance: per block
// row the nearest non-empty column (forward and backward sweep), then per
// block the best row found by walking rows outward until the row offset
// alone exceeds the best distance.  near[cy * n1x + cx] = bmask index of the
// chosen block, -1 when the grid has no points.
__global__ void k_block_rows(BinGrid g, const uint64_t* __restrict__ bmask, int* __restrict__ rownear) {
    const int n1x = g.nbx >> 3, n1y = g.nby >> 3;
    const int cy = blockIdx.x * blockDim.x + threadIdx.x;
    if (cy >= n1y) return;
    int* row = rownear + (int64_t)cy * n1x;
    int last = -1;
    for (int cx = 0; cx < n1x; ++cx) {
        if (bmask[block_index(g, cx, cy)]) last = cx;
        row[cx] = last;
    }
    last = -1;
    for (int cx = n1x - 1; cx >= 0; --cx) {
        if (bmask[block_index(g, cx, cy)]) last = cx;
        const int l = row[cx];
        if (last >= 0 && (l < 0 || last - cx < cx - l)) row[cx] = last;
    }
}

__global__ void k_block_near(BinGrid g, const int* __restrict__ rownear, int64_t* __restrict__ near) {
    const int n1x = g.nbx >> 3, n1y = g.nby >> 3;
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= (int64_t)n1x * n1y) return;
    const int cx = (int)(k % n1x), cy = (int)(k / n1x);
    long long best = LLONG_MAX;
    int bxn = -1, byn = -1;
    for (int d = 0; d < n1y; ++d) {
        if ((long long)d * d > best) break;
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            if (d == 0 && sgn > 0) continue;
            const int y = cy + sgn * d;
            if (y < 0 || y >= n1y) continue;
            const int x = rownear[(int64_t)y * n1x + cx];
            if (x < 0) continue;
            const long long v = (long long)(x - cx) * (x - cx) + (long long)d * d;
            if (v < best) { best = v; bxn = x; byn = y; }
        }
    }
    near[k] = bxn >= 0 ? block_index(g, bxn, byn) : -1;
}

// ---- exclusive scan of the bin counts (three passes, 4096 items per block) ----

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;

// Exclusive block-wide sum over 256 threads (8 warps).  tid is the thread's
// linear index in the block (warps are formed from linear indices), so the
// helper works for any block shape with 256 threads.
template <typename T>
__device__ __forceinline__ T block_exclusive_sum(T v, T* wsum, T& total, int tid) {
    const int lane = tid & 31, warp = tid >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < 8 ? wsum[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) wsum[lane] = w;
    }
    __syncthreads();
    total = wsum[7];
    const T excl = x - v + (warp ? wsum[warp - 1] : T(0));
    __syncthreads();
    return excl;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_partial(const int* __restrict__ cnt, int64_t m, int* __restrict__ bsum) {
    __shared__ int wsum[8];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t idx = base + k * kScanThreads + threadIdx.x;
        if (idx < m) s += cnt[idx];
    }
    int total;
    block_exclusive_sum(s, wsum, total, (int)threadIdx.x);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_bsum(int* __restrict__ bsum, int nb) {
    __shared__ int wsum[32];
    const int per = (nb + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    int s = 0;
    for (int k = 0; k < per; ++k) if (b0 + k < nb) s += bsum[b0 + k];
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
        if (b0 + k < nb) { const int v = bsum[b0 + k]; bsum[b0 + k] = run; run += v; }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_final(const int* __restrict__ cnt, int64_t m,
                                                             const int* __restrict__ bsum, int* __restrict__ start) {
    __shared__ int tile[kScanTile];
    __shared__ int wsum[8];
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int li = k * kScanThreads + threadIdx.x;
        const int64_t idx = base + li;
        tile[li] = idx < m ? cnt[idx] : 0;
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
        if (idx < m) start[idx] = tile[li];
    }
}

// ---- nearest site per raster pixel ----

constexpr int kWinMaxBins = 2048;
constexpr int kWinMaxRows = 256;
constexpr int kWinMaxPts = 3072;
constexpr size_t kDenseSmem = sizeof(int4) * kWinMaxPts + sizeof(int) * (2 * kWinMaxBins + 1);

// Records a settled pixel: its record and site.
__device__ __forceinline__ void settle_pixel(const TileParams& t, int i, int j, const Best& b, int2* __restrict__ pix,
                                             uint32_t* __restrict__ site) {
    const int R2 = r2_of(b.d2, (long long)t.cs * t.cs, t.r2cap);
    const int64_t o = (int64_t)j * t.rw + i;
    pix[o] = make_int2(b.z, R2);
    if (site) site[o] = b.gid;
}

__device__ __forceinline__ void warp_stats(const TileParams& t, int R2, Scalars* __restrict__ sc, int slot) {
    const int rs2 = t.rs * t.rs;
    const unsigned big = (R2 > rs2) ? 1u : 0u;
    const unsigned sp = big ? 2u * (unsigned)isqrt_i32(R2) + 1u : 0u;
    const unsigned nbig = __reduce_add_sync(0xffffffffu, big);
    const unsigned nsp = __reduce_add_sync(0xffffffffu, sp);
    const int mx = __reduce_max_sync(0xffffffffu, R2);
    if ((threadIdx.x & 31) == 0) {
        slot &= kStatSlots - 1;
        if (nbig) {
            atomicAdd(&sc->big_pixels[slot], (unsigned long long)nbig);
            atomicAdd(&sc->spans[slot], (unsigned long long)nsp);
        }
        if (mx >= 0) atomicMax(&sc->max_r2[slot], mx);
    }
}

// Dense pass.  One CTA per 32 x 8 pixel tile (blockDim 256, warp = one
// pixel row of the tile): the tile's bin window (bin rings of every pixel)
// is staged in shared memory and the rings are searched there; windows too
// large for shared memory use the global arrays.  Pixels the rings do not
// settle go to the far worklist (sc->nfar slots, in groups of 32), each with
// its best site so far.  With no points every pixel is settled as "no site".
__global__ void __launch_bounds__(256, 3) k_near_dense(TileParams t, const int4* __restrict__ pts,
                                                    const int* __restrict__ start, int2* __restrict__ pix,
                                                    uint32_t* __restrict__ site, int2* __restrict__ far,
                                                    Scalars* __restrict__ sc) {
    extern __shared__ int4 smem[];
    int4* s_pts = smem;
    int* s_lstart = (int*)(smem + kWinMaxPts);
    int* s_gstart = s_lstart + kWinMaxBins + 1;
    __shared__ int s_rowbase[kWinMaxRows];
    __shared__ int s_total;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    const int i0 = blockIdx.x * kTileX, j0 = blockIdx.y * kTileY;
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const bool valid = i < t.rw && j < t.rh;
    const BinGrid& g = t.bg;
    int wx0 = 0, wy0 = 0, wnx = 0, wny = 0;
    bool staged = false;
    if (t.npts > 0) {
        tile_window(t, i0, j0, wx0, wy0, wnx, wny);
        const int nwb = wnx * wny;
        if (nwb <= kWinMaxBins && wny <= kWinMaxRows) {
            // per-bin counts -> local starts: warp w takes window rows w, w+8,
            // ...; lanes take columns, with a warp scan along the row
            const int warp = tid >> 5, lane = tid & 31;
            for (int r = warp; r < wny; r += 8) {
                int rowsum = 0;
                for (int c0 = 0; c0 < wnx; c0 += 32) {
                    const int c = c0 + lane;
                    int cnt = 0;
                    if (c < wnx) {
                        const int64_t id = bin_id(g, wx0 + c, wy0 + r);
                        const int gs = __ldg(&start[id]);
                        cnt = __ldg(&start[id + 1]) - gs;
                        s_gstart[r * wnx + c] = gs;
                    }
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
            staged = s_total <= kWinMaxPts;
            if (staged) {
                // copy the window's points run by run: the bins of one window
                // row inside one block are consecutive in both layouts; one
                // warp per run, lanes striding over its points
                const int cb0 = wx0 >> 3, cb1 = (wx0 + wnx - 1) >> 3;
                const int nseg = cb1 - cb0 + 1, nrun = nseg * wny;
                const int warp = tid >> 5, lane = tid & 31;
                for (int run = warp; run < nrun; run += 8) {
                    const int r = run / nseg, sg = run - r * nseg;
                    const int xa = (cb0 + sg) * 8 > wx0 ? (cb0 + sg) * 8 : wx0;
                    const int xb = (cb0 + sg) * 8 + 7 < wx0 + wnx - 1 ? (cb0 + sg) * 8 + 7 : wx0 + wnx - 1;
                    const int lk0 = r * wnx + (xa - wx0), lk1 = r * wnx + (xb - wx0);
                    const int l0 = s_lstart[lk0], cntp = s_lstart[lk1 + 1] - l0, g0 = s_gstart[lk0];
                    for (int q = lane; q < cntp; q += 32) s_pts[l0 + q] = __ldg(&pts[g0 + q]);
                }
            }
            __syncthreads();
        }
    }
    int R2 = -1;
    bool far_pixel = false;
    Best b{LLONG_MAX, 0xFFFFFFFFu, INT_MAX, -1};
    if (valid) {
        if (t.npts > 0) {
            const int px = (t.rx0 + i) * t.cs, py = (t.ry0 + j) * t.cs;
            bool done;
            if (staged) {
                const BinWindow w{wx0, wy0, wnx, wny, s_lstart, s_gstart, s_pts};
                done = window_fits32(g, w) ? search_window_fast32(g, w, px, py, b) : search_window_fast(g, w, px, py, b);
                if (!done) b.idx = window_global_index(w, b.idx);
            } else {
                done = search_bins(g, pts, start, px, py, b);
            }
            if (done) {
                settle_pixel(t, i, j, b, pix, site);
                R2 = r2_of(b.d2, (long long)t.cs * t.cs, t.r2cap);
            } else {
                far_pixel = true;
            }
        } else {
            const int64_t o = (int64_t)j * t.rw + i;
            pix[o] = make_int2(0, -1);
            if (site) site[o] = 0xFFFFFFFFu;
        }
    }
    // worklist: a warp with any unsettled pixel appends its whole row of 32
    // slots as one group (settled or absent pixels as x = -1), so that a far
    // warp later takes 32 neighbouring pixels
    const unsigned mfar = __ballot_sync(0xffffffffu, far_pixel);
    const int lane = threadIdx.x;
    if (mfar) {
        int base = 0;
        if (lane == 0) base = atomicAdd(&sc->nfar, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        far[base + lane] = far_pixel ? make_int2(j * t.rw + i, b.idx) : make_int2(-1, -1);
    }
    warp_stats(t, R2, sc, blockIdx.x + blockIdx.y * 7 + threadIdx.y);
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

// Warp-cooperative exact search for the 32 pixels of one worklist group
// (neighbouring pixels of one tile row; inactive lanes have act = false).
// The warp walks the superblocks of the union of the lanes' bound boxes
// (rows outward from the group's centre) and, uniformly, the set bits of
// the occupancy masks; each lane tests every cell's box bound against its
// own best, a cell is entered when any lane needs it, and every point of an
// entered bin is loaded once and considered by the lanes that need the bin.
// Complete for each active lane whose b holds a real site on entry, by the
// same argument as search_disc.
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

// Warp-cooperative exact search for the 32 pixels of one worklist group
// (neighbouring pixels of one tile row; inactive lanes have act = false).
// The warp walks the superblocks of the union of the lanes' bound boxes
// (rows outward from the group's centre).  Inside a superblock, candidate
// blocks are the non-empty ones inside some lane's bound box (an OR of the
// lanes' box masks); each candidate gets every lane's exact box test and is
// entered when any lane needs it; bins likewise; every point of an entered
// bin is loaded once and considered by the lanes that need the bin.  All
// control flow is uniform across the warp.  Complete for each active lane
// whose b holds a real site on entry, by the same argument as search_disc.
__device__ void search_disc_warp(const BinGrid& g, const int4* __restrict__ pts, const int* __restrict__ start,
                                 const uint64_t* __restrict__ bmask, const uint64_t* __restrict__ smask, bool act,
                                 int px, int py, Best& b) {
    const unsigned full = 0xffffffffu;
    const long long gx0 = g.gx0, gy0 = g.gy0, bs = g.bs;
    const long long u1 = bs * kBinsPerBlockEdge, u2 = bs * kBinsPerSuperEdge;
    const float inv_u1 = 1.0f / (float)u1, inv_bs = 1.0f / (float)bs;
    long long reach = act ? reach_of(b.d2) : 0;
    const long long xlo = warp_min64(act ? px - reach : LLONG_MAX), xhi = warp_max64(act ? px + reach : LLONG_MIN);
    const long long ylo = warp_min64(act ? py - reach : LLONG_MAX), yhi = warp_max64(act ? py + reach : LLONG_MIN);
    if (xlo > xhi) return;   // no active lane
    int sx0, sx1, sy0, sy1;
    cell_range((xlo + xhi) / 2, (xhi - xlo) / 2 + 1, gx0, u2, g.n2x, sx0, sx1);
    cell_range((ylo + yhi) / 2, (yhi - ylo) / 2 + 1, gy0, u2, g.n2y, sy0, sy1);
    if (sx0 > sx1 || sy0 > sy1) return;
    // 32-bit tests are exact while every active lane's bound is below 2^31
    const bool small = __all_sync(full, !act || b.d2 < (1LL << 31));
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
            // candidate blocks: inside some needing lane's bound box
            reach = act ? reach_of(b.d2) : 0;
            uint64_t lm = 0;
            if (need_s) {
                int a0, a1, b0, b1;
                cell_span8(px, reach, SX0, inv_u1, a0, a1);
                cell_span8(py, reach, SY0, inv_u1, b0, b1);
                lm = box_mask8(a0, a1, b0, b1);
            }
            uint64_t cand = sm & warp_or64(lm);
            // pixel relative to the superblock (in range whenever the lane needs it)
            const long long rxl = px - SX0, ryl = py - SY0;
            const int rx = (int)(rxl < -(1LL << 30) ? -(1LL << 30) : (rxl > (1LL << 30) ? (1LL << 30) : rxl));
            const int ry = (int)(ryl < -(1LL << 30) ? -(1LL << 30) : (ryl > (1LL << 30) ? (1LL << 30) : ryl));
            while (cand) {
                const int m = ffs64(cand);
                cand &= cand - 1;
                const int bx0 = (m & 7) * (int)u1, by0 = (m >> 3) * (int)u1;
                bool need_b;
                if (small) need_b = act && (long long)box_lb32(rx, ry, bx0, bx0 + (int)u1 - 1, by0, by0 + (int)u1 - 1) <= b.d2;
                else need_b = act && box_lb(px, py, SX0 + bx0, SX0 + bx0 + u1 - 1, SY0 + by0, SY0 + by0 + u1 - 1) <= b.d2;
                if (!__any_sync(full, need_b)) continue;
                const int64_t blk = ((int64_t)sidx << 6) + m;
                const uint64_t bm = __ldg(&bmask[blk]);
                uint64_t lq = 0;
                if (need_b) {
                    int a0, a1, b0, b1;
                    const long long rr = reach_of(b.d2);
                    cell_span8(px, rr, SX0 + bx0, inv_bs, a0, a1);
                    cell_span8(py, rr, SY0 + by0, inv_bs, b0, b1);
                    lq = box_mask8(a0, a1, b0, b1);
                }
                uint64_t qc = bm & warp_or64(lq);
                while (qc) {
                    const int l = ffs64(qc);
                    qc &= qc - 1;
                    const int qx0 = bx0 + (l & 7) * (int)bs, qy0 = by0 + (l >> 3) * (int)bs;
                    bool need;
                    if (small) need = act && (long long)box_lb32(rx, ry, qx0, qx0 + (int)bs - 1, qy0, qy0 + (int)bs - 1) <= b.d2;
                    else need = act && box_lb(px, py, SX0 + qx0, SX0 + qx0 + bs - 1, SY0 + qy0, SY0 + qy0 + bs - 1) <= b.d2;
                    if (!__any_sync(full, need)) continue;
                    const int64_t id = (blk << 6) + l;
                    const int s0 = __ldg(&start[id]), e0 = __ldg(&start[id + 1]);
                    for (int q = s0; q < e0; ++q) {
                        const int4 p = __ldg(&pts[q]);
                        if (need) consider(b, p, q, px, py);
                    }
                }
            }
        }
    }
}

// Far pass over the worklist: one warp per group of 32 slots (grid-stride).
// Each lane seeds its bound (its best site so far, else the nearest
// non-empty block's closest bin, else the nearest non-empty superblock) and
// the warp searches the union of the bound discs cooperatively.
__global__ void __launch_bounds__(256, 3) k_near_far(TileParams t, const int4* __restrict__ pts,
                                                     const int* __restrict__ start, const uint64_t* __restrict__ bmask,
                                                     const uint64_t* __restrict__ smask,
                                                     const int64_t* __restrict__ near, const int2* __restrict__ far,
                                                     int2* __restrict__ pix, uint32_t* __restrict__ site,
                                                     Scalars* __restrict__ sc) {
    const int count = sc->nfar;
    const int lane = threadIdx.x & 31;
    const int n1x = t.bg.nbx >> 3;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < count; base += gridDim.x * blockDim.x) {
        const int2 item = far[base + lane];
        const bool act = item.x >= 0;
        int i = 0, j = 0, px = 0, py = 0;
        Best b{LLONG_MAX, 0xFFFFFFFFu, INT_MAX, -1};
        if (act) {
            i = item.x % t.rw;
            j = item.x / t.rw;
            px = (t.rx0 + i) * t.cs;
            py = (t.ry0 + j) * t.cs;
            if (item.y >= 0) consider(b, __ldg(&pts[item.y]), item.y, px, py);
            int bx = udiv32((long long)px - t.bg.gx0, t.bg.bs), by = udiv32((long long)py - t.bg.gy0, t.bg.bs);
            bx = bx < t.bg.nbx - 1 ? bx : t.bg.nbx - 1;
            by = by < t.bg.nby - 1 ? by : t.bg.nby - 1;
            const int64_t nb = __ldg(&near[(int64_t)(by >> 3) * n1x + (bx >> 3)]);
            if (nb >= 0) seed_from_block(t.bg, pts, start, bmask, nb, px, py, b);
            if (b.d2 == LLONG_MAX) seed_from_superblocks(t.bg, pts, start, bmask, smask, px, py, b);
        }
        search_disc_warp(t.bg, pts, start, bmask, smask, act, px, py, b);
        int R2 = -1;
        if (act) {
            settle_pixel(t, i, j, b, pix, site);
            R2 = r2_of(b.d2, (long long)t.cs * t.cs, t.r2cap);
        }
        warp_stats(t, R2, sc, blockIdx.x * 3 + (threadIdx.x >> 5));
    }
}

// Picks the accumulator form for the span path.  The per-cell count from big
// discs is at most the lattice points of a disc of radius^2 max_r2, (2r+1)^2,
// and at most the raster size; z enters relative to zbase (the mid-range),
// so |Zrel| <= C * zabs.  Packed: word = (Zrel << K) + C with C < 2^K and
// |Zrel| < 2^(62-K); otherwise separate int64 Z and int32 C.
DNNI_HD void decide_packing(int max_r2, long long npix, long long zmin, long long zmax, int& packed, int& K,
                            long long& zbase) {
    long long cb = 0;
    if (max_r2 >= 0) {
        const long long r = isqrt_i32(max_r2);
        cb = (2 * r + 1) * (2 * r + 1);
        if (cb > npix) cb = npix;
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

__global__ void k_decide(Scalars* sc, long long npix) {
    const int l = threadIdx.x;
    int mx = sc->max_r2[l];
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (l == 0) {
        int packed, K;
        long long zbase;
        decide_packing(mx, npix, sc->bbox[4], sc->bbox[5], packed, K, zbase);
        sc->packed = packed;
        sc->kbits = K;
        sc->zbase = zbase;
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

// Span path: every pixel with R2 > rs^2 adds its disc as row spans
// (+v at the first cell, -v after the last) to the per-row difference array.
// Warp = 32 consecutive pixels of one raster row, so one iteration's markers
// fall on two rows near each other in memory.
__global__ void __launch_bounds__(256) k_scatter_spans(TileParams t, const int2* __restrict__ pix,
                                                       const Scalars* __restrict__ sc,
                                                       unsigned long long* __restrict__ D, int* __restrict__ Dc) {
    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 8 + threadIdx.y;
    int R2 = -1, z = 0;
    if (i < t.rw && j < t.rh) {
        const int2 r = pix[(int64_t)j * t.rw + i];
        z = r.x;
        R2 = r.y;
    }
    const bool big = R2 > t.rs * t.rs;
    if (!__any_sync(0xffffffffu, big)) return;
    const int r = big ? isqrt_i32(R2) : -1;
    const int rmax = __reduce_max_sync(0xffffffffu, r);
    const bool packed = sc->packed != 0;
    const int K = sc->kbits;
    const unsigned long long v = span_word(z, sc->zbase, K);
    const int px = t.rx0 + i, py = t.ry0 + j;
    int w = r;
    for (int dy = 0; dy <= rmax; ++dy) {
        if (dy <= r) {
            const long long t2 = (long long)R2 - (long long)dy * dy;
            while ((long long)w * w > t2) --w;
            emit_span(py + dy, px - w, px + w, t.ncols, t.nrows, packed, v, z, D, Dc);
            if (dy) emit_span(py - dy, px - w, px + w, t.ncols, t.nrows, packed, v, z, D, Dc);
        }
    }
}

// In-place inclusive prefix along each grid row.  which: 0 = the 64-bit
// words (always), 1 = the int32 counts (only when not packed).
template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_rowscan(T* __restrict__ D, int ncols, const Scalars* __restrict__ sc,
                                                          int which) {
    if (which == 1 && sc->packed) return;
    __shared__ T wsum[8];
    T* row = D + (int64_t)blockIdx.x * ncols;
    T carry = 0;
    for (int base = 0; base < ncols; base += kScanThreads * 4) {
        const int idx = base + threadIdx.x * 4;
        T v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) v[k] = (idx + k < ncols) ? row[idx + k] : T(0);
        v[1] += v[0]; v[2] += v[1]; v[3] += v[2];
        T total;
        const T excl = block_exclusive_sum(v[3], wsum, total, (int)threadIdx.x) + carry;
#pragma unroll
        for (int k = 0; k < 4; ++k) if (idx + k < ncols) row[idx + k] = v[k] + excl;
        carry += total;
    }
}

__device__ __forceinline__ float finalize_height(long long Z, long long C, double zs, double zo, float nodata) {
    if (C <= 0) return nodata;
    const double q = __ddiv_rn(__ll2double_rn(Z), __ll2double_rn(C));
    return __double2float_rn(__dadd_rn(__dmul_rn(q, zs), zo));
}

// Stencil path + finalize: each cell gathers the small discs (R2 <= H^2) of
// the pixels within H, adds the prefix-summed span words, and divides.
template <int H>
__global__ void __launch_bounds__(512) k_final(TileParams t, const int2* __restrict__ pix,
                                               Scalars* __restrict__ sc,
                                               const unsigned long long* __restrict__ S,
                                               const int* __restrict__ Sc, float* __restrict__ h) {
    constexpr int TX = 32, TY = 16, SW = TX + 2 * H, SH = TY + 2 * H;
    __shared__ int2 tile[SH][SW];
    const int cx0 = blockIdx.x * TX, cy0 = blockIdx.y * TY;
    for (int idx = threadIdx.y * TX + threadIdx.x; idx < SW * SH; idx += TX * TY) {
        const int ly = idx / SW, lx = idx - ly * SW;
        const int rxi = cx0 - H + lx - t.rx0, ryi = cy0 - H + ly - t.ry0;
        int2 v = make_int2(0, -1);
        if (rxi >= 0 && rxi < t.rw && ryi >= 0 && ryi < t.rh) v = pix[(int64_t)ryi * t.rw + rxi];
        tile[ly][lx] = v;
    }
    __syncthreads();
    const int qx = cx0 + threadIdx.x, qy = cy0 + threadIdx.y;
    const bool in = qx < t.ncols && qy < t.nrows;
    long long Z = 0, C = 0;
#pragma unroll
    for (int dy = -H; dy <= H; ++dy)
#pragma unroll
        for (int dx = -H; dx <= H; ++dx) {
            if (dx * dx + dy * dy > H * H) continue;
            const int2 p = tile[threadIdx.y + H + dy][threadIdx.x + H + dx];
            if (p.y >= dx * dx + dy * dy && p.y <= H * H) { Z += p.x; C += 1; }
        }
    unsigned nod = 0;
    if (in) {
        const int64_t q = (int64_t)qy * t.ncols + qx;
        const unsigned long long w = S[q];
        if (sc->packed) {
            long long zb, cb;
            decode_span_word(w, sc->kbits, sc->zbase, zb, cb);
            Z += zb;
            C += cb;
        } else {
            Z += (long long)w;
            C += Sc[q];
        }
        const float hv = finalize_height(Z, C, t.z_scale, t.z_offset, t.nodata);
        h[q] = hv;
        nod = C <= 0 ? 1u : 0u;
    }
    nod = __reduce_add_sync(0xffffffffu, nod);
    if ((threadIdx.x & 31) == 0 && nod) {
        const int slot = (blockIdx.x + blockIdx.y * 5 + threadIdx.y) & (kStatSlots - 1);
        atomicAdd(&sc->nodata[slot], (unsigned long long)nod);
    }
}

}  // namespace dnni
