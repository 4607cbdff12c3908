// dnni_plan.h -- host-side planning of one work package: validation of the
// work package and the choice of the search-bin grid.  Shared by the engine
// and by the host build of the kernels that the test suite checks.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/dnni.h"
#include "dnni_search.cuh"

namespace dnni {

constexpr int64_t kMaxBins = 1LL << 26;
constexpr int kMaxSide = 32767;

// Validates the work package (nni::WorkPackage, nni.h:66-70, in LAS units)
// and fills the geometry part of t.  On failure returns the status and sets
// *msg to a static description.
inline dnni_status plan_geometry(const dnni_workpackage* wp, int64_t n, int small_radius, TileParams& t,
                                 const char** msg) {
    *msg = "";
    if (!wp) { *msg = "work package is NULL"; return DNNI_E_INVAL; }
    if (wp->ncols <= 0 || wp->nrows <= 0 || wp->ncols > kMaxSide || wp->nrows > kMaxSide) {
        *msg = "grid sides must be in [1, 32767]";
        return DNNI_E_INVAL;
    }
    if (wp->cell_size <= 0) { *msg = "cell_size must be positive"; return DNNI_E_INVAL; }
    if (n < 0 || n > (int64_t)INT32_MAX - 1) { *msg = "point count out of range"; return DNNI_E_INVAL; }
    int32_t rx0 = wp->raster_x0, ry0 = wp->raster_y0, rx1 = wp->raster_x1, ry1 = wp->raster_y1;
    if (rx0 == 0 && ry0 == 0 && rx1 == 0 && ry1 == 0) {
        rx1 = wp->ncols;
        ry1 = wp->nrows;
    }
    if (rx1 <= rx0 || ry1 <= ry0) { *msg = "empty raster"; return DNNI_E_INVAL; }
    const int64_t ex = (int64_t)std::max(rx1, wp->ncols) - std::min(rx0, 0);
    const int64_t ey = (int64_t)std::max(ry1, wp->nrows) - std::min(ry0, 0);
    if (ex > kMaxSide || ey > kMaxSide) { *msg = "grid+raster extent exceeds 32767 cells"; return DNNI_E_INVAL; }
    const int64_t cs = wp->cell_size;
    const int64_t corners[6] = {rx0 * cs, (int64_t)(rx1 - 1) * cs, ry0 * cs, (int64_t)(ry1 - 1) * cs,
                                (int64_t)(wp->ncols - 1) * cs, (int64_t)(wp->nrows - 1) * cs};
    for (int64_t v : corners)
        if (v <= -kCoordLimit || v >= kCoordLimit) {
            *msg = "grid or raster lies beyond +-2^30 LAS units of the origin";
            return DNNI_E_RANGE;
        }
    memset(&t, 0, sizeof(t));
    t.ncols = wp->ncols;
    t.nrows = wp->nrows;
    t.cs = wp->cell_size;
    t.ox = wp->origin_x;
    t.oy = wp->origin_y;
    t.rx0 = rx0;
    t.ry0 = ry0;
    t.rw = rx1 - rx0;
    t.rh = ry1 - ry0;
    t.r2cap = (int32_t)(ex * ex + ey * ey);
    t.rs = small_radius;
    t.npts = n;
    t.z_scale = wp->z_scale;
    t.z_offset = wp->z_offset;
    t.nodata = wp->nodata;
    return DNNI_OK;
}

// Search-bin grid over the union of the point bounding box (relative to the
// WP origin; bbox = minx,maxx,miny,maxy,...) and the raster: bins hold about
// bin_target points on average; the grid is padded to whole superblocks.
inline void plan_bins(const int32_t bbox[6], int64_t n, double bin_target, TileParams& t) {
    const int64_t cs = t.cs;
    int64_t xlo = (int64_t)t.rx0 * cs, xhi = (int64_t)(t.rx0 + t.rw - 1) * cs;
    int64_t ylo = (int64_t)t.ry0 * cs, yhi = (int64_t)(t.ry0 + t.rh - 1) * cs;
    if (n > 0 && bbox[0] <= bbox[1]) {
        xlo = std::min<int64_t>(xlo, bbox[0]);
        xhi = std::max<int64_t>(xhi, bbox[1]);
        ylo = std::min<int64_t>(ylo, bbox[2]);
        yhi = std::max<int64_t>(yhi, bbox[3]);
    }
    const int64_t W = xhi - xlo + 1, Hh = yhi - ylo + 1;
    const double target = bin_target > 0 ? bin_target : 4.0;
    const double bsd = std::sqrt(target * (double)W * (double)Hh / (double)std::max<int64_t>(n, 1));
    int64_t bs = (int64_t)std::ceil(bsd);
    if (bs < 1) bs = 1;
    if (bs > (1LL << 24)) bs = 1LL << 24;
    int64_t nbx, nby;
    for (;;) {
        nbx = (W + bs - 1) / bs;
        nby = (Hh + bs - 1) / bs;
        nbx = (nbx + kBinsPerSuperEdge - 1) / kBinsPerSuperEdge * kBinsPerSuperEdge;
        nby = (nby + kBinsPerSuperEdge - 1) / kBinsPerSuperEdge * kBinsPerSuperEdge;
        if (nbx * nby <= kMaxBins || bs >= (1LL << 24)) break;
        bs = bs + bs / 4 + 1;
    }
    t.bg.gx0 = (int32_t)xlo;
    t.bg.gy0 = (int32_t)ylo;
    t.bg.bs = (int32_t)bs;
    t.bg.nbx = (int32_t)nbx;
    t.bg.nby = (int32_t)nby;
    t.bg.n2x = (int32_t)(nbx / kBinsPerSuperEdge);
    t.bg.n2y = (int32_t)(nby / kBinsPerSuperEdge);
    t.bg.nbins = nbx * nby;
}

}  // namespace dnni

#include <vector>

#include "dnni_kernels.cuh"

namespace dnni {

// Host-side plan of a batch: every tile's geometry, bin grid and offsets,
// plus the prefix arrays that map launch indices to tiles.
// Largest launch index (blocks of a kind, far worklist slots) of a batch.
constexpr int64_t kMaxLaunchIndex = INT32_MAX - 1024;

struct HostBatch {
    std::vector<TileParams> tiles;
    std::vector<int> chunk_base{0}, scan_base{0}, row1_base{0}, rt_base{0}, ct_base{0}, grow_base{0}, band_base{0};
    std::vector<int64_t> blk_base{0}, sup_base{0};
    int64_t n_rows = 0;                  // input point rows the tiles reference
    int64_t n_pts = 0, n_bins = 0, n_pix = 0, n_cells = 0, n_far = 0;
    int64_t out_end = 0, site_end = 0;   // extent of the caller's output arrays used
    int64_t cost = 0;
    int rs = 3;                          // stencil radius shared by the batch
    int win_words = kSpanWindowWords;    // shared-memory words of the span window per CTA
    int far_blocks = kFarBlocksDefault;  // far groups: 1 = 8 x 4 pixel blocks, 0 = 32 x 1 rows
    int dense_band = kTileY;             // ring search: pixel rows of a 32-wide band sharing one staged window
    bool too_big = false;                // a launch index or the far worklist would pass int32
};

// Worklist capacity of a tile: every dense warp (32 pixels of a tile row, the
// raster padded to whole 32 x kTileY tiles) may append one group of 32 slots.
inline int64_t far_slots(const TileParams& t) {
    return (int64_t)((t.rw + kTileX - 1) / kTileX * kTileX) * ((t.rh + kTileY - 1) / kTileY * kTileY);
}

// Appends a tile whose geometry and bin grid are set; its point range starts
// at pt_off of the batch's point arrays and its heights at out_off of the
// caller's output (site_off: site map offset or -1).
inline void batch_add(HostBatch& hb, TileParams t, int64_t pt_off, int64_t out_off, int64_t site_off) {
    t.pt_off = pt_off;
    t.srt_off = hb.n_pts;
    t.bin_off = hb.n_bins;
    t.blk_off = hb.blk_base.back();
    t.sup_off = hb.sup_base.back();
    t.pix_off = hb.n_pix;
    t.cell_off = hb.n_cells;
    t.out_off = out_off;
    t.site_off = site_off;
    const int64_t nbins = t.bg.nbins;
    hb.n_bins += nbins + 1;
    hb.blk_base.push_back(t.blk_off + nbins / kBinsPerBlock);
    hb.sup_base.push_back(t.sup_off + nbins / kBinsPerSuper);
    // the int32 prefix arrays saturate; too_big then rejects the batch
    auto add = [&](std::vector<int>& v, int64_t k) {
        const int64_t x = (int64_t)v.back() + k;
        if (x > kMaxLaunchIndex) hb.too_big = true;
        v.push_back((int)std::min<int64_t>(x, kMaxLaunchIndex));
    };
    add(hb.chunk_base, (t.npts + kChunk - 1) / kChunk);
    add(hb.scan_base, (nbins + 1 + kScanTile - 1) / kScanTile);
    add(hb.row1_base, t.npts > 0 ? (t.bg.nby >> 3) : 0);
    add(hb.rt_base, (int64_t)((t.rw + kTileX - 1) / kTileX) * ((t.rh + kTileY - 1) / kTileY));
    add(hb.ct_base, (int64_t)((t.ncols + 31) / 32) * ((t.nrows + 15) / 16));
    add(hb.grow_base, t.nrows);
    add(hb.band_base, (t.nrows + 15) / 16);
    hb.n_rows = std::max<int64_t>(hb.n_rows, pt_off + t.npts);
    hb.n_pts += t.npts;
    hb.n_pix += (int64_t)t.rw * t.rh;
    hb.n_cells += (int64_t)t.ncols * t.nrows;
    hb.n_far += far_slots(t);
    if (hb.n_far > kMaxLaunchIndex) hb.too_big = true;
    hb.out_end = std::max<int64_t>(hb.out_end, out_off + (int64_t)t.ncols * t.nrows);
    if (site_off >= 0) hb.site_end = std::max<int64_t>(hb.site_end, site_off + (int64_t)t.rw * t.rh);
    t.tile_id = (int32_t)hb.tiles.size();
    hb.tiles.push_back(t);
}

// Squared distance transform in one dimension: d[q] = min_p (q - p)^2 + f[p],
// from the lower envelope of the parabolas rooted at each p (Felzenszwalb and
// Huttenlocher, "Distance Transforms of Sampled Functions", Theory of
// Computing 8, 2012).  Empty entries carry kEdtFar, far above any real
// squared distance.  v, z: scratch of n and n + 1 entries.
constexpr double kEdtFar = 1e20;
inline void edt_1d(const double* f, int n, double* d, int* v, double* z) {
    if (n <= 0) return;
    auto meet = [&](int q, int p) { return ((f[q] + (double)q * q) - (f[p] + (double)p * p)) / (2.0 * (q - p)); };
    int k = 0;
    v[0] = 0;
    z[0] = -1e300;
    z[1] = 1e300;
    for (int q = 1; q < n; ++q) {
        double sq = meet(q, v[k]);
        while (sq <= z[k]) {       // z[0] = -inf ends the loop at k = 0
            --k;
            sq = meet(q, v[k]);
        }
        ++k;
        v[k] = q;
        z[k] = sq;
        z[k + 1] = 1e300;
    }
    k = 0;
    for (int q = 0; q < n; ++q) {
        while (z[k + 1] < q) ++k;
        const double dq = (double)q - v[k];
        d[q] = dq * dq + f[v[k]];
    }
}

// Squared distance (in blocks) from every block of an nx x ny grid to the
// nearest occupied one (kEdtFar or more when there is none).
inline std::vector<double> edt_2d(const unsigned char* occ, int nx, int ny) {
    std::vector<double> g((size_t)nx * ny);
    const int m = std::max(nx, ny);
    std::vector<double> f(m), d(m), z(m + 1);
    std::vector<int> v(m);
    for (int x = 0; x < nx; ++x) {
        for (int y = 0; y < ny; ++y) f[y] = occ[(size_t)y * nx + x] ? 0.0 : kEdtFar;
        edt_1d(f.data(), ny, d.data(), v.data(), z.data());
        for (int y = 0; y < ny; ++y) g[(size_t)y * nx + x] = d[y];
    }
    for (int y = 0; y < ny; ++y) {
        for (int x = 0; x < nx; ++x) f[x] = g[(size_t)y * nx + x];
        edt_1d(f.data(), nx, d.data(), v.data(), z.data());
        for (int x = 0; x < nx; ++x) g[(size_t)y * nx + x] = d[x];
    }
    return g;
}

// Byte layout of the device copy of a batch's tables (one upload).
struct TableLayout {
    size_t tiles, chunk, scan, blk, sup, row1, rt, ct, grow, band, total;
    explicit TableLayout(int n) {
        size_t o = 0;
        auto take = [&](size_t b) { const size_t r = o; o = (o + b + 15) & ~(size_t)15; return r; };
        tiles = take(sizeof(TileParams) * n);
        chunk = take(sizeof(int) * (n + 1));
        scan = take(sizeof(int) * (n + 1));
        blk = take(sizeof(int64_t) * (n + 1));
        sup = take(sizeof(int64_t) * (n + 1));
        row1 = take(sizeof(int) * (n + 1));
        rt = take(sizeof(int) * (n + 1));
        ct = take(sizeof(int) * (n + 1));
        grow = take(sizeof(int) * (n + 1));
        band = take(sizeof(int) * (n + 1));
        total = o;
    }
};

// Serialises the tables into host memory laid out as TableLayout.
inline void pack_tables(const HostBatch& hb, unsigned char* dst) {
    const int n = (int)hb.tiles.size();
    const TableLayout L(n);
    memcpy(dst + L.tiles, hb.tiles.data(), sizeof(TileParams) * n);
    memcpy(dst + L.chunk, hb.chunk_base.data(), sizeof(int) * (n + 1));
    memcpy(dst + L.scan, hb.scan_base.data(), sizeof(int) * (n + 1));
    memcpy(dst + L.blk, hb.blk_base.data(), sizeof(int64_t) * (n + 1));
    memcpy(dst + L.sup, hb.sup_base.data(), sizeof(int64_t) * (n + 1));
    memcpy(dst + L.row1, hb.row1_base.data(), sizeof(int) * (n + 1));
    memcpy(dst + L.rt, hb.rt_base.data(), sizeof(int) * (n + 1));
    memcpy(dst + L.ct, hb.ct_base.data(), sizeof(int) * (n + 1));
    memcpy(dst + L.grow, hb.grow_base.data(), sizeof(int) * (n + 1));
    memcpy(dst + L.band, hb.band_base.data(), sizeof(int) * (n + 1));
}

// Device view of tables uploaded to `dev` (laid out as TableLayout).
inline BatchTables device_tables(const unsigned char* dev, int n) {
    const TableLayout L(n);
    BatchTables bt;
    bt.tiles = (const TileParams*)(dev + L.tiles);
    bt.ntiles = n;
    bt.chunk_base = (const int*)(dev + L.chunk);
    bt.scan_base = (const int*)(dev + L.scan);
    bt.blk_base = (const int64_t*)(dev + L.blk);
    bt.sup_base = (const int64_t*)(dev + L.sup);
    bt.row1_base = (const int*)(dev + L.row1);
    bt.rt_base = (const int*)(dev + L.rt);
    bt.ct_base = (const int*)(dev + L.ct);
    bt.grow_base = (const int*)(dev + L.grow);
    bt.band_base = (const int*)(dev + L.band);
    return bt;
}

}  // namespace dnni
