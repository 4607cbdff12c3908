// dnni_plan.h -- host-side planning of one work package: validation of the
// work package and the choice of the search-bin grid.  Shared by the engine
// and by the host build of the kernels that the test suite checks.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "../../include/dnni.h"
#include "dnni_kernels.cuh"

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
