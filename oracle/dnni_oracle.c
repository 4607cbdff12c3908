/*
 * dnni_oracle.c -- CPU oracle for the discrete natural-neighbour interpolation
 * (NNI) hot path.  TEST INFRASTRUCTURE ONLY: this file is the checker that the
 * pytest suite, the smoke entry and the bench's cpu_baseline leg compare the
 * CUDA engine against.  Nothing in the product library links or calls it.
 *
 * PARITY UNPINNED: the reference (TerraNNI) ships no tests, golden vectors or
 * known-answer fixtures, and its own implementation cannot be built or run
 * here (it needs OpenGL/GLX, TPIE, libLAS and Boost; its CUDA file uses
 * texture references that CUDA 12 removed).  This oracle is therefore pinned by
 * analytic known answers (constant field, single site, two-site bisector,
 * symmetric lattices, exact ties) and by brute-force O(pixels x points)
 * restatements, all in the test suite.
 *
 * What the reference computes (per work package, 2-D):
 *   - nni.cpp:722-790 renderInputPoints + nni.cpp:171-230 drawPlane: every
 *     site is drawn as a depth-tested lifted plane, so each raster pixel keeps
 *     the z-code of its nearest site (GL_LEQUAL, later-drawn wins ties);
 *   - nni.cpp:794-820 performNNIQueries + nni.cpp:483-534 makeBlocks: every
 *     query cell q draws its own plane with depth writes off; a query fragment
 *     survives at pixel p iff |p-q|^2 <= |p-s(p)|^2 (the discrete Sibson
 *     "stealing" test);
 *   - cuda_nni.cu:407-488 calcNNI/cudaCheckBits: for each surviving
 *     (pixel, query) pair numer[q] += zcode(s(p)), denom[q] += 1;
 *   - cuda_nni.cu:491-503 divide and nni.cpp:824-866: h = numer/denom, NODATA
 *     when denom == 0.
 *
 * Canonical semantics restated here (scatter form, exact):
 *   pixel lattice == cell lattice (scaling 1), pixel/cell (i,j) at LAS
 *   position (origin_x + i*cell, origin_y + j*cell); s(p) = the site with the
 *   smallest (d^2, gid, z) key, d^2 in int64 on int32 LAS coordinates;
 *   R2(p) = floor(d^2 / cell^2); every grid cell q with |q-p|^2 <= R2(p)
 *   (cell-index units) gets Z[q] += z(s(p)), C[q] += 1;
 *   h = float((double)Z / (double)C * z_scale + z_offset), nodata if C == 0.
 *
 * A reference-compatible emulation (squares of half-side r/sqrt(2), scaling,
 * zMultiplier quantisation, int32 truncating divide) and a float32
 * lifted-plane depth emulation (to measure how often the reference's depth
 * buffer picks a different site than the exact search) are also provided.
 * Both approximate the GL rasteriser (pixel-centre coverage, plane evaluated at
 * the centre); that is stated wherever their numbers are reported.
 *
 * Build: gcc -O3 -fPIC -shared -ffp-contract=off (see oracle/Makefile).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <limits.h>

#define ORC_OK 0
#define ORC_E_INVAL 1
#define ORC_E_NOMEM 2
#define ORC_NO_SITE 0xFFFFFFFFu

/* Same field order and meaning as dnni_workpackage in include/dnni.h. */
typedef struct {
    int32_t ncols, nrows;
    int32_t cell_size;
    int32_t origin_x, origin_y;
    int32_t raster_x0, raster_y0, raster_x1, raster_y1;
    int32_t pad0;
    double z_scale, z_offset;
    float nodata;
    int32_t pad1;
} orc_wp;

typedef struct { int32_t x, y, z; uint32_t gid; } orc_pt;

/* ------------------------------------------------------------------ */
/* small helpers                                                        */
/* ------------------------------------------------------------------ */

static void resolve_raster(const orc_wp *wp, int32_t r[4]) {
    if (wp->raster_x0 == 0 && wp->raster_y0 == 0 && wp->raster_x1 == 0 && wp->raster_y1 == 0) {
        r[0] = 0; r[1] = 0; r[2] = wp->ncols; r[3] = wp->nrows;
    } else {
        r[0] = wp->raster_x0; r[1] = wp->raster_y0; r[2] = wp->raster_x1; r[3] = wp->raster_y1;
    }
}

static int check_wp(const orc_wp *wp, int32_t r[4]) {
    if (wp->ncols <= 0 || wp->nrows <= 0 || wp->cell_size <= 0) return ORC_E_INVAL;
    resolve_raster(wp, r);
    if (r[2] <= r[0] || r[3] <= r[1]) return ORC_E_INVAL;
    int64_t ex = (int64_t)(r[2] > wp->ncols ? r[2] : wp->ncols) - (r[0] < 0 ? r[0] : 0);
    int64_t ey = (int64_t)(r[3] > wp->nrows ? r[3] : wp->nrows) - (r[1] < 0 ? r[1] : 0);
    if (ex > 32767 || ey > 32767) return ORC_E_INVAL;
    return ORC_OK;
}

/* cap for R2: no pixel/cell pair of this work package is farther apart */
static int64_t r2_cap(const orc_wp *wp, const int32_t r[4]) {
    int64_t ex = (int64_t)(r[2] > wp->ncols ? r[2] : wp->ncols) - (r[0] < 0 ? r[0] : 0);
    int64_t ey = (int64_t)(r[3] > wp->nrows ? r[3] : wp->nrows) - (r[1] < 0 ? r[1] : 0);
    return ex * ex + ey * ey;
}

static uint64_t isqrt_u64(uint64_t v) {
    uint64_t s = (uint64_t)sqrt((double)v);
    while (s * s > v) s--;
    while ((s + 1) * (s + 1) <= v) s++;
    return s;
}

/* lexicographic (d2, gid, z): returns 1 if candidate beats best */
static inline int key_less(int64_t d2, uint32_t gid, int32_t z,
                           int64_t bd2, uint32_t bgid, int32_t bz) {
    if (d2 != bd2) return d2 < bd2;
    if (gid != bgid) return gid < bgid;
    return z < bz;
}

float orc_height(int64_t Z, int64_t C, double z_scale, double z_offset, float nodata) {
    if (C <= 0) return nodata;
    double q = (double)Z / (double)C;
    double v = q * z_scale;
    v = v + z_offset;
    return (float)v;
}

/* ------------------------------------------------------------------ */
/* k-d tree for the exact nearest site (independent of the GPU's bins)  */
/* ------------------------------------------------------------------ */

#define KD_LEAF 8

typedef struct {
    orc_pt *p;          /* permuted copy of the points */
    int64_t n;
    int32_t *split;     /* per node split value */
    uint8_t *axis;      /* per node split axis */
    int64_t nnodes;
} kdtree;

static inline int32_t coord(const orc_pt *p, int a) { return a ? p->y : p->x; }

static void kd_select(orc_pt *p, int64_t lo, int64_t hi, int64_t k, int a) {
    /* quickselect on [lo, hi): afterwards p[k] is the k-th smallest on axis a,
       everything left of k is <=, everything right is >= */
    while (hi - lo > 1) {
        int64_t mid = lo + (hi - lo) / 2;
        int32_t v0 = coord(&p[lo], a), v1 = coord(&p[mid], a), v2 = coord(&p[hi - 1], a);
        int32_t piv = v0 < v1 ? (v1 < v2 ? v1 : (v0 < v2 ? v2 : v0)) : (v0 < v2 ? v0 : (v1 < v2 ? v2 : v1));
        int64_t i = lo, j = hi - 1;
        while (i <= j) {
            while (coord(&p[i], a) < piv) i++;
            while (coord(&p[j], a) > piv) j--;
            if (i <= j) { orc_pt t = p[i]; p[i] = p[j]; p[j] = t; i++; j--; }
        }
        if (k <= j) hi = j + 1;
        else if (k >= i) lo = i;
        else return;
    }
}

static void kd_build_rec(kdtree *t, int64_t node, int64_t lo, int64_t hi) {
    if (hi - lo <= KD_LEAF || node >= t->nnodes) return;
    int32_t mnx = INT32_MAX, mxx = INT32_MIN, mny = INT32_MAX, mxy = INT32_MIN;
    for (int64_t i = lo; i < hi; i++) {
        if (t->p[i].x < mnx) mnx = t->p[i].x;
        if (t->p[i].x > mxx) mxx = t->p[i].x;
        if (t->p[i].y < mny) mny = t->p[i].y;
        if (t->p[i].y > mxy) mxy = t->p[i].y;
    }
    int a = ((int64_t)mxy - mny) > ((int64_t)mxx - mnx) ? 1 : 0;
    int64_t mid = lo + (hi - lo) / 2;
    kd_select(t->p, lo, hi, mid, a);
    t->axis[node] = (uint8_t)a;
    t->split[node] = coord(&t->p[mid], a);
    kd_build_rec(t, 2 * node + 1, lo, mid);
    kd_build_rec(t, 2 * node + 2, mid, hi);
}

static int kd_build(kdtree *t, const int32_t *xyz, const uint32_t *gid, int64_t n) {
    memset(t, 0, sizeof(*t));
    t->n = n;
    t->p = (orc_pt *)malloc(sizeof(orc_pt) * (size_t)(n > 0 ? n : 1));
    if (!t->p) return ORC_E_NOMEM;
    for (int64_t i = 0; i < n; i++) {
        t->p[i].x = xyz[3 * i]; t->p[i].y = xyz[3 * i + 1]; t->p[i].z = xyz[3 * i + 2];
        t->p[i].gid = gid ? gid[i] : (uint32_t)i;
    }
    int64_t leaves = 1;
    while (leaves * KD_LEAF < n) leaves *= 2;
    t->nnodes = 2 * leaves;
    t->split = (int32_t *)calloc((size_t)t->nnodes, sizeof(int32_t));
    t->axis = (uint8_t *)calloc((size_t)t->nnodes, 1);
    if (!t->split || !t->axis) return ORC_E_NOMEM;
    kd_build_rec(t, 0, 0, n);
    return ORC_OK;
}

static void kd_free(kdtree *t) { free(t->p); free(t->split); free(t->axis); }

typedef struct { int64_t d2; uint32_t gid; int32_t z; } nn_best;

static void kd_query_rec(const kdtree *t, int64_t node, int64_t lo, int64_t hi,
                         int64_t qx, int64_t qy, nn_best *b) {
    if (hi - lo <= KD_LEAF || node >= t->nnodes) {
        for (int64_t i = lo; i < hi; i++) {
            int64_t dx = t->p[i].x - qx, dy = t->p[i].y - qy;
            int64_t d2 = dx * dx + dy * dy;
            if (key_less(d2, t->p[i].gid, t->p[i].z, b->d2, b->gid, b->z)) {
                b->d2 = d2; b->gid = t->p[i].gid; b->z = t->p[i].z;
            }
        }
        return;
    }
    int a = t->axis[node];
    int64_t s = t->split[node];
    int64_t q = a ? qy : qx;
    int64_t mid = lo + (hi - lo) / 2;
    int64_t diff = q - s;
    if (diff < 0) {
        kd_query_rec(t, 2 * node + 1, lo, mid, qx, qy, b);
        if (diff * diff <= b->d2) kd_query_rec(t, 2 * node + 2, mid, hi, qx, qy, b);
    } else {
        kd_query_rec(t, 2 * node + 2, mid, hi, qx, qy, b);
        if (diff * diff <= b->d2) kd_query_rec(t, 2 * node + 1, lo, mid, qx, qy, b);
    }
}

/* ------------------------------------------------------------------ */
/* exact nearest-site map                                               */
/* ------------------------------------------------------------------ */

/* Nearest site for every raster pixel.  Outputs (each optional):
 *   site_gid[p]  gid of the nearest site, ORC_NO_SITE when n == 0
 *   site_z[p]    its z
 *   r2[p]        min(floor(d^2/cell^2), cap), -1 when n == 0
 * Raster layout: row-major, (raster_y1-raster_y0) rows of
 * (raster_x1-raster_x0) pixels, row 0 = smallest y. */
int orc_nearest(const orc_wp *wp, const int32_t *xyz, const uint32_t *gid, int64_t n,
                uint32_t *site_gid, int32_t *site_z, int32_t *r2) {
    int32_t r[4];
    if (check_wp(wp, r)) return ORC_E_INVAL;
    int64_t rw = r[2] - r[0], rh = r[3] - r[1];
    int64_t cap = r2_cap(wp, r);
    int64_t cs2 = (int64_t)wp->cell_size * wp->cell_size;
    kdtree t;
    if (n > 0 && kd_build(&t, xyz, gid, n)) { kd_free(&t); return ORC_E_NOMEM; }
    for (int64_t j = 0; j < rh; j++) {
        for (int64_t i = 0; i < rw; i++) {
            int64_t pidx = j * rw + i;
            if (n == 0) {
                if (site_gid) site_gid[pidx] = ORC_NO_SITE;
                if (site_z) site_z[pidx] = 0;
                if (r2) r2[pidx] = -1;
                continue;
            }
            int64_t qx = (int64_t)wp->origin_x + (r[0] + i) * (int64_t)wp->cell_size;
            int64_t qy = (int64_t)wp->origin_y + (r[1] + j) * (int64_t)wp->cell_size;
            nn_best b = { INT64_MAX, 0xFFFFFFFFu, INT32_MAX };
            kd_query_rec(&t, 0, 0, n, qx, qy, &b);
            if (site_gid) site_gid[pidx] = b.gid;
            if (site_z) site_z[pidx] = b.z;
            if (r2) { int64_t v = b.d2 / cs2; r2[pidx] = (int32_t)(v > cap ? cap : v); }
        }
    }
    if (n > 0) kd_free(&t);
    return ORC_OK;
}

/* O(pixels x points) nearest site; tiny cases only. */
int orc_nearest_brute(const orc_wp *wp, const int32_t *xyz, const uint32_t *gid, int64_t n,
                      uint32_t *site_gid, int32_t *site_z, int32_t *r2) {
    int32_t r[4];
    if (check_wp(wp, r)) return ORC_E_INVAL;
    int64_t rw = r[2] - r[0], rh = r[3] - r[1];
    int64_t cap = r2_cap(wp, r);
    int64_t cs2 = (int64_t)wp->cell_size * wp->cell_size;
    for (int64_t j = 0; j < rh; j++)
        for (int64_t i = 0; i < rw; i++) {
            int64_t pidx = j * rw + i;
            int64_t qx = (int64_t)wp->origin_x + (r[0] + i) * (int64_t)wp->cell_size;
            int64_t qy = (int64_t)wp->origin_y + (r[1] + j) * (int64_t)wp->cell_size;
            nn_best b = { INT64_MAX, 0xFFFFFFFFu, INT32_MAX };
            for (int64_t k = 0; k < n; k++) {
                int64_t dx = xyz[3 * k] - qx, dy = xyz[3 * k + 1] - qy;
                int64_t d2 = dx * dx + dy * dy;
                uint32_t g = gid ? gid[k] : (uint32_t)k;
                if (key_less(d2, g, xyz[3 * k + 2], b.d2, b.gid, b.z)) { b.d2 = d2; b.gid = g; b.z = xyz[3 * k + 2]; }
            }
            if (site_gid) site_gid[pidx] = n ? b.gid : ORC_NO_SITE;
            if (site_z) site_z[pidx] = n ? b.z : 0;
            if (r2) { int64_t v = n ? b.d2 / cs2 : -1; r2[pidx] = (int32_t)(v > cap ? cap : v); }
        }
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* scatter-accumulate + finalize                                        */
/* ------------------------------------------------------------------ */

static void finalize_grid(const orc_wp *wp, const int64_t *Z, const int64_t *C, float *h) {
    int64_t cells = (int64_t)wp->ncols * wp->nrows;
    for (int64_t q = 0; q < cells; q++) h[q] = orc_height(Z[q], C[q], wp->z_scale, wp->z_offset, wp->nodata);
}

/* Row-span scatter: each pixel's disc becomes 2*floor(sqrt(R2))+1 row spans,
 * each span adds (+z,+1) at its first cell and (-z,-1) after its last one, and
 * a row prefix sum turns the differences into Z and C. */
static int scatter_spans(const orc_wp *wp, const int32_t r[4], const int32_t *site_z,
                         const int32_t *r2, int64_t *Z, int64_t *C) {
    int64_t rw = r[2] - r[0], rh = r[3] - r[1];
    int64_t nc = wp->ncols, nr = wp->nrows;
    memset(Z, 0, sizeof(int64_t) * (size_t)(nc * nr));
    memset(C, 0, sizeof(int64_t) * (size_t)(nc * nr));
    for (int64_t j = 0; j < rh; j++)
        for (int64_t i = 0; i < rw; i++) {
            int64_t pidx = j * rw + i;
            int64_t R2 = r2[pidx];
            if (R2 < 0) continue;
            int64_t px = r[0] + i, py = r[1] + j;
            int64_t z = site_z[pidx];
            int64_t rr = (int64_t)isqrt_u64((uint64_t)R2);
            for (int64_t dy = -rr; dy <= rr; dy++) {
                int64_t row = py + dy;
                if (row < 0 || row >= nr) continue;
                int64_t w = (int64_t)isqrt_u64((uint64_t)(R2 - dy * dy));
                int64_t a = px - w, b = px + w;
                if (a < 0) a = 0;
                if (b > nc - 1) b = nc - 1;
                if (a > b) continue;
                Z[row * nc + a] += z; C[row * nc + a] += 1;
                if (b + 1 < nc) { Z[row * nc + b + 1] -= z; C[row * nc + b + 1] -= 1; }
            }
        }
    for (int64_t row = 0; row < nr; row++) {
        int64_t sz = 0, sc = 0;
        for (int64_t x = 0; x < nc; x++) {
            sz += Z[row * nc + x]; sc += C[row * nc + x];
            Z[row * nc + x] = sz; C[row * nc + x] = sc;
        }
    }
    return ORC_OK;
}

/* Full canonical interpolation (exact site search + span scatter).
 * h: nrows*ncols floats (row 0 = smallest y); site_gid: raster pixels
 * (optional); Z, C: per-cell int64 sums (optional). */
int orc_interpolate(const orc_wp *wp, const int32_t *xyz, const uint32_t *gid, int64_t n,
                    float *h, uint32_t *site_gid, int64_t *Zout, int64_t *Cout) {
    int32_t r[4];
    if (check_wp(wp, r)) return ORC_E_INVAL;
    int64_t npix = (int64_t)(r[2] - r[0]) * (r[3] - r[1]);
    int64_t cells = (int64_t)wp->ncols * wp->nrows;
    int32_t *sz = (int32_t *)malloc(sizeof(int32_t) * (size_t)npix);
    int32_t *r2 = (int32_t *)malloc(sizeof(int32_t) * (size_t)npix);
    int64_t *Z = Zout ? Zout : (int64_t *)malloc(sizeof(int64_t) * (size_t)cells);
    int64_t *C = Cout ? Cout : (int64_t *)malloc(sizeof(int64_t) * (size_t)cells);
    int rc = ORC_E_NOMEM;
    if (sz && r2 && Z && C) {
        rc = orc_nearest(wp, xyz, gid, n, site_gid, sz, r2);
        if (rc == ORC_OK) {
            scatter_spans(wp, r, sz, r2, Z, C);
            if (h) finalize_grid(wp, Z, C, h);
        }
    }
    free(sz); free(r2);
    if (!Zout) free(Z);
    if (!Cout) free(C);
    return rc;
}

/* Direct area scatter over every (pixel, cell) pair; tiny cases only. */
int orc_interpolate_brute(const orc_wp *wp, const int32_t *xyz, const uint32_t *gid, int64_t n,
                          float *h, uint32_t *site_gid, int64_t *Zout, int64_t *Cout) {
    int32_t r[4];
    if (check_wp(wp, r)) return ORC_E_INVAL;
    int64_t rw = r[2] - r[0], rh = r[3] - r[1];
    int64_t npix = rw * rh;
    int64_t nc = wp->ncols, nr = wp->nrows, cells = nc * nr;
    int32_t *sz = (int32_t *)malloc(sizeof(int32_t) * (size_t)npix);
    int32_t *r2 = (int32_t *)malloc(sizeof(int32_t) * (size_t)npix);
    int64_t *Z = Zout ? Zout : (int64_t *)malloc(sizeof(int64_t) * (size_t)cells);
    int64_t *C = Cout ? Cout : (int64_t *)malloc(sizeof(int64_t) * (size_t)cells);
    if (!sz || !r2 || !Z || !C) return ORC_E_NOMEM;
    orc_nearest_brute(wp, xyz, gid, n, site_gid, sz, r2);
    memset(Z, 0, sizeof(int64_t) * (size_t)cells);
    memset(C, 0, sizeof(int64_t) * (size_t)cells);
    for (int64_t j = 0; j < rh; j++)
        for (int64_t i = 0; i < rw; i++) {
            int64_t R2 = r2[j * rw + i];
            if (R2 < 0) continue;
            int64_t px = r[0] + i, py = r[1] + j;
            for (int64_t qy = 0; qy < nr; qy++)
                for (int64_t qx = 0; qx < nc; qx++) {
                    int64_t dx = qx - px, dy = qy - py;
                    if (dx * dx + dy * dy <= R2) { Z[qy * nc + qx] += sz[j * rw + i]; C[qy * nc + qx] += 1; }
                }
        }
    if (h) finalize_grid(wp, Z, C, h);
    free(sz); free(r2);
    if (!Zout) free(Z);
    if (!Cout) free(C);
    return ORC_OK;
}

/* Work figures for a work package (used by tests and reports):
 * out[0] = sum over pixels of (2*floor(sqrt(R2))+1) row spans (all rows,
 *          unclipped), out[1] = max R2, out[2] = pixels with a site. */
int orc_work_stats(const orc_wp *wp, const int32_t *r2, int64_t out[3]) {
    int32_t r[4];
    if (check_wp(wp, r)) return ORC_E_INVAL;
    int64_t npix = (int64_t)(r[2] - r[0]) * (r[3] - r[1]);
    int64_t spans = 0, mx = -1, cnt = 0;
    for (int64_t p = 0; p < npix; p++) {
        if (r2[p] < 0) continue;
        cnt++;
        spans += 2 * (int64_t)isqrt_u64((uint64_t)r2[p]) + 1;
        if (r2[p] > mx) mx = r2[p];
    }
    out[0] = spans; out[1] = mx; out[2] = cnt;
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* reference depth-buffer emulation (float32 lifted planes)             */
/* ------------------------------------------------------------------ */

/* The lifted plane of a site (or query) whose offset from the work-package
 * origin is (dx, dy) metres, as drawPlane forms it (nni.cpp:186-200): the
 * offset stays in double (site.p - x_offset), zpx = (dx + halfwidth) /
 * halfwidth and the slopes a = -2.0 * zpx / halfwidth are evaluated in
 * double and rounded to float once each, and z_offset is the float sum of
 * the float squares (the time term is zero in 2-D). */
typedef struct { float a, b, zoff; } orc_plane;

static inline orc_plane plane_of(float hw, double dx, double dy) {
    orc_plane P;
    float zpx = (float)((dx + (double)hw) / (double)hw);
    float zpy = (float)((dy + (double)hw) / (double)hw);
    P.zoff = zpx * zpx + zpy * zpy;
    P.a = (float)((-2.0 * (double)zpx) / (double)hw);
    P.b = (float)((-2.0 * (double)zpy) / (double)hw);
    return P;
}

/* Depth of a plane at a pixel centre (px, py), in float as the vertex depths
 * of nni.cpp:208-216 are formed.  The rasteriser interpolates the plane
 * between the square's vertices; evaluating the same plane at the pixel
 * centre is the approximation made here. */
static inline float plane_depth(const orc_plane *P, float hw, float px, float py) {
    float zx = px + hw, zy = py + hw;
    return P->a * zx + P->b * zy + P->zoff;
}

/* optional quantisation to an unsigned fixed-point depth buffer of `bits` bits
 * (glOrtho near/far -200..200 as nni.cpp:644-660 sets for planes) */
static inline double quant_depth(float z, int bits) {
    if (bits <= 0) return (double)z;
    double w = 0.5 + (double)z / 400.0;   /* window depth in [0,1] */
    double scale = ldexp(1.0, bits) - 1.0;
    return floor(w * scale + 0.5);
}

/* For each raster pixel, the site the reference's depth test would keep when
 * every site's plane covers the pixel (LEQUAL, later draw order wins on
 * equal depth), compared with the exact nearest site.  Draw order = array
 * order.  xy_scale converts LAS units to metres.  Candidates are the sites
 * whose exact d^2 lies within `slack_units2` of the exact minimum (the float
 * depth cannot separate sites farther apart than its rounding error; the
 * caller sizes the slack generously).  Returns counts in out[]:
 *   out[0] pixels compared, out[1] pixels whose kept site differs,
 *   out[2] pixels whose kept site has a different z. */
int orc_gl_disagreement(const orc_wp *wp, const int32_t *xyz, const uint32_t *gid, int64_t n,
                        double xy_scale, int depth_bits, int64_t slack_units2, int64_t out[3]) {
    int32_t r[4];
    if (check_wp(wp, r)) return ORC_E_INVAL;
    out[0] = out[1] = out[2] = 0;
    if (n == 0) return ORC_OK;
    int64_t rw = r[2] - r[0], rh = r[3] - r[1];
    kdtree t;
    if (kd_build(&t, xyz, gid, n)) { kd_free(&t); return ORC_E_NOMEM; }
    /* index by gid -> array position for draw order */
    float hw = (float)(((double)(wp->nrows - 1) * wp->cell_size * xy_scale) / 2.0);
    int64_t cap = 4096;
    int64_t *cand = (int64_t *)malloc(sizeof(int64_t) * (size_t)cap);
    for (int64_t j = 0; j < rh; j++)
        for (int64_t i = 0; i < rw; i++) {
            int64_t qx = (int64_t)wp->origin_x + (r[0] + i) * (int64_t)wp->cell_size;
            int64_t qy = (int64_t)wp->origin_y + (r[1] + j) * (int64_t)wp->cell_size;
            nn_best b = { INT64_MAX, 0xFFFFFFFFu, INT32_MAX };
            kd_query_rec(&t, 0, 0, n, qx, qy, &b);
            /* brute candidate sweep restricted by a box around the pixel */
            int64_t lim = b.d2 + slack_units2;
            int64_t nc = 0;
            /* walk the tree collecting candidates within lim (stack) */
            int64_t stk[256][3]; int sp = 0;
            stk[sp][0] = 0; stk[sp][1] = 0; stk[sp][2] = n; sp++;
            while (sp) {
                sp--;
                int64_t node = stk[sp][0], lo = stk[sp][1], hi = stk[sp][2];
                if (hi - lo <= KD_LEAF || node >= t.nnodes) {
                    for (int64_t k = lo; k < hi; k++) {
                        int64_t dx = t.p[k].x - qx, dy = t.p[k].y - qy;
                        if (dx * dx + dy * dy <= lim) {
                            if (nc == cap) { cap *= 2; cand = (int64_t *)realloc(cand, sizeof(int64_t) * (size_t)cap); }
                            cand[nc++] = k;
                        }
                    }
                    continue;
                }
                int a = t.axis[node];
                int64_t s = t.split[node], q = a ? qy : qx, mid = lo + (hi - lo) / 2;
                int64_t diff = q - s;
                if (diff < 0 || diff * diff <= lim) { stk[sp][0] = 2 * node + 1; stk[sp][1] = lo; stk[sp][2] = mid; sp++; }
                if (diff >= 0 || diff * diff <= lim) { stk[sp][0] = 2 * node + 2; stk[sp][1] = mid; stk[sp][2] = hi; sp++; }
            }
            /* draw order = gid order here (array order with default gids) */
            float px = (float)((double)(r[0] + i) * wp->cell_size * xy_scale);
            float py = (float)((double)(r[1] + j) * wp->cell_size * xy_scale);
            double bestd = INFINITY; uint32_t bg = 0; int32_t bz = 0; int have = 0;
            /* sort candidates by gid so "later wins" follows draw order */
            for (int64_t a1 = 1; a1 < nc; a1++) {
                int64_t v = cand[a1], b1 = a1 - 1;
                while (b1 >= 0 && t.p[cand[b1]].gid > t.p[v].gid) { cand[b1 + 1] = cand[b1]; b1--; }
                cand[b1 + 1] = v;
            }
            for (int64_t c = 0; c < nc; c++) {
                const orc_pt *s = &t.p[cand[c]];
                const orc_plane P = plane_of(hw, (double)(s->x - wp->origin_x) * xy_scale,
                                             (double)(s->y - wp->origin_y) * xy_scale);
                double d = quant_depth(plane_depth(&P, hw, px, py), depth_bits);
                if (!have || d <= bestd) { bestd = d; bg = s->gid; bz = s->z; have = 1; }
            }
            out[0]++;
            if (bg != b.gid) out[1]++;
            if (bz != b.z) out[2]++;
        }
    free(cand);
    kd_free(&t);
    return ORC_OK;
}

/* ------------------------------------------------------------------ */
/* reference-compatible emulation of nni::performNNI (2-D, planes)      */
/* ------------------------------------------------------------------ */

typedef struct {
    int32_t scale;          /* Settings::scale            (nni.h:73) */
    float cell_size;        /* Settings::cell_size        (nni.h:74) */
    float site_radius;      /* Settings::site_radius      (nni.h:76) */
    double query_radius;    /* Settings::query_radius     (nni.h:77) */
    int32_t point_min;      /* Settings::pointMin         (nni.h:79) */
    int32_t multiplier;     /* Settings::multiplier       (nni.h:80) */
    int32_t total_ncols, total_nrows;   /* Settings::ncols/nrows */
} orc_compat_settings;

typedef struct {
    float origin_x, origin_y, grid_origin_x, grid_origin_y;
    int32_t nrows, ncols;
} orc_compat_wp;            /* WorkPackage (nni.h:66-70) */

/* Emulates nni.cpp:870-944 for timeRadius == 0 with the plane algorithm:
 *   pixel_offset / raster size        nni.cpp:879-886
 *   site squares, z-code, LEQUAL       nni.cpp:171-230, 470-479, 538-549, 733-737
 *   query squares vs stored depth      nni.cpp:483-534, 803-807
 *   int32 numer/denom, trunc divide    cuda_nni.cu:423-448, 491-503
 *   dequantise                         nni.cpp:836-848
 * Points are world coordinates (x, y, z doubles) in draw order.  Outputs the
 * per-cell height as completeBufferAnalysis writes it (i-major over the
 * work package, nrows*ncols, row-major j*ncols+i) and res[] = the int32
 * division result.  Pixel coverage is tested at pixel centres over the
 * half-open square [x-r, x+r) x [y-r, y+r); the real rasteriser's fill rule
 * and interpolation rounding are not reproduced. */
int orc_compat(const orc_compat_settings *s, const orc_compat_wp *wp, const double *pts, int64_t n,
               float *h_out, int32_t *res_out) {
    if (s->scale <= 0 || s->cell_size <= 0 || wp->nrows <= 0 || wp->ncols <= 0) return ORC_E_INVAL;
    /* The reference splits queries into 5x5 blocks and spacingFactor^2 rounds
       (nni.cpp:498-534, 879) only to fit 32 one-hot bits per pixel; every
       query still tests every pixel of its square, which is what is done
       directly below. */
    double query_spacing = s->cell_size;
    int scaling = s->scale;
    double pixel_size = query_spacing / scaling;
    float qr = (float)s->query_radius;  /* the reference keeps query_radius as float (nni.cpp:69) */
    int pixel_offset = (int)ceil((qr - floor(scaling / 2.0) * pixel_size) / pixel_size) + 1;
    int64_t xp = (int64_t)wp->ncols * scaling + 2 * pixel_offset;
    int64_t yp = (int64_t)wp->nrows * scaling + 2 * pixel_offset;
    double left = 0 - (query_spacing / 2.0) - (pixel_offset * pixel_size);
    double bottom = left;
    float hw = (float)(((wp->nrows - 1) * query_spacing) / 2.0);
    int zOffset = -1 * s->point_min;
    int zMult = s->multiplier;
    uint32_t *col = (uint32_t *)calloc((size_t)(xp * yp), sizeof(uint32_t));
    float *dep = (float *)malloc(sizeof(float) * (size_t)(xp * yp));
    int32_t *numer = (int32_t *)calloc((size_t)wp->nrows * wp->ncols, sizeof(int32_t));
    int32_t *denom = (int32_t *)calloc((size_t)wp->nrows * wp->ncols, sizeof(int32_t));
    if (!col || !dep || !numer || !denom) return ORC_E_NOMEM;
    for (int64_t k = 0; k < xp * yp; k++) dep[k] = INFINITY;
    double rs = s->site_radius / sqrt(2.0);
    /* site step */
    for (int64_t k = 0; k < n; k++) {
        double dx = pts[3 * k] - (double)wp->origin_x, dy = pts[3 * k + 1] - (double)wp->origin_y;
        float sx = (float)dx, sy = (float)dy;
        const orc_plane P = plane_of(hw, dx, dy);
        uint32_t zc = (uint32_t)floor((pts[3 * k + 2] + zOffset + 1) * zMult);
        float x0 = (float)(sx - rs), x1 = (float)(sx + rs), y0 = (float)(sy - rs), y1 = (float)(sy + rs);
        int64_t i0 = (int64_t)ceil((x0 - left) / pixel_size - 0.5), i1 = (int64_t)ceil((x1 - left) / pixel_size - 0.5) - 1;
        int64_t j0 = (int64_t)ceil((y0 - bottom) / pixel_size - 0.5), j1 = (int64_t)ceil((y1 - bottom) / pixel_size - 0.5) - 1;
        if (i0 < 0) i0 = 0;
        if (j0 < 0) j0 = 0;
        if (i1 > xp - 1) i1 = xp - 1;
        if (j1 > yp - 1) j1 = yp - 1;
        for (int64_t pj = j0; pj <= j1; pj++)
            for (int64_t pi = i0; pi <= i1; pi++) {
                float cx = (float)(left + (pi + 0.5) * pixel_size);
                float cy = (float)(bottom + (pj + 0.5) * pixel_size);
                float d = plane_depth(&P, hw, cx, cy);
                if (d <= dep[pj * xp + pi]) { dep[pj * xp + pi] = d; col[pj * xp + pi] = zc; }
            }
    }
    /* query step: every query cell, square of half-side qr/sqrt(2) */
    double rq = qr / sqrt(2.0);
    for (int64_t j = 0; j < wp->nrows; j++)
        for (int64_t i = 0; i < wp->ncols; i++) {
            float qx = (float)(i * query_spacing), qy = (float)(j * query_spacing);
            const orc_plane Q = plane_of(hw, i * query_spacing, j * query_spacing);
            float x0 = (float)(qx - rq), x1 = (float)(qx + rq), y0 = (float)(qy - rq), y1 = (float)(qy + rq);
            int64_t i0 = (int64_t)ceil((x0 - left) / pixel_size - 0.5), i1 = (int64_t)ceil((x1 - left) / pixel_size - 0.5) - 1;
            int64_t j0 = (int64_t)ceil((y0 - bottom) / pixel_size - 0.5), j1 = (int64_t)ceil((y1 - bottom) / pixel_size - 0.5) - 1;
            if (i0 < 0) i0 = 0;
            if (j0 < 0) j0 = 0;
            if (i1 > xp - 1) i1 = xp - 1;
            if (j1 > yp - 1) j1 = yp - 1;
            for (int64_t pj = j0; pj <= j1; pj++)
                for (int64_t pi = i0; pi <= i1; pi++) {
                    uint32_t zc = col[pj * xp + pi];
                    if (zc == 0) continue;                       /* cuda_nni.cu:423 */
                    float cx = (float)(left + (pi + 0.5) * pixel_size);
                    float cy = (float)(bottom + (pj + 0.5) * pixel_size);
                    float d = plane_depth(&Q, hw, cx, cy);
                    if (d <= dep[pj * xp + pi]) {
                        int64_t w = j * wp->ncols + i;
                        numer[w] = (int32_t)((uint32_t)numer[w] + zc);   /* int32 wrap as atomicAdd */
                        denom[w] += 1;
                    }
                }
        }
    for (int64_t j = 0; j < wp->nrows; j++)
        for (int64_t i = 0; i < wp->ncols; i++) {
            int64_t w = j * wp->ncols + i;
            int32_t res = denom[w] == 0 ? -9999 * zMult : numer[w] / denom[w];
            if (res_out) res_out[w] = res;
            double z = 1.0 * res / zMult;
            if (z != -9999) z = z - zOffset - 1;
            if (h_out) h_out[w] = (float)z;
        }
    free(col); free(dep); free(numer); free(denom);
    return ORC_OK;
}

/* zMultiplier as terranni.cpp:675-684 derives it. */
int32_t orc_compat_multiplier(float site_radius, int32_t scale, float cell_size, double zmax, int32_t point_min) {
    int pw = (int)ceil(2.0 * site_radius * scale / cell_size);
    double max_sum = (double)pw * pw * (zmax - point_min);
    int m = 1;
    if (max_sum < (double)INT_MAX) {
        m = (int)floor(1.0 * INT_MAX / max_sum);
        m = (int)pow(10, floor(log10(m)));
    }
    return m;
}

/* ------------------------------------------------------------------ */
/* space-time (3-D) interpolation, timeRadius > 0                       */
/* ------------------------------------------------------------------ */

/* Canonical restatement of nni::performNNI with a time radius
 * (nni.cpp:902-933 slice loop, nni.cpp:722-790 site selection per slice,
 * nni.cpp:171-230 drawPlane's time term timeOffset^2 in the plane offset,
 * nni.cpp:483-493 query planes lifted by the slice offset):
 *   slices ts = cur + j, j = -rt..rt;
 *   the sites of slice ts are the points with |ts - t| <= rt, each at lifted
 *   squared distance d_l^2 = dx^2 + dy^2 + ((ts - t) * tau)^2 from a pixel
 *   (tau = LAS units per time step); s(p) = min (d_l^2, index, z);
 *   cell q (at time cur) takes pixel p of slice ts iff
 *   |q - p|^2 * cell^2 + (j * tau)^2 <= d_l^2, i.e. |q - p|^2 <= R2 =
 *   floor((d_l^2 - (j tau)^2) / cell^2), none when negative (capped as 2-D);
 *   Z and C are summed over all slices, h as orc_height.
 * Ties go to the lower input index (the earlier point of the stream).
 * brute = 1: every point for every (slice, pixel); brute = 0: one k-d tree
 * per time value, whose 2-D nearest site plus the value's constant time term
 * is that value's best -- the minimum over the values is s(p). */
static int st_scatter_layer(const orc_wp *wp, const int32_t r[4], const int32_t *sz, const int32_t *r2,
                            int64_t *Z, int64_t *C) {
    int64_t rw = r[2] - r[0], rh = r[3] - r[1];
    int64_t nc = wp->ncols, nr = wp->nrows;
    for (int64_t j = 0; j < rh; j++)
        for (int64_t i = 0; i < rw; i++) {
            int64_t R2 = r2[j * rw + i];
            if (R2 < 0) continue;
            int64_t px = r[0] + i, py = r[1] + j, z = sz[j * rw + i];
            int64_t rr = (int64_t)isqrt_u64((uint64_t)R2);
            for (int64_t dy = -rr; dy <= rr; dy++) {
                int64_t row = py + dy;
                if (row < 0 || row >= nr) continue;
                int64_t w = (int64_t)isqrt_u64((uint64_t)(R2 - dy * dy));
                int64_t a = px - w, b = px + w;
                if (a < 0) a = 0;
                if (b > nc - 1) b = nc - 1;
                if (a > b) continue;
                Z[row * nc + a] += z; C[row * nc + a] += 1;
                if (b + 1 < nc) { Z[row * nc + b + 1] -= z; C[row * nc + b + 1] -= 1; }
            }
        }
    return ORC_OK;
}

static int32_t st_r2(uint64_t dl2, int64_t jt, int64_t cs2, int64_t cap) {
    uint64_t q2 = (uint64_t)(jt * jt);
    if (dl2 < q2) return -1;
    uint64_t v = (dl2 - q2) / (uint64_t)cs2;
    return (int32_t)(v > (uint64_t)cap ? (uint64_t)cap : v);
}

int orc_interpolate_st(const orc_wp *wp, const int32_t *xyz, const int32_t *tt, int64_t n, int32_t cur,
                       int32_t rt, int32_t tau, int brute, float *h, int64_t *Zout, int64_t *Cout) {
    int32_t r[4];
    if (check_wp(wp, r) || rt < 0 || rt > 16 || tau <= 0 || (int64_t)rt * tau > (1LL << 30)) return ORC_E_INVAL;
    int64_t rw = r[2] - r[0], rh = r[3] - r[1], npix = rw * rh;
    int64_t cells = (int64_t)wp->ncols * wp->nrows;
    int64_t cap = r2_cap(wp, r), cs2 = (int64_t)wp->cell_size * wp->cell_size;
    int nv = 4 * rt + 1;
    int64_t *Z = Zout ? Zout : (int64_t *)malloc(sizeof(int64_t) * (size_t)cells);
    int64_t *C = Cout ? Cout : (int64_t *)malloc(sizeof(int64_t) * (size_t)cells);
    int32_t *sz = (int32_t *)malloc(sizeof(int32_t) * (size_t)npix);
    int32_t *r2 = (int32_t *)malloc(sizeof(int32_t) * (size_t)npix);
    kdtree *kd = (kdtree *)calloc((size_t)nv, sizeof(kdtree));
    int64_t *cnt = (int64_t *)calloc((size_t)nv, sizeof(int64_t));
    int rc = ORC_E_NOMEM;
    if (!Z || !C || !sz || !r2 || !kd || !cnt) goto out;
    memset(Z, 0, sizeof(int64_t) * (size_t)cells);
    memset(C, 0, sizeof(int64_t) * (size_t)cells);
    if (!brute) {
        /* per time value: the points with that time, in input order */
        int32_t *sx = (int32_t *)malloc(sizeof(int32_t) * 3 * (size_t)(n > 0 ? n : 1));
        uint32_t *sg = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
        if (!sx || !sg) { free(sx); free(sg); goto out; }
        for (int v = 0; v < nv; v++) {
            int64_t m = 0;
            for (int64_t k = 0; k < n; k++)
                if ((int64_t)tt[k] == (int64_t)cur - 2 * rt + v) {
                    sx[3 * m] = xyz[3 * k]; sx[3 * m + 1] = xyz[3 * k + 1]; sx[3 * m + 2] = xyz[3 * k + 2];
                    sg[m++] = (uint32_t)k;
                }
            cnt[v] = m;
            if (m > 0 && kd_build(&kd[v], sx, sg, m)) { free(sx); free(sg); goto out; }
        }
        free(sx); free(sg);
    }
    for (int s = 0; s <= 2 * rt; s++) {
        int64_t ts = (int64_t)cur - rt + s, jt = (int64_t)(s - rt) * tau;
        for (int64_t j = 0; j < rh; j++)
            for (int64_t i = 0; i < rw; i++) {
                int64_t qx = (int64_t)wp->origin_x + (r[0] + i) * (int64_t)wp->cell_size;
                int64_t qy = (int64_t)wp->origin_y + (r[1] + j) * (int64_t)wp->cell_size;
                uint64_t bd = UINT64_MAX;
                uint32_t bg = 0xFFFFFFFFu;
                int32_t bz = INT32_MAX;
                if (brute) {
                    for (int64_t k = 0; k < n; k++) {
                        int64_t dt = ts - tt[k];
                        if (dt < -rt || dt > rt) continue;
                        int64_t dx = xyz[3 * k] - qx, dy = xyz[3 * k + 1] - qy;
                        uint64_t d2 = (uint64_t)(dx * dx) + (uint64_t)(dy * dy) + (uint64_t)(dt * tau * dt * tau);
                        int32_t z = xyz[3 * k + 2];
                        if (d2 < bd || (d2 == bd && ((uint32_t)k < bg || ((uint32_t)k == bg && z < bz)))) {
                            bd = d2; bg = (uint32_t)k; bz = z;
                        }
                    }
                } else {
                    for (int v = s; v <= s + 2 * rt; v++) {
                        if (!cnt[v]) continue;
                        int64_t dt = ts - ((int64_t)cur - 2 * rt + v);
                        nn_best b = { INT64_MAX, 0xFFFFFFFFu, INT32_MAX };
                        kd_query_rec(&kd[v], 0, 0, cnt[v], qx, qy, &b);
                        uint64_t d2 = (uint64_t)b.d2 + (uint64_t)(dt * tau * dt * tau);
                        if (d2 < bd || (d2 == bd && (b.gid < bg || (b.gid == bg && b.z < bz)))) {
                            bd = d2; bg = b.gid; bz = b.z;
                        }
                    }
                }
                sz[j * rw + i] = bz;
                r2[j * rw + i] = bg == 0xFFFFFFFFu ? -1 : st_r2(bd, jt, cs2, cap);
            }
        st_scatter_layer(wp, r, sz, r2, Z, C);
    }
    for (int64_t row = 0; row < wp->nrows; row++) {
        int64_t a = 0, b = 0;
        for (int64_t x = 0; x < wp->ncols; x++) {
            a += Z[row * wp->ncols + x]; b += C[row * wp->ncols + x];
            Z[row * wp->ncols + x] = a; C[row * wp->ncols + x] = b;
        }
    }
    if (h) finalize_grid(wp, Z, C, h);
    rc = ORC_OK;
out:
    if (kd) for (int v = 0; v < nv; v++) if (cnt && cnt[v]) kd_free(&kd[v]);
    free(kd); free(cnt); free(sz); free(r2);
    if (!Zout) free(Z);
    if (!Cout) free(C);
    return rc;
}
