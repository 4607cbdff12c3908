/*
 * dnni.h -- C ABI of the B200 discrete natural-neighbour interpolation engine.
 *
 * This is the drop-in boundary for TerraNNI's hot path, the per-work-package
 * call nni::performNNI (nni.h:93-95, implemented nni.cpp:870-944) together
 * with the calls that bracket it (nni.h:83-97).  Plain pointers and sizes
 * only; every entry point returns a dnni_status; one context per host thread.
 *
 * Semantics (canonical mode; the reference approximates the same quantity
 * with GL rasterisation, nni.cpp:171-230 and nni.cpp:483-534):
 *   - points are int32 LAS-unit coordinates (x, y, z), n x 3, row-major, with
 *     an optional uint32 global id per point (NULL: the id is the index);
 *   - cell (i, j) of the output grid sits at LAS position
 *     (origin_x + i*cell_size, origin_y + j*cell_size); raster pixels use the
 *     same lattice (the reference's `scaling` is 1);
 *   - s(p), the nearest site of raster pixel p, minimises (d^2, gid, z) with
 *     d^2 computed exactly in int64 (ties go to the lowest global id);
 *   - every grid cell q with |q-p|^2 <= floor(d^2(p,s(p)) / cell_size^2)
 *     (cell-index units) receives z(s(p)) and a count of one;
 *   - h[q] = float((double)Z / (double)C * z_scale + z_offset), or nodata when
 *     no pixel reaches q.  Z is an exact int64 sum, so heights are
 *     deterministic and independent of launch order.
 *   Output grids are row-major, nrows x ncols, row 0 = smallest y.  The site
 *   map holds one gid per raster pixel (DNNI_NO_SITE when there are no points).
 *
 * Coordinates relative to (origin_x, origin_y) must lie within +-2^30 LAS
 * units for points and raster pixels; grid and raster sides are at most
 * 32767 cells.
 */
#ifndef DNNI_H
#define DNNI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DNNI_NO_SITE 0xFFFFFFFFu
#define DNNI_VERSION 10000

typedef enum dnni_status {
    DNNI_OK = 0,
    DNNI_E_INVAL = 1,      /* bad argument or work package */
    DNNI_E_NOMEM = 2,      /* device or host allocation failed / over budget */
    DNNI_E_TIMEOUT = 3,    /* a bounded wait expired */
    DNNI_E_CUDA = 4,       /* CUDA runtime error (see dnni_last_error) */
    DNNI_E_RANGE = 5,      /* coordinates outside the supported range */
    DNNI_E_STATE = 6,      /* call out of order (e.g. no setup) */
    DNNI_E_IO = 7,         /* file could not be read / parsed */
    DNNI_E_CANCELLED = 8,  /* request cancelled before completion */
    DNNI_E_BUSY = 9,       /* admission refused: no slot or memory free now */
    DNNI_E_SCRATCH = 10    /* work package needs more than the fixed scratch of
                              dnni_interpolate_segment_device_noalloc */
} dnni_status;

typedef struct dnni_ctx dnni_ctx;

/* Replaces nni::Settings (nni.h:72-81) for the engine.  The reference's
 * scale/site_radius/query_radius/zMultiplier fields have no counterpart in
 * canonical mode (scaling 1, unbounded discs, exact int64 sums). */
typedef struct dnni_settings {
    int32_t device;         /* CUDA device ordinal */
    int32_t small_radius;   /* pixels with floor(d^2/cell^2) <= r^2 use the
                               per-tile stencil, others the span scatter;
                               1..6, 0 = default (3) */
    int32_t bin_target;     /* mean points per search bin; 0 = default (4) */
    int32_t flags;          /* DNNI_F_* */
    uint64_t mem_budget;    /* bytes of device scratch a context may hold;
                               0 = no limit */
} dnni_settings;

#define DNNI_F_TIMING 1     /* record per-phase CUDA-event times in dnni_stats */

/* One work package: the output grid and the raster of pixels that scatter
 * into it.  Replaces nni::WorkPackage (nni.h:66-70), whose float origins are
 * replaced by int32 LAS units.  raster_* are cell indices relative to cell
 * (0,0), half-open; all four zero means "the grid itself". */
typedef struct dnni_workpackage {
    int32_t ncols, nrows;
    int32_t cell_size;              /* LAS units per cell edge, > 0 */
    int32_t origin_x, origin_y;     /* LAS position of cell (0,0) */
    int32_t raster_x0, raster_y0, raster_x1, raster_y1;
    int32_t pad0;
    double z_scale, z_offset;       /* metres = z_scale * LAS z + z_offset */
    float nodata;                   /* value for cells no pixel reaches */
    int32_t pad1;
} dnni_workpackage;

typedef struct dnni_stats {
    double ms_total;        /* device time of the call (CUDA events) */
    double ms_bin, ms_nearest, ms_scatter, ms_finalize;
    int64_t n_points, n_cells, n_pixels;
    int64_t big_pixels;     /* pixels scattered by the span path */
    int64_t spans;          /* row spans those pixels cover (unclipped) */
    int64_t nodata_cells;
    int64_t h2d_bytes, d2h_bytes;
    int32_t max_r2;         /* largest floor(d^2/cell^2) over the raster */
    int32_t packed;         /* 1 when (Z,C) shared one 64-bit accumulator */
    int32_t bin_size;       /* search-bin edge chosen, LAS units */
    int32_t pad;
    int64_t evals_dense;    /* candidate distance evaluations of the ring search */
    int64_t evals_far;      /* and of the far pass (seeds and disc search) */
    int64_t span_hist[16];  /* spans per radius bucket: bucket k holds the
                               span-path pixels with floor(sqrt(R2)) in
                               [2^(k-1), 2^k) (k = 15: all larger); filled
                               by statistics runs without a graph */
    double ms_dense;        /* of ms_nearest: the ring search (k_near_dense) */
    double ms_far;          /* and the far pass after it */
} dnni_stats;

/* ---- lifecycle: nni::init / nni::cleanup (nni.h:83-85, nni.cpp:563-598) ---- */

int32_t dnni_version(void);
/* Create a context bound to settings->device (NULL settings: defaults). */
dnni_status dnni_init(const dnni_settings *settings, dnni_ctx **out);
/* Release every device and host resource of the context. */
dnni_status dnni_destroy(dnni_ctx *ctx);
/* Message for the last failing call on this context ("" if none). */
const char *dnni_last_error(const dnni_ctx *ctx);

/* ---- per work package: nni::setupRun (nni.h:91, nni.cpp:601-668) ---- */

/* Optional: reserve device scratch for work packages up to this size and
 * point count, so that the first interpolate call does not allocate. */
dnni_status dnni_setup_run(dnni_ctx *ctx, const dnni_workpackage *wp, int64_t max_points);

/* ---- hot path: nni::performNNI (nni.h:93-95, nni.cpp:870-944) ---- */

/* Host buffers: copies the points in, interpolates, copies h (nrows*ncols
 * floats) and, if out_site is not NULL, the site map (raster pixels) out.
 * Returns after the results are in host memory. */
dnni_status dnni_interpolate_segment(dnni_ctx *ctx, const dnni_workpackage *wp,
                                     const int32_t *xyz, const uint32_t *gid, int64_t n,
                                     float *out_h, uint32_t *out_site, dnni_stats *stats);

/* Device buffers on the context's device.  Work is queued on `stream`
 * (a cudaStream_t; NULL = the context's own stream, a blocking stream
 * ordered with the legacy default stream).  The call synchronises
 * once, after the point bounding box, to size the search bins; it returns
 * with the remaining work queued unless stats is non-NULL, in which case it
 * waits for completion to fill the counters. */
dnni_status dnni_interpolate_segment_device(dnni_ctx *ctx, const dnni_workpackage *wp,
                                            const int32_t *d_xyz, const uint32_t *d_gid, int64_t n,
                                            float *d_h, uint32_t *d_site, void *stream,
                                            dnni_stats *stats);

/* ---- the same call without any allocation (no counterpart in the reference) ----
 *
 * For callers that cannot let a library call cudaMalloc or cudaFree: host
 * applications that own all device memory through their own pool and forbid
 * libraries from allocating (plug-in hosts with a fixed device budget), and
 * latency-critical callers that cannot absorb the implicit device-wide
 * synchronisation of those calls.  Needs no context.  All scratch comes from
 * one fixed 32 MiB device array compiled into this library; every GPU that
 * loads the library holds it until the process exits.
 *
 * Limit: the work package must fit that array, at about 12 B per grid cell +
 * 24 B per raster pixel + 16 B per point + 8.2 B per search bin (about one
 * bin per four points), each region rounded up to 256 B; e.g. a 512 x 512
 * grid with 500k points fits.  Larger work packages return DNNI_E_SCRATCH, before
 * any work is queued or, for the search bins (sized from the point bounding
 * box), right after the bounding-box pass.
 *
 * Runs on the calling thread's current device and queues on `stream`
 * (a cudaStream_t, NULL = the legacy default stream).  With n > 0 it waits
 * on `stream` once, for the points' bounding box (the search bins are sized
 * from it), and returns with the rest queued.  A point beyond +-2^30 LAS
 * units of the origin returns DNNI_E_RANGE after that wait; the bin-grid
 * check that the other calls report is not read back here, because a grid
 * planned from the measured bounding box holds every point.
 *
 * The first call on each device looks up the array's device address, with
 * that device current, and keeps it for the life of the process; make that
 * first call before any stream capture.  The address does not survive
 * cudaDeviceReset: after resetting a device, do not use this entry point on
 * it again in the same process.  Every call shares the one array and
 * overwrites what the previous call left in it (what must start at zero is
 * cleared on each call), so calls whose work overlaps on the GPU race:
 * serialise them, e.g. on one stream. */
dnni_status dnni_interpolate_segment_device_noalloc(const dnni_workpackage *wp, const int32_t *d_xyz,
                                                    const uint32_t *d_gid, int64_t n, float *d_h,
                                                    uint32_t *d_site, void *stream);

/* ---- batches: the loop of binRun (terranni.cpp:394-426) as one launch ----
 *
 * Many work packages ("tiles") of uneven size run through one launch sequence
 * whose kernels cover every tile; with use_graph the sequence is captured in a
 * CUDA graph on the first run and replayed afterwards.  Planning happens once,
 * at creation, from each tile's geometry and its declared point extent, so a
 * run never waits on the host. */
typedef struct dnni_tile {
    dnni_workpackage wp;
    int64_t pt_offset, pt_count;   /* the tile's points: rows [pt_offset,
                                      pt_offset + pt_count) of the xyz (and gid)
                                      arrays given to the run */
    int32_t ext_x0, ext_y0, ext_x1, ext_y1;  /* absolute LAS box (inclusive)
                                      holding every point of the tile; all zero
                                      = the raster; a point outside fails the
                                      run with DNNI_E_RANGE */
    int64_t out_offset;            /* first float of the tile's grid in the
                                      output array */
    int64_t site_offset;           /* first uint32 of its site map in the site
                                      array, -1 = none */
} dnni_tile;

typedef struct dnni_batch dnni_batch;

typedef struct dnni_batch_options {
    int32_t small_radius;          /* 0 = the context's setting */
    int32_t bin_target;            /* 0 = the context's setting */
    int32_t use_graph;             /* capture the launch sequence in a CUDA graph */
    int32_t order_by_cost;         /* schedule the largest tiles first */
    int32_t span_window;           /* 8-byte cells of shared memory per raster
                                      tile in which the span path merges its
                                      markers (256..26624), 1 = no window (every
                                      marker straight to the grid); 0 = default
                                      (4096) */
    int32_t far_group;             /* pixels the far pass searches together:
                                      1 = 32 x 1 rows, 2 = 8 x 4 blocks;
                                      0 = default (2) */
    int32_t dense_band;            /* ring search: rows of the 32-pixel-wide
                                      block that shares one bin window staged
                                      in shared memory (8, 16, 32 or 64; a
                                      window that does not fit halves it);
                                      0 = default (64) */
} dnni_batch_options;

/* Plans the tiles and allocates the batch's device scratch (allocates). */
dnni_status dnni_batch_create(dnni_ctx *ctx, const dnni_tile *tiles, int32_t ntiles,
                              const dnni_batch_options *options, dnni_batch **out);
/* Runs every tile on device buffers, queued on `stream` (NULL = the
 * context's stream, a blocking stream: ordered with the legacy default
 * stream).  Returns with the work queued unless stats is non-NULL,
 * in which case it waits, reports totals over the tiles (ms_total is the
 * device time of the run; per-phase times too when the batch runs without
 * a graph) and checks the points against the declared extents
 * (DNNI_E_RANGE); without stats that check is not read back. */
dnni_status dnni_batch_run_device(dnni_batch *batch, const int32_t *d_xyz, const uint32_t *d_gid,
                                  float *d_h, uint32_t *d_site, void *stream, dnni_stats *stats);
/* The same from host buffers: n_rows point rows are copied in, the output
 * (the largest out_offset + cells of the tiles) and site maps copied out;
 * always waits and checks the extents. */
dnni_status dnni_batch_run(dnni_batch *batch, const int32_t *xyz, const uint32_t *gid, int64_t n_rows,
                           float *out_h, uint32_t *out_site, dnni_stats *stats);
dnni_status dnni_batch_destroy(dnni_batch *batch);

/* ---- segment driver: one large grid in tiles with halos ----
 *
 * Replaces the reference's out-of-core pipeline around performNNI for one
 * grid: binning of the points into work packages with duplicated borders
 * (terranni.cpp:203-368, 271-302), the work-package loop of binRun
 * (terranni.cpp:394-426) and the assembly of the grid (terranni.cpp:430-488).
 * The points (absolute int32 LAS xyz, host memory, pinned for full copy
 * speed) are uploaded in chunks and bucketed by position on the device; the
 * grid is cut into tile x tile cell tiles, each interpolated with a raster
 * halo and a point halo, in batches.  After each batch every tile's largest
 * nearest-site distance is checked against its halo: a tile whose halo could
 * have missed a pixel whose disc reaches it, or a site nearer than the one
 * found, runs again with a larger halo.  The result (heights and site map,
 * gid = the point's index in the input) is therefore bit-identical to one
 * work package covering the whole grid with raster = grid. */
typedef struct dnni_segment {
    int32_t ncols, nrows;          /* the whole grid, cells (each side <= 2^20) */
    int32_t cell_size;             /* LAS units */
    int32_t origin_x, origin_y;    /* LAS position of cell (0,0) */
    int32_t tile;                  /* tile side in cells (0 = 2048) */
    int32_t halo;                  /* first raster halo tried, cells; 0 = per tile, from an
                                      upper bound of the nearest-site distance computed
                                      from the occupancy of 16-cell blocks */
    int32_t tiles_per_batch;       /* 0 = 64 */
    double z_scale, z_offset;
    float nodata;
    int32_t small_radius;          /* 0 = the context's setting */
    int32_t part, parts;           /* parts > 1: run only the tiles of part `part`
                                      (0 <= part < parts), a contiguous range of
                                      the row-major tiles balanced by cost
                                      (cells + points, dnni_partition_contiguous),
                                      and write only their cells; the other
                                      parts' calls, on other GPUs, fill the rest.
                                      0 or 1 = every tile */
} dnni_segment;

typedef struct dnni_segment_stats {
    double ms_total;               /* wall time of the call */
    double ms_upload, ms_bucket;   /* host->device copy, device bucketing */
    double ms_bound;               /* occupancy distance transform and halo planning (host) */
    double ms_tiles;               /* the tile batches, planning, launches and copies included */
    int64_t points, cells, tiles;
    int64_t tile_runs;             /* tiles + reruns with a larger halo */
    int64_t h2d_bytes, d2h_bytes;
    int32_t max_halo;              /* largest raster halo any tile needed */
    int32_t batches;               /* launch sequences run */
} dnni_segment_stats;

/* Splits n items with non-negative costs into `parts` contiguous ranges of
 * about equal total cost: part p is [first[p], first[p+1]), first[0] = 0,
 * first[parts] = n.  Host code only (no device needed); the same inputs give
 * the same ranges on every rank. */
dnni_status dnni_partition_contiguous(const int64_t *cost, int32_t n, int32_t parts, int32_t *first);

/* h_out: nrows x ncols floats, row-major, row 0 = lowest y; h_site (optional):
 * nrows x ncols uint32 site ids. */
dnni_status dnni_segment_run(dnni_ctx *ctx, const dnni_segment *seg, const int32_t *h_xyz, int64_t n,
                             float *h_out, uint32_t *h_site, dnni_segment_stats *stats);

/* ---- serving: DEM requests against a resident point cloud ----
 *
 * No counterpart in the reference (its CLI interpolates one whole dataset per
 * run, terranni.cpp:544-700).  dnni_server_create uploads and buckets a
 * point cloud once and keeps it in HBM; requests (a bounding box at a cell
 * size) are submitted at any time from any thread and run by a server thread
 * with continuous batching: queued requests are admitted in arrival order
 * into the next batch while their device footprint fits a free slot's arena,
 * and up to `slots` batches are in flight at once on separate streams.
 *
 * A request's result is the window of the interpolation whose raster is the
 * cloud's bounding box on the request's cell lattice, with every point of
 * the cloud as a site: its raster halo and point box come from an upper bound
 * of the nearest-site distance (exact distance transform of the occupancy of
 * fine blocks) and are checked after the run as in dnni_segment_run (a
 * request that fails the check runs again with a larger halo).  So a result
 * does not depend on which other requests share its batch. */
typedef struct dnni_server_options {
    int32_t bucket;                /* bucket side, LAS units (0 = 25600) */
    int32_t fine;                  /* fine block side of the halo bound, LAS units
                                      (0 = at least 1600, at most 4096 blocks a side) */
    int32_t slots;                 /* batches in flight (0 = 2) */
    int32_t max_batch;             /* requests per batch (0 = 64) */
    uint64_t slot_bytes;           /* device arena of each slot (0 = 16 GiB) */
    int32_t small_radius, bin_target;   /* 0 = the context's settings */
} dnni_server_options;

typedef struct dnni_server dnni_server;

typedef struct dnni_request {
    int32_t x0, y0;                /* absolute LAS position of cell (0,0) */
    int32_t ncols, nrows;          /* cells, each side <= 32767 */
    int32_t cell_size;             /* LAS units */
    int32_t pad0;
    double z_scale, z_offset;
    float nodata;
    int32_t pad1;
    float *out_h;                  /* host, nrows x ncols; must stay valid until the wait */
    uint32_t *out_site;            /* optional host site map, nrows x ncols */
} dnni_request;

typedef struct dnni_request_result {
    int32_t status;                /* DNNI_OK or why the request failed */
    int32_t halo;                  /* raster halo used, cells */
    double ms_queue;               /* submit -> launch */
    double ms_latency;             /* submit -> result in host memory */
    int64_t points, cells;
    int32_t batch_size, runs;      /* requests in its batch; runs (1 + reruns) */
} dnni_request_result;

typedef struct dnni_server_stats {
    int64_t submitted, completed, failed, batches, cells, points;
    int64_t resident_bytes;        /* the bucketed cloud */
    double ms_build;               /* upload, bucketing and bound at creation */
    double ms_device_busy;         /* device time with at least one batch running */
    double ms_device_overlap;      /* of it, time with two or more batches (slots) at once */
    double ms_device_span;         /* first batch start to last batch end */
} dnni_server_stats;

dnni_status dnni_server_create(dnni_ctx *ctx, const int32_t *h_xyz, int64_t n, const dnni_server_options *options,
                               dnni_server **out);
/* Queues a request; returns at once with its ticket. Thread-safe. */
dnni_status dnni_server_submit(dnni_server *srv, const dnni_request *req, uint64_t *ticket);
/* Waits up to timeout_s (< 0: forever) for the ticket's result; DNNI_E_TIMEOUT
 * leaves the ticket pending.  Each ticket is waited for once. Thread-safe. */
dnni_status dnni_server_wait(dnni_server *srv, uint64_t ticket, double timeout_s, dnni_request_result *result);
dnni_status dnni_server_get_stats(dnni_server *srv, dnni_server_stats *stats);
/* Finishes the queued requests, stops the server thread, frees the cloud. */
dnni_status dnni_server_destroy(dnni_server *srv);

/* ---- autotuning of the batch options (no counterpart in the reference) ----
 *
 * Times candidate settings, by coordinate search, of the search-bin size
 * (bin_target: points per bin), the split between the stencil path and the
 * span path (small_radius: discs up to this radius are gathered by the
 * stencil, larger ones spill into row spans), the span path's shared-memory
 * window (span_window), the far pass's pixel groups (far_group) and the
 * ring search's pixel-block shape (dense_band: 32 x 8..64 pixels per staged
 * bin window) on a sample of the tiles stratified by size, on device buffers
 * that already hold the points, and writes the fastest settings into
 * *options (use_graph and order_by_cost are left as given).  Results do not
 * depend on any of these settings; only the time does. */
typedef struct dnni_tune_trial {
    int32_t small_radius, bin_target;
    float ms;                          /* device time of one run of the sample */
    int32_t span_window, far_group, dense_band;
} dnni_tune_trial;

typedef struct dnni_tune_report {
    int32_t ntrials, best, sample_tiles, pad;
    double ms_default;                 /* the sample at the settings given on entry */
    dnni_tune_trial trial[32];
} dnni_tune_report;

dnni_status dnni_batch_autotune(dnni_ctx *ctx, const dnni_tile *tiles, int32_t ntiles, const int32_t *d_xyz,
                                const uint32_t *d_gid, int32_t sample_tiles, dnni_batch_options *options,
                                dnni_tune_report *report);

/* ---- the reference's default semantics (compatibility mode) ----
 *
 * nni::performNNI as the reference computes it by default (timeRadius 0,
 * plane algorithm; nni.cpp:870-944, cuda_nni.cu:407-503), on the GPU: each
 * site covers only a square of half-side site_radius/sqrt(2) on a pixel
 * lattice `scale` times finer than the cells (nni.cpp:183, 879-886); in it
 * the site's float32 lifted plane competes by depth, the later-drawn site
 * winning equal depths (GL_LEQUAL, nni.cpp:171-230, 733-737); each cell
 * collects, over its square of half-side query_radius/sqrt(2), the z-codes
 * floor((z - point_min + 1) * multiplier) of the pixels where its own plane
 * is no deeper (nni.cpp:483-534, 538-549), sums them in int32 with
 * wrap-around and truncates the division (cuda_nni.cu:423-503); heights are
 * dequantised as nni.cpp:836-848 does (-9999 where no pixel counts).
 * Planes are evaluated at pixel centres over half-open squares; the GL
 * rasteriser's fill rule and depth interpolation are not reproduced.  Points
 * are world coordinates (x, y, z doubles) in draw order; res_out (optional)
 * receives the int32 division results.  Heights are row-major, row 0 the
 * lowest y. */
typedef struct dnni_compat_settings {   /* nni::Settings (nni.h:72-81), the fields used */
    int32_t scale;
    float cell_size;
    float site_radius;
    int32_t pad0;
    double query_radius;
    int32_t point_min;
    int32_t multiplier;                 /* zMult (terranni.cpp:675-684) */
    int32_t total_ncols, total_nrows;
} dnni_compat_settings;

typedef struct dnni_compat_wp {         /* nni::WorkPackage (nni.h:66-70) */
    float origin_x, origin_y, grid_origin_x, grid_origin_y;
    int32_t nrows, ncols;
} dnni_compat_wp;

dnni_status dnni_interpolate_compat(dnni_ctx *ctx, const dnni_compat_settings *settings, const dnni_compat_wp *wp,
                                    const double *xyz, int64_t n, float *h_out, int32_t *res_out);
/* The same on device buffers, queued on `stream` (NULL = the context's
 * stream); returns with the work queued. */
dnni_status dnni_interpolate_compat_device(dnni_ctx *ctx, const dnni_compat_settings *settings,
                                           const dnni_compat_wp *wp, const double *d_xyz, int64_t n, float *d_h,
                                           int32_t *d_res, void *stream);

/* ---- space-time interpolation: nni::performNNI with timeRadius > 0 ----
 *
 * Replaces the slice loop of nni::performNNI (nni.cpp:902-933) with its
 * per-slice site drawing (nni.cpp:722-790; drawPlane's time term,
 * nni.cpp:171-230) and query drawing lifted by the slice offset
 * (nni.cpp:483-493), in the canonical semantics of the 2-D path:
 *   slices ts = cur_time + j, j = -time_radius .. time_radius;
 *   the sites of slice ts are the points whose time t has |ts - t| <=
 *   time_radius (nni.cpp:770), each at lifted squared distance
 *   dx^2 + dy^2 + ((ts - t) * time_scale)^2 from a pixel (time_scale = LAS
 *   units per time step; the reference's GL units make one time step one
 *   metre); a pixel's site is the lifted-nearest one, ties to the lower
 *   input index (the earlier point of the stream);
 *   cell q (at cur_time) takes pixel p of slice ts iff
 *   |q - p|^2 * cell^2 + (j * time_scale)^2 <= that lifted distance;
 *   Z and C are summed over every slice; h as in the 2-D path.
 * time_radius = 0 gives exactly dnni_interpolate_segment over the points
 * with t == cur_time.  Points whose time is farther than 2 * time_radius from
 * cur_time take part in no slice and may be passed or left out.
 * Limits: 0 <= time_radius <= 16, time_scale > 0,
 * time_radius * time_scale <= 2^30; (2 * time_radius + 1) x raster pixels
 * < 2^31. */
typedef struct dnni_st_options {
    int32_t cur_time;       /* curTime of nni::performNNI (integer times) */
    int32_t time_radius;    /* timeRadius (terranni --time-radius) */
    int32_t time_scale;     /* LAS units per time step in the lifted distance */
    int32_t pad;
} dnni_st_options;

dnni_status dnni_interpolate_spacetime(dnni_ctx *ctx, const dnni_workpackage *wp, const dnni_st_options *opt,
                                       const int32_t *xyz, const int32_t *t, int64_t n, float *h_out,
                                       dnni_stats *stats);
/* The same on device buffers (points, times and heights on the context's
 * device), queued on `stream` (NULL = the context's stream); the call waits
 * once, for the per-time-value counts that size the batch, and returns with
 * the rest queued unless stats is non-NULL. */
dnni_status dnni_interpolate_spacetime_device(dnni_ctx *ctx, const dnni_workpackage *wp, const dnni_st_options *opt,
                                              const int32_t *d_xyz, const int32_t *d_t, int64_t n, float *d_h,
                                              void *stream, dnni_stats *stats);

/* ---- input: LAS point files ----
 *
 * Replaces the reference's nni_io::las_reader (las_reader.h:34-58,
 * las_reader.inl:25-84, on libLAS 1.6) for the engine's input: the public
 * LAS layout (1.0-1.4, point formats 0-10, uncompressed) read directly.
 * dnni_las_read returns the records' raw X, Y, Z integers -- the engine's
 * int32 LAS units, position = integer * scale + offset from the header --
 * for records [first, first + count), parsed on nthreads host threads
 * (0 = all cores), optionally with each record's intensity (which the
 * reference reads as the point's time, las_reader.inl:64). */
typedef struct dnni_las_header {
    uint8_t version_major, version_minor, point_format, pad0;
    uint16_t record_length, pad1;
    uint32_t offset_to_points;
    uint64_t n_points;
    double scale[3], offset[3], min[3], max[3];
} dnni_las_header;

dnni_status dnni_las_read_header(const char *path, dnni_las_header *header);
dnni_status dnni_las_read(const char *path, int64_t first, int64_t count, int32_t *xyz, uint16_t *intensity,
                          int32_t nthreads);
/* Writes n points as a LAS 1.2 file of point format 0 (for fixtures and
 * exchange); scale/offset: 3 doubles each (NULL = 0.01 and 0). */
dnni_status dnni_las_write(const char *path, const int32_t *xyz, const uint16_t *intensity, int64_t n,
                           const double *scale, const double *offset);

/* ---- output: grids ----
 *
 * dnni_write_asc writes an ESRI ASCII grid as the reference's outputASC does
 * (terranni.cpp:428-488): header NROWS, NCOLS, XLLCORNER, YLLCORNER,
 * CELLSIZE, NODATA_VALUE, then one line per grid row from the top (highest
 * y) row, each value in 6 significant digits followed by a space.  The grid
 * is row-major with row 0 the lowest y, as the engine writes it, so no sort
 * of an OutPoint stream is needed; corner and cell size are printed in 10
 * significant digits (the reference's stream default of 6 rounds UTM
 * coordinates).  dnni_write_grid_bin writes a 64-byte header ("DNNIGRD1",
 * ncols, nrows as int32, xll, yll, cellsize as double, nodata as float, zero
 * padding) and the float32 cells row-major from row 0. */
dnni_status dnni_write_asc(const char *path, const float *h, int32_t ncols, int32_t nrows, double xll, double yll,
                           double cellsize, float nodata, int32_t nthreads);
dnni_status dnni_write_grid_bin(const char *path, const float *h, int32_t ncols, int32_t nrows, double xll,
                                double yll, double cellsize, float nodata);

/* ---- nni::clearRenderbuffers / nni::printTimes (nni.h:87-97) ---- */

/* Free the context's scratch (it is re-created on demand). */
dnni_status dnni_clear(dnni_ctx *ctx);
/* Print accumulated per-phase device times to stdout (needs DNNI_F_TIMING). */
dnni_status dnni_print_times(dnni_ctx *ctx);

/* ---- measured peaks of the operations that bound the hot path ----
 *
 * Calibration beside dnni::printTimes (nni.cpp:554-560): the throughput this
 * device reaches on the operations that bound the hot path's kernels, each
 * from a microbenchmark kernel timed with CUDA events on every SM: 32-bit
 * integer multiply-adds (the distance evaluations of the nearest-site
 * search), conflict-free 32-bit shared-memory atomic adds (the span
 * window's markers) and coalesced 64-bit global atomic adds on an
 * L2-resident buffer (the window's flush and the direct span path).  The
 * op-count rooflines divide the kernels' counted work by these.  Allocates
 * about 32 MB for the duration of the call. */
typedef struct dnni_peaks {
    double int_ops_per_s;          /* lane multiply-adds per second */
    double smem_atomics_per_s;     /* lane atomic adds per second */
    double l2_red64_per_s;         /* lane atomic adds per second */
    double sm_clock_mhz;           /* the device's nominal SM clock */
    int32_t sm_count, pad;
} dnni_peaks;

dnni_status dnni_measure_peaks(int32_t device, dnni_peaks *out);

/* ---- pinned host memory for the host-buffer entry points ---- */

dnni_status dnni_host_alloc(size_t bytes, void **out);
dnni_status dnni_host_free(void *p);

#ifdef __cplusplus
}
#endif

#endif /* DNNI_H */
