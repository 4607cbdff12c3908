// dnni_engine.cu -- context, device scratch, batch planning and the launch
// sequence behind the C ABI in include/dnni.h.
//
// Reference counterparts:
//   nni::init / cuda_nni::init          nni.cpp:569-598, cuda_nni.cu:641-669
//   nni::setupRun / cuda_nni::setup_run nni.cpp:601-668, cuda_nni.cu:110-126
//   nni::performNNI                     nni.cpp:870-944
//   nni::clearRenderbuffers / cleanup   nni.cpp:362-379, 563-566
//   nni::printTimes                     nni.cpp:554-560
//   binRun's loop over work packages    terranni.cpp:394-426 (the batch API)
// The GL context, framebuffers, renderbuffers and GL/CUDA interop of the
// reference have no counterpart: the engine works on plain device buffers.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>

#include "../../include/dnni.h"
#include "dnni_internal.h"

using namespace dnni;

namespace {

dnni_status set_err(dnni_ctx* c, dnni_status st, const std::string& msg) {
    if (c) c->err = msg;
    return st;
}

dnni_status cuda_err(dnni_ctx* c, cudaError_t e, const char* what) {
    return set_err(c, DNNI_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_err(c, e_, #call);     \
    } while (0)

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

// Every scratch array a batch needs, in bytes.
struct ScratchSizes {
    size_t sorted, cnt, bsum, bmask, smask, rownear, near, pix, far, D, Dc, sc, ctr, tables;
};

ScratchSizes scratch_sizes(const HostBatch& hb) {
    const int n = (int)hb.tiles.size();
    ScratchSizes z;
    z.sorted = sizeof(int4) * std::max<int64_t>(hb.n_pts, 1);
    z.cnt = sizeof(int) * std::max<int64_t>(hb.n_bins, 1);
    z.bsum = sizeof(int) * std::max<int64_t>(hb.scan_base.back(), 1);
    z.bmask = sizeof(uint64_t) * std::max<int64_t>(hb.blk_base.back(), 1);
    z.smask = sizeof(uint64_t) * std::max<int64_t>(hb.sup_base.back(), 1);
    z.rownear = sizeof(int) * std::max<int64_t>(hb.blk_base.back(), 1);
    z.near = sizeof(int64_t) * std::max<int64_t>(hb.blk_base.back(), 1);
    z.pix = sizeof(int2) * std::max<int64_t>(hb.n_pix, 1);
    z.far = sizeof(FarSlot) * std::max<int64_t>(hb.n_far, 1);
    z.D = sizeof(unsigned long long) * std::max<int64_t>(hb.n_cells, 1);
    z.Dc = sizeof(int) * std::max<int64_t>(hb.n_cells, 1);
    z.sc = sizeof(Scalars) * n;
    z.ctr = sizeof(BatchCounters);
    z.tables = TableLayout(n).total;
    return z;
}

dnni_status ensure_scratch(dnni_ctx* c, Scratch& s, const ScratchSizes& z, DevArrays& a) {
    dnni_status rs;
    if ((rs = dnni_ensure(c, s.sorted, z.sorted)) || (rs = dnni_ensure(c, s.cnt, z.cnt)) || (rs = dnni_ensure(c, s.start, z.cnt)) ||
        (rs = dnni_ensure(c, s.bsum, z.bsum)) || (rs = dnni_ensure(c, s.bmask, z.bmask)) ||
        (rs = dnni_ensure(c, s.smask, z.smask)) || (rs = dnni_ensure(c, s.rownear, z.rownear)) ||
        (rs = dnni_ensure(c, s.near, z.near)) || (rs = dnni_ensure(c, s.pix, z.pix)) ||
        (rs = dnni_ensure(c, s.far, z.far)) || (rs = dnni_ensure(c, s.D, z.D)) || (rs = dnni_ensure(c, s.Dc, z.Dc)) ||
        (rs = dnni_ensure(c, s.sc, z.sc)) || (rs = dnni_ensure(c, s.ctr, z.ctr)) ||
        (rs = dnni_ensure(c, s.tables, z.tables)))
        return rs;
    a.sorted = (int4*)s.sorted.p;
    a.cnt = (int*)s.cnt.p;
    a.start = (int*)s.start.p;
    a.bsum = (int*)s.bsum.p;
    a.bmask = (uint64_t*)s.bmask.p;
    a.smask = (uint64_t*)s.smask.p;
    a.rownear = (int*)s.rownear.p;
    a.near = (int64_t*)s.near.p;
    a.pix = (int2*)s.pix.p;
    a.far = (FarSlot*)s.far.p;
    a.D = (unsigned long long*)s.D.p;
    a.Dc = (int*)s.Dc.p;
    a.sc = (Scalars*)s.sc.p;
    a.ctr = (BatchCounters*)s.ctr.p;
    a.tables = (unsigned char*)s.tables.p;
    return DNNI_OK;
}

void release_scratch(dnni_ctx* c, Scratch& s) {
    DevBuf* bufs[] = {&s.sorted, &s.list, &s.cnt, &s.start, &s.bsum, &s.bmask, &s.smask, &s.rownear,
                      &s.near, &s.pix, &s.far, &s.D, &s.Dc, &s.sc, &s.ctr, &s.tables};
    for (DevBuf* b : bufs) dnni_release(*b, c);
}

// Row scan, stencil and finalize, for the batch's stencil radius.
void launch_rows_final(const BatchTables& bt, int ncta, int rs, const int2* pix, Scalars* sc,
                       const unsigned long long* S, const int* Sc, float* h, cudaStream_t st) {
    dim3 blk(32, 16);
    switch (rs) {
        case 1: k_rows_final<1><<<ncta, blk, 0, st>>>(bt, pix, sc, S, Sc, h); break;
        case 2: k_rows_final<2><<<ncta, blk, 0, st>>>(bt, pix, sc, S, Sc, h); break;
        case 4: k_rows_final<4><<<ncta, blk, 0, st>>>(bt, pix, sc, S, Sc, h); break;
        case 5: k_rows_final<5><<<ncta, blk, 0, st>>>(bt, pix, sc, S, Sc, h); break;
        case 6: k_rows_final<6><<<ncta, blk, 0, st>>>(bt, pix, sc, S, Sc, h); break;
        default: k_rows_final<3><<<ncta, blk, 0, st>>>(bt, pix, sc, S, Sc, h); break;
    }
}

void set_dense_smem_attr() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && !done[dev]) {
        cudaFuncSetAttribute(k_near_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDenseSmem);
        cudaFuncSetAttribute(k_scatter_window, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(unsigned long long) * kSpanWindowMaxWords));
        done[dev] = true;
    }
}

// Launch sequence, part 1: per-tile scalars and (with bbox) the point
// bounding boxes, which a single work package needs before its bins are
// planned; batches pass bbox = false and have k_bin_count take the boxes.
void launch_prologue(const HostBatch& hb, const BatchTables& bt, const DevArrays& a, const int32_t* d_xyz,
                     cudaStream_t st, bool bbox = true) {
    const int n = (int)hb.tiles.size();
    k_init_scalars<<<n, 32, 0, st>>>(bt, a.sc, a.ctr);
    const int nchunk = hb.chunk_base.back();
    if (bbox && nchunk > 0) k_bbox<<<nchunk, 256, 0, st>>>(bt, d_xyz, a.sc, a.ctr);
}

// Launch sequence, part 2: binning, nearest sites, spans, stencil, finalize.
// Needs no host synchronisation (a batch's whole sequence can be captured).
// ev[0..2] (optional) mark the ends of binning, nearest sites and spans, and
// ev[4] the end of the ring search (k_near_dense) inside the nearest sites.
// sites_only: stop after the nearest-site kernels (the site map is the result).
void launch_body(const HostBatch& hb, const BatchTables& bt, const DevArrays& a, const int32_t* d_xyz,
                 const uint32_t* d_gid, float* d_h, uint32_t* d_site, int sms, cudaStream_t st,
                 const cudaEvent_t* ev, bool bbox_in_count = false, bool sites_only = false) {
    const int nchunk = hb.chunk_base.back();
    const int64_t nblk = hb.blk_base.back(), nsup = hb.sup_base.back();
    if (nchunk > 0) {
        cudaMemsetAsync(a.cnt, 0, sizeof(int) * hb.n_bins, st);
        k_bin_count<<<nchunk, 256, 0, st>>>(bt, d_xyz, a.cnt, a.sc, a.ctr, bbox_in_count ? 1 : 0);
        const int nscan = hb.scan_base.back();
        k_scan_partial<<<nscan, kScanThreads, 0, st>>>(bt, a.cnt, a.bsum);
        k_scan_bsum<<<(int)hb.tiles.size(), 1024, 0, st>>>(bt, a.bsum);
        k_scan_final<<<nscan, kScanThreads, 0, st>>>(bt, a.cnt, a.bsum, a.start);
        k_bin_scatter<<<nchunk, 256, 0, st>>>(bt, d_xyz, d_gid, a.start, a.cnt, a.sorted);
        if (nblk > 0) k_block_masks<<<(int)((nblk * 32 + 255) / 256), 256, 0, st>>>(bt, a.start, a.bmask);
        if (nsup > 0) k_super_masks<<<(int)((nsup * 32 + 255) / 256), 256, 0, st>>>(bt, a.bmask, a.smask);
        const int nrow1 = hb.row1_base.back();
        if (nrow1 > 0) k_block_rows<<<(nrow1 + 127) / 128, 128, 0, st>>>(bt, a.bmask, a.rownear);
        if (nblk > 0) k_block_near<<<(int)((nblk + 255) / 256), 256, 0, st>>>(bt, a.rownear, a.near);
    }
    if (ev) cudaEventRecord(ev[0], st);
    const int nrt = hb.rt_base.back();
    k_near_dense<<<nrt, dim3(32, 8), kDenseSmem, st>>>(bt, a.sorted, a.start, a.pix, d_site, a.far, a.sc, a.ctr,
                                                       hb.far_blocks, hb.dense_band);
    if (ev) cudaEventRecord(ev[4], st);
    if (nchunk > 0)
        k_near_far<<<sms * 6, 256, 0, st>>>(bt, a.sorted, a.start, a.bmask, a.smask, a.near, a.far, a.pix, d_site,
                                            a.sc, a.ctr);
    if (sites_only) return;
    k_decide<<<(int)hb.tiles.size(), 32, 0, st>>>(bt, a.sc);
    if (ev) cudaEventRecord(ev[1], st);
    cudaMemsetAsync(a.D, 0, sizeof(unsigned long long) * hb.n_cells, st);
    cudaMemsetAsync(a.Dc, 0, sizeof(int) * hb.n_cells, st);
    k_scatter_window<<<nrt, dim3(32, 8), sizeof(unsigned long long) * hb.win_words, st>>>(bt, a.pix, a.sc, a.D,
                                                                                         a.Dc, hb.win_words);
    if (ev) cudaEventRecord(ev[2], st);
    launch_rows_final(bt, hb.band_base.back(), hb.rs, a.pix, a.sc, a.D, a.Dc, d_h, st);
}

// Sums the per-tile scalars into dnni_stats.
void fold_stats(const Scalars* s, int n, dnni_stats* st) {
    int64_t big = 0, sp = 0, nod = 0, evd = 0, evf = 0;
    int mx = -1, packed = 1;
    for (int k = 0; k < kSpanHistBuckets; ++k) st->span_hist[k] = 0;
    for (int t = 0; t < n; ++t) {
        for (int k = 0; k < kStatSlots; ++k) {
            big += (int64_t)s[t].big_pixels[k];
            sp += (int64_t)s[t].spans[k];
            nod += (int64_t)s[t].nodata[k];
            evd += (int64_t)s[t].evals_dense[k];
            evf += (int64_t)s[t].evals_far[k];
            mx = std::max(mx, s[t].max_r2[k]);
        }
        for (int k = 0; k < kSpanHistBuckets; ++k) st->span_hist[k] += (int64_t)s[t].span_hist[k];
        packed &= s[t].packed;
    }
    st->big_pixels = big;
    st->spans = sp;
    st->nodata_cells = nod;
    st->evals_dense = evd;
    st->evals_far = evf;
    st->max_r2 = mx;
    st->packed = packed;
}

// Uploads a batch's tables through the context's pinned staging buffer.
dnni_status stage_tables(dnni_ctx* c, const HostBatch& hb, unsigned char* d_tables, cudaStream_t st) {
    const size_t bytes = TableLayout((int)hb.tiles.size()).total;
    // the previous upload from the staging buffer must have completed
    CK(cudaStreamSynchronize(st));
    if (bytes > c->h_tables_cap) {
        if (c->h_tables) cudaFreeHost(c->h_tables);
        c->h_tables = nullptr;
        c->h_tables_cap = 0;
        if (cudaMallocHost((void**)&c->h_tables, bytes) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, DNNI_E_NOMEM, "pinned staging for the tile tables");
        }
        c->h_tables_cap = bytes;
    }
    pack_tables(hb, c->h_tables);
    CK(cudaMemcpyAsync(d_tables, c->h_tables, bytes, cudaMemcpyHostToDevice, st));
    return DNNI_OK;
}

}  // namespace

dnni_status dnni_ensure(dnni_ctx* c, DevBuf& b, size_t bytes) {
    if (bytes <= b.cap) return DNNI_OK;
    size_t want = bytes + bytes / 4;
    want = (want + 255) & ~(size_t)255;
    if (c->s.mem_budget) {
        if (c->held - b.cap + want > c->s.mem_budget) want = (bytes + 255) & ~(size_t)255;
        if (c->held - b.cap + want > c->s.mem_budget)
            return set_err(c, DNNI_E_NOMEM, "device scratch would exceed the context's mem_budget");
    }
    if (b.p) {
        cudaDeviceSynchronize();   // work queued on any stream may still use it
        cudaFree(b.p);
        c->held -= b.cap;
        b.p = nullptr;
        b.cap = 0;
    }
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return set_err(c, DNNI_E_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
    b.cap = want;
    c->held += want;
    return DNNI_OK;
}

void dnni_release(DevBuf& b, dnni_ctx* c) {
    if (b.p) {
        cudaFree(b.p);
        c->held -= b.cap;
    }
    b.p = nullptr;
    b.cap = 0;
}

// The plain per-work-package call: a batch of one.  The bin grid is planned
// from the points' bounding box, which costs one synchronisation.
static dnni_status run_device(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* d_xyz, const uint32_t* d_gid,
                              int64_t n, float* d_h, uint32_t* d_site, cudaStream_t st, dnni_stats* stats) {
    TileParams t;
    const char* msg = "";
    dnni_status rs = plan_geometry(wp, n, c->s.small_radius, t, &msg);
    if (rs) return set_err(c, rs, msg);
    if (!d_h) return set_err(c, DNNI_E_INVAL, "output grid pointer is NULL");
    if (n > 0 && !d_xyz) return set_err(c, DNNI_E_INVAL, "point pointer is NULL");
    t.has_gid = d_gid ? 1 : 0;
    const bool timing = stats || (c->s.flags & DNNI_F_TIMING);
    // provisional plan (geometry only) for the bounding-box pass
    int32_t bb[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN};
    plan_bins(bb, 0, c->s.bin_target, t);
    HostBatch hb;
    hb.rs = c->s.small_radius;
    batch_add(hb, t, 0, 0, d_site ? 0 : -1);
    DevArrays a;
    if ((rs = ensure_scratch(c, c->scr, scratch_sizes(hb), a))) return rs;
    BatchTables bt = device_tables(a.tables, 1);
    if ((rs = stage_tables(c, hb, a.tables, st))) return rs;
    if (timing) CK(cudaEventRecord(c->ev[0], st));
    launch_prologue(hb, bt, a, d_xyz, st);
    CK(cudaGetLastError());
    if (n > 0) {
        CK(cudaMemcpyAsync(c->h_sc, a.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c->h_sc->err & kErrRange)
            return set_err(c, DNNI_E_RANGE, "a point lies beyond +-2^30 LAS units of the work-package origin");
        plan_bins(c->h_sc->bbox, n, c->s.bin_target, t);
        hb = HostBatch();
        hb.rs = c->s.small_radius;
        batch_add(hb, t, 0, 0, d_site ? 0 : -1);
        if ((rs = ensure_scratch(c, c->scr, scratch_sizes(hb), a))) return rs;
        bt = device_tables(a.tables, 1);
        if ((rs = stage_tables(c, hb, a.tables, st))) return rs;
    }
    launch_body(hb, bt, a, d_xyz, d_gid, d_h, d_site, c->sm_count, st, timing ? &c->ev[1] : nullptr);
    CK(cudaGetLastError());
    if (timing) CK(cudaEventRecord(c->ev[4], st));
    if (stats) k_span_hist<<<hb.rt_base.back(), dim3(32, 8), 0, st>>>(bt, a.pix, a.sc);
    c->calls++;
    if (timing) {
        CK(cudaEventSynchronize(c->ev[4]));
        float ms[4];
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ms[k], c->ev[k], c->ev[k + 1]);
        for (int k = 0; k < 4; ++k) c->acc_ms[k] += ms[k];
        if (stats) {
            stats->ms_bin = ms[0];
            stats->ms_nearest = ms[1];
            stats->ms_scatter = ms[2];
            stats->ms_finalize = ms[3];
            stats->ms_total = ms[0] + ms[1] + ms[2] + ms[3];
            float md = 0;
            cudaEventElapsedTime(&md, c->ev[1], c->ev[5]);
            stats->ms_dense = md;
            stats->ms_far = ms[1] - md;
        }
    }
    if (stats) {
        CK(cudaMemcpyAsync(c->h_sc, a.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(c->h_ctr, a.ctr, sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c->h_ctr->err & kErrRange) return set_err(c, DNNI_E_RANGE, "a point lies outside the search-bin grid");
        stats->n_points = n;
        stats->n_cells = (int64_t)t.ncols * t.nrows;
        stats->n_pixels = (int64_t)t.rw * t.rh;
        fold_stats(c->h_sc, 1, stats);
        stats->bin_size = t.bg.bs;
    }
    return DNNI_OK;
}

// Plans a batch: every tile from its geometry and declared point extent, in
// cost order when asked.  order[k] = the caller's index of batch position k.
static dnni_status plan_batch(dnni_ctx* c, const dnni_tile* tiles, int32_t ntiles, const dnni_batch_options& o,
                              HostBatch& hb, std::vector<int>& order) {
    const int rs_ = o.small_radius ? o.small_radius : c->s.small_radius;
    const int bt_ = o.bin_target ? o.bin_target : c->s.bin_target;
    const int ww_ = o.span_window ? o.span_window : kSpanWindowWords;
    if (rs_ < 1 || rs_ > kMaxSmallRadius || bt_ < 0 || (ww_ != 1 && ww_ < 256) || ww_ > kSpanWindowMaxWords ||
        o.far_group < 0 || o.far_group > 2 ||
        (o.dense_band != 0 && o.dense_band != 8 && o.dense_band != 16 && o.dense_band != 32 && o.dense_band != 64))
        return set_err(c, DNNI_E_INVAL, "bad batch options");
    const int fb_ = o.far_group ? o.far_group - 1 : kFarBlocksDefault;
    const int db_ = o.dense_band ? o.dense_band : kTileY;
    std::vector<TileParams> plan(ntiles);
    std::vector<int64_t> cost(ntiles);
    for (int k = 0; k < ntiles; ++k) {
        const dnni_tile& d = tiles[k];
        const char* msg = "";
        dnni_status rs = plan_geometry(&d.wp, d.pt_count, rs_, plan[k], &msg);
        if (rs) return set_err(c, rs, std::string("tile ") + std::to_string(k) + ": " + msg);
        if (d.pt_offset < 0 || d.pt_count < 0 || d.out_offset < 0)
            return set_err(c, DNNI_E_INVAL, "negative tile offset");
        int32_t bb[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, 0, 0};
        if (d.ext_x0 || d.ext_y0 || d.ext_x1 || d.ext_y1) {
            const long long ex0 = (long long)d.ext_x0 - d.wp.origin_x, ex1 = (long long)d.ext_x1 - d.wp.origin_x;
            const long long ey0 = (long long)d.ext_y0 - d.wp.origin_y, ey1 = (long long)d.ext_y1 - d.wp.origin_y;
            if (ex1 < ex0 || ey1 < ey0) return set_err(c, DNNI_E_INVAL, "empty point extent");
            if (ex0 <= -kCoordLimit || ex1 >= kCoordLimit || ey0 <= -kCoordLimit || ey1 >= kCoordLimit)
                return set_err(c, DNNI_E_RANGE, "point extent beyond +-2^30 LAS units of the origin");
            bb[0] = (int32_t)ex0;
            bb[1] = (int32_t)ex1;
            bb[2] = (int32_t)ey0;
            bb[3] = (int32_t)ey1;
        }
        plan_bins(bb, d.pt_count, bt_, plan[k]);
        if (bb[0] <= bb[1]) {
            plan[k].has_ext = 1;
            plan[k].ex0 = bb[0];
            plan[k].ex1 = bb[1];
            plan[k].ey0 = bb[2];
            plan[k].ey1 = bb[3];
        }
        cost[k] = (int64_t)plan[k].rw * plan[k].rh + d.pt_count;
    }
    order.resize(ntiles);
    std::iota(order.begin(), order.end(), 0);
    if (o.order_by_cost) std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
    hb = HostBatch();
    hb.rs = rs_;
    hb.win_words = ww_;
    hb.far_blocks = fb_;
    hb.dense_band = db_;
    for (int k : order) batch_add(hb, plan[k], tiles[k].pt_offset, tiles[k].out_offset, tiles[k].site_offset);
    if (hb.too_big) return set_err(c, DNNI_E_INVAL, "batch too large for one launch sequence: split it");
    return DNNI_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

int32_t dnni_version(void) { return DNNI_VERSION; }

dnni_status dnni_init(const dnni_settings* settings, dnni_ctx** out) {
    if (!out) return DNNI_E_INVAL;
    *out = nullptr;
    dnni_settings s{};
    if (settings) s = *settings;
    if (s.small_radius == 0) s.small_radius = 3;
    if (s.small_radius < 1 || s.small_radius > kMaxSmallRadius) return DNNI_E_INVAL;
    if (s.bin_target < 0) return DNNI_E_INVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return DNNI_E_CUDA;
    }
    if (s.device < 0 || s.device >= ndev) return DNNI_E_INVAL;
    dnni_ctx* c = new dnni_ctx();
    c->s = s;
    c->device = s.device;
    DeviceGuard g(c->device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) { delete c; return DNNI_E_CUDA; }
    c->sm_count = prop.multiProcessorCount;
    // a blocking stream: work queued on the context's stream is ordered with
    // the legacy default stream, so callers that pass NULL (or a framework's
    // default stream, whose handle is 0) read finished results there
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamDefault) != cudaSuccess) { delete c; return DNNI_E_CUDA; }
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) { dnni_destroy(c); return DNNI_E_CUDA; }
    if (cudaMallocHost(&c->h_sc, sizeof(Scalars)) != cudaSuccess ||
        cudaMallocHost(&c->h_ctr, sizeof(BatchCounters)) != cudaSuccess) {
        dnni_destroy(c);
        return DNNI_E_NOMEM;
    }
    memset(c->h_sc, 0, sizeof(Scalars));
    memset(c->h_ctr, 0, sizeof(BatchCounters));
    set_dense_smem_attr();
    *out = c;
    return DNNI_OK;
}

dnni_status dnni_destroy(dnni_ctx* c) {
    if (!c) return DNNI_E_INVAL;
    {
        DeviceGuard g(c->device);
        if (c->stream) cudaStreamSynchronize(c->stream);
        dnni_free_all(c);
        if (c->h_sc) cudaFreeHost(c->h_sc);
        if (c->h_ctr) cudaFreeHost(c->h_ctr);
        if (c->h_tables) cudaFreeHost(c->h_tables);
        for (auto& e : c->ev)
            if (e) cudaEventDestroy(e);
        if (c->stream) cudaStreamDestroy(c->stream);
    }
    delete c;
    return DNNI_OK;
}

const char* dnni_last_error(const dnni_ctx* c) { return c ? c->err.c_str() : "context is NULL"; }

dnni_status dnni_setup_run(dnni_ctx* c, const dnni_workpackage* wp, int64_t max_points) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    TileParams t;
    const char* msg = "";
    dnni_status rs = plan_geometry(wp, max_points, c->s.small_radius, t, &msg);
    if (rs) return set_err(c, rs, msg);
    // bins are sized from the points; reserve for the densest grid allowed
    int32_t bb[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, 0, 0};
    plan_bins(bb, max_points, c->s.bin_target, t);
    HostBatch hb;
    batch_add(hb, t, 0, 0, 0);
    DevArrays a;
    return ensure_scratch(c, c->scr, scratch_sizes(hb), a);
}

dnni_status dnni_interpolate_segment_device(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* d_xyz,
                                            const uint32_t* d_gid, int64_t n, float* d_h, uint32_t* d_site,
                                            void* stream, dnni_stats* stats) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (stats) memset(stats, 0, sizeof(*stats));
    return run_device(c, wp, d_xyz, d_gid, n, d_h, d_site, st, stats);
}

dnni_status dnni_interpolate_segment(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* xyz, const uint32_t* gid,
                                     int64_t n, float* out_h, uint32_t* out_site, dnni_stats* stats) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    if (!out_h) return set_err(c, DNNI_E_INVAL, "output grid pointer is NULL");
    if (n > 0 && !xyz) return set_err(c, DNNI_E_INVAL, "point pointer is NULL");
    DeviceGuard g(c->device);
    TileParams t;
    const char* msg = "";
    dnni_status rs = plan_geometry(wp, n, c->s.small_radius, t, &msg);
    if (rs) return set_err(c, rs, msg);
    const int64_t npix = (int64_t)t.rw * t.rh, cells = (int64_t)t.ncols * t.nrows;
    cudaStream_t st = c->stream;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n > 0) {
        if ((rs = dnni_ensure(c, c->in_xyz, sizeof(int32_t) * 3 * n))) return rs;
        CK(cudaMemcpyAsync(c->in_xyz.p, xyz, sizeof(int32_t) * 3 * n, cudaMemcpyHostToDevice, st));
        if (gid) {
            if ((rs = dnni_ensure(c, c->in_gid, sizeof(uint32_t) * n))) return rs;
            CK(cudaMemcpyAsync(c->in_gid.p, gid, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
        }
    }
    if ((rs = dnni_ensure(c, c->out_h, sizeof(float) * cells))) return rs;
    if (out_site && (rs = dnni_ensure(c, c->out_site, sizeof(uint32_t) * npix))) return rs;
    rs = run_device(c, wp, (const int32_t*)c->in_xyz.p, gid ? (const uint32_t*)c->in_gid.p : nullptr, n,
                    (float*)c->out_h.p, out_site ? (uint32_t*)c->out_site.p : nullptr, st, stats);
    if (rs) return rs;
    CK(cudaMemcpyAsync(out_h, c->out_h.p, sizeof(float) * cells, cudaMemcpyDeviceToHost, st));
    if (out_site) CK(cudaMemcpyAsync(out_site, c->out_site.p, sizeof(uint32_t) * npix, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (stats) {
        stats->h2d_bytes = n > 0 ? (int64_t)(sizeof(int32_t) * 3 * n + (gid ? sizeof(uint32_t) * n : 0)) : 0;
        stats->d2h_bytes = (int64_t)(sizeof(float) * cells + (out_site ? sizeof(uint32_t) * npix : 0));
    }
    return DNNI_OK;
}

dnni_status dnni_clear(dnni_ctx* c) {
    if (!c) return DNNI_E_INVAL;
    DeviceGuard g(c->device);
    cudaStreamSynchronize(c->stream);
    dnni_free_all(c);
    return DNNI_OK;
}

dnni_status dnni_print_times(dnni_ctx* c) {
    if (!c) return DNNI_E_INVAL;
    fprintf(stdout, "Time Results (%lld calls, device ms):\n", (long long)c->calls);
    fprintf(stdout, "\tbin points       : \t%f\n", c->acc_ms[0]);
    fprintf(stdout, "\tnearest site     : \t%f\n", c->acc_ms[1]);
    fprintf(stdout, "\tspan scatter     : \t%f\n", c->acc_ms[2]);
    fprintf(stdout, "\tstencil/finalize : \t%f\n", c->acc_ms[3]);
    return DNNI_OK;
}

dnni_status dnni_partition_contiguous(const int64_t* cost, int32_t n, int32_t parts, int32_t* first) {
    if (!first || parts < 1 || n < 0 || (n > 0 && !cost)) return DNNI_E_INVAL;
    long double total = 0;
    for (int32_t k = 0; k < n; ++k) {
        if (cost[k] < 0) return DNNI_E_INVAL;
        total += (long double)cost[k];
    }
    // boundary p: where the running cost is closest to p / parts of the total
    first[0] = 0;
    int32_t k = 0;
    long double run = 0;
    for (int32_t p = 1; p < parts; ++p) {
        const long double goal = total * p / parts;
        while (k < n && run + (long double)cost[k] / 2 <= goal) run += (long double)cost[k++];
        first[p] = k;
    }
    first[parts] = n;
    return DNNI_OK;
}

dnni_status dnni_host_alloc(size_t bytes, void** out) {
    if (!out) return DNNI_E_INVAL;
    if (cudaMallocHost(out, bytes ? bytes : 1) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return DNNI_E_NOMEM;
    }
    return DNNI_OK;
}

dnni_status dnni_host_free(void* p) {
    if (p) cudaFreeHost(p);
    return DNNI_OK;
}

// ---- batches ---------------------------------------------------------------

dnni_status dnni_batch_create(dnni_ctx* c, const dnni_tile* tiles, int32_t ntiles, const dnni_batch_options* opt,
                              dnni_batch** out) {
    if (!c || !out || !tiles || ntiles <= 0) return DNNI_E_INVAL;
    *out = nullptr;
    c->err.clear();
    DeviceGuard g(c->device);
    dnni_batch_options o{};
    if (opt) o = *opt;
    dnni_batch* b = new dnni_batch();
    b->ctx = c;
    b->use_graph = o.use_graph;
    b->opt = o;
    b->tiles_in.assign(tiles, tiles + ntiles);
    {
        dnni_status rs = plan_batch(c, tiles, ntiles, o, b->hb, b->order);
        if (rs) {
            delete b;
            return rs;
        }
    }
    dnni_status rs = ensure_scratch(c, b->scr, scratch_sizes(b->hb), b->arr);
    if (!rs) {
        b->bt = device_tables(b->arr.tables, ntiles);
        rs = stage_tables(c, b->hb, b->arr.tables, c->stream);
        if (!rs && cudaStreamSynchronize(c->stream) != cudaSuccess) rs = cuda_err(c, cudaGetLastError(), "upload");
    }
    if (rs) {
        release_scratch(c, b->scr);
        delete b;
        return rs;
    }
    b->h_sc.resize(ntiles);
    *out = b;
    return DNNI_OK;
}

dnni_status dnni_batch_run_device(dnni_batch* b, const int32_t* d_xyz, const uint32_t* d_gid, float* d_h,
                                  uint32_t* d_site, void* stream, dnni_stats* stats) {
    if (!b) return DNNI_E_INVAL;
    dnni_ctx* c = b->ctx;
    c->err.clear();
    DeviceGuard g(c->device);
    if (!d_h || (b->hb.n_rows > 0 && !d_xyz)) return set_err(c, DNNI_E_INVAL, "NULL buffer");
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (stats) CK(cudaEventRecord(c->ev[0], st));
    if (b->use_graph) {
        const void* key[4] = {d_xyz, d_gid, d_h, d_site};
        if (!b->exec || memcmp(key, b->graph_key, sizeof(key)) != 0) {
            if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
            if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
            cudaStream_t cap;
            CK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                launch_prologue(b->hb, b->bt, b->arr, d_xyz, cap, false);
                launch_body(b->hb, b->bt, b->arr, d_xyz, d_gid, d_h, d_site, c->sm_count, cap, nullptr, true);
                e = cudaStreamEndCapture(cap, &b->graph);
            }
            cudaStreamDestroy(cap);
            if (e != cudaSuccess) return cuda_err(c, e, "graph capture");
            CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
            memcpy(b->graph_key, key, sizeof(key));
        }
        CK(cudaGraphLaunch(b->exec, st));
    } else {
        // with stats, ev[1..3] mark the ends of binning, nearest sites and spans
        launch_prologue(b->hb, b->bt, b->arr, d_xyz, st, false);
        launch_body(b->hb, b->bt, b->arr, d_xyz, d_gid, d_h, d_site, c->sm_count, st, stats ? &c->ev[1] : nullptr,
                    true);
        CK(cudaGetLastError());
    }
    if (stats) {
        CK(cudaEventRecord(c->ev[4], st));
        if (!b->use_graph) k_span_hist<<<b->hb.rt_base.back(), dim3(32, 8), 0, st>>>(b->bt, b->arr.pix, b->arr.sc);
        const int n = (int)b->hb.tiles.size();
        CK(cudaMemcpyAsync(b->h_sc.data(), b->arr.sc, sizeof(Scalars) * n, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(c->h_ctr, b->arr.ctr, sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[4]);
        stats->ms_total = ms;
        if (!b->use_graph) {
            float ph[4];
            for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ph[k], c->ev[k], c->ev[k + 1]);
            stats->ms_bin = ph[0];
            stats->ms_nearest = ph[1];
            stats->ms_scatter = ph[2];
            stats->ms_finalize = ph[3];
            float md = 0;
            cudaEventElapsedTime(&md, c->ev[1], c->ev[5]);
            stats->ms_dense = md;
            stats->ms_far = ph[1] - md;
        }
        if (c->h_ctr->err & kErrRange)
            return set_err(c, DNNI_E_RANGE, "a point lies beyond its tile's declared extent or the coordinate range");
        fold_stats(b->h_sc.data(), n, stats);
        for (const TileParams& t : b->hb.tiles) stats->n_points += t.npts;
        stats->n_cells = b->hb.n_cells;
        stats->n_pixels = b->hb.n_pix;
    }
    return DNNI_OK;
}

// Cuts a batch into up to kSlices slices of consecutive point rows, with work
// in the proportions of kSliceWeight, plans each and uploads its tables; the
// slices share the batch's scratch (they run one after another on the
// compute stream).
static dnni_status plan_slices(dnni_batch* b) {
    dnni_ctx* c = b->ctx;
    // slice sizes: a small first slice shortens the wait for the first upload,
    // the next ones grow by 1.5x (each upload, at about two thirds of the
    // compute rate, then ends before the compute of its predecessor), and a
    // small last slice shortens the final download
    constexpr int kSlices = 16;
    constexpr double kSliceWeight[kSlices] = {0.05, 0.075, 0.11, 0.17, 0.25, 0.38, 0.57, 0.85,
                                              1.0, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 0.12};
    const int n = (int)b->tiles_in.size();
    // fewer tiles than slices: one tile per slice, equal weights
    const int S = b->hb.n_rows >= (4 << 20) ? std::min(n, kSlices) : 1;
    const bool ramp = S == kSlices;
    b->sliced = S > 1;
    b->slices.clear();
    if (!b->sliced) {
        b->slices_planned = true;
        return DNNI_OK;
    }
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int x, int y) { return b->tiles_in[x].pt_offset < b->tiles_in[y].pt_offset; });
    auto cost = [&](int k) {
        const dnni_tile& t = b->tiles_in[k];
        return (double)t.wp.ncols * t.wp.nrows + (double)t.pt_count;
    };
    double total = 0;
    for (int k : idx) total += cost(k);
    auto weight = [&](int s) { return ramp ? kSliceWeight[s] : 1.0; };
    double wsum = 0;
    for (int s = 0; s < S; ++s) wsum += weight(s);
    dnni_batch_options o = b->opt;
    o.order_by_cost = 0;
    double run = 0, wrun = 0;
    size_t k0 = 0;
    for (int s = 0; s < S; ++s) {
        size_t k1 = k0;
        wrun += weight(s);
        const double goal = total * wrun / wsum;
        while (k1 < idx.size() && (s == S - 1 || run + cost(idx[k1]) <= goal || k1 == k0)) run += cost(idx[k1++]);
        if (k1 == k0) break;
        std::vector<dnni_tile> part;
        for (size_t k = k0; k < k1; ++k) part.push_back(b->tiles_in[idx[k]]);
        BatchSlice sl;
        std::vector<int> order;
        dnni_status rs = plan_batch(c, part.data(), (int)part.size(), o, sl.hb, order);
        if (rs) return rs;
        sl.row0 = INT64_MAX;
        sl.out0 = INT64_MAX;
        sl.site0 = INT64_MAX;
        for (const dnni_tile& t : part) {
            sl.row0 = std::min(sl.row0, t.pt_offset);
            sl.row1 = std::max(sl.row1, t.pt_offset + t.pt_count);
            sl.out0 = std::min<int64_t>(sl.out0, t.out_offset);
            sl.out1 = std::max<int64_t>(sl.out1, t.out_offset + (int64_t)t.wp.ncols * t.wp.nrows);
        }
        for (const TileParams& t : sl.hb.tiles)
            if (t.site_off >= 0) {
                sl.site0 = std::min<int64_t>(sl.site0, t.site_off);
                sl.site1 = std::max<int64_t>(sl.site1, t.site_off + (int64_t)t.rw * t.rh);
            }
        if (sl.site0 == INT64_MAX) sl.site0 = sl.site1 = 0;
        if ((rs = dnni_ensure(c, sl.tables, TableLayout((int)part.size()).total))) return rs;
        sl.bt = device_tables((const unsigned char*)sl.tables.p, (int)part.size());
        if ((rs = stage_tables(c, sl.hb, (unsigned char*)sl.tables.p, c->stream))) return rs;
        b->slices.push_back(std::move(sl));
        k0 = k1;
    }
    // the full batch's view of its scratch (the graph captured for it is
    // rebuilt if the arrays moved)
    DevArrays full;
    dnni_status rs = ensure_scratch(c, b->scr, scratch_sizes(b->hb), full);
    if (rs) return rs;
    full.tables = b->arr.tables;
    if (full.sorted != b->arr.sorted || full.pix != b->arr.pix) {
        if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    }
    b->arr = full;
    const int ns = (int)b->slices.size();
    // each slice works in its own part of the batch's scratch (the parts add
    // up to the whole batch's sizes), so that consecutive slices can compute
    // on two streams at once
    if ((rs = dnni_ensure(c, b->slice_ctrs, sizeof(BatchCounters) * (size_t)ns))) return rs;
    {
        int64_t pts = 0, bins = 0, scan = 0, blk = 0, sup = 0, pix = 0, far = 0, cells = 0, tiles = 0;
        for (int s = 0; s < ns; ++s) {
            BatchSlice& sl = b->slices[s];
            const HostBatch& h = sl.hb;
            DevArrays v = full;
            v.sorted += pts;
            v.cnt += bins;
            v.start += bins;
            v.bsum += scan;
            v.bmask += blk;
            v.smask += sup;
            v.rownear += blk;
            v.near += blk;
            v.pix += pix;
            v.far += far;
            v.D += cells;
            v.Dc += cells;
            v.sc += tiles;
            v.ctr = (BatchCounters*)b->slice_ctrs.p + s;
            v.tables = (unsigned char*)sl.tables.p;
            sl.arr = v;
            pts += h.n_pts;
            bins += h.n_bins;
            scan += h.scan_base.back();
            blk += h.blk_base.back();
            sup += h.sup_base.back();
            pix += h.n_pix;
            far += h.n_far;
            cells += h.n_cells;
            tiles += (int64_t)h.tiles.size();
        }
    }
    if (cudaStreamCreateWithFlags(&b->s_in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->s_out, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->s_cmp, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMallocHost((void**)&b->h_ctrs, sizeof(BatchCounters) * ns) != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, DNNI_E_CUDA, "slice streams");
    }
    b->ev_in.assign(ns, nullptr);
    b->ev_done.assign(ns, nullptr);
    for (int s = 0; s < ns; ++s)
        if (cudaEventCreateWithFlags(&b->ev_in[s], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_done[s], cudaEventDisableTiming) != cudaSuccess)
            return set_err(c, DNNI_E_CUDA, "slice events");
    CK(cudaStreamSynchronize(c->stream));
    b->slices_planned = true;
    return DNNI_OK;
}

dnni_status dnni_batch_run(dnni_batch* b, const int32_t* xyz, const uint32_t* gid, int64_t n_rows, float* out_h,
                           uint32_t* out_site, dnni_stats* stats) {
    if (!b) return DNNI_E_INVAL;
    dnni_ctx* c = b->ctx;
    c->err.clear();
    DeviceGuard g(c->device);
    if (n_rows < b->hb.n_rows) return set_err(c, DNNI_E_INVAL, "fewer point rows than the tiles reference");
    if (!out_h || (n_rows > 0 && !xyz)) return set_err(c, DNNI_E_INVAL, "NULL buffer");
    cudaStream_t st = c->stream;
    dnni_status rs;
    if (n_rows > 0) {
        if ((rs = dnni_ensure(c, b->in_xyz, sizeof(int32_t) * 3 * n_rows))) return rs;
        if (gid && (rs = dnni_ensure(c, b->in_gid, sizeof(uint32_t) * n_rows))) return rs;
    }
    const int64_t nh = std::max<int64_t>(b->hb.out_end, 1), ns = std::max<int64_t>(b->hb.site_end, 1);
    if ((rs = dnni_ensure(c, b->out_h, sizeof(float) * nh))) return rs;
    if (out_site && (rs = dnni_ensure(c, b->out_site, sizeof(uint32_t) * ns))) return rs;
    if (!b->slices_planned && (rs = plan_slices(b))) return rs;
    if (!b->sliced) {
        if (n_rows > 0) {
            CK(cudaMemcpyAsync(b->in_xyz.p, xyz, sizeof(int32_t) * 3 * n_rows, cudaMemcpyHostToDevice, st));
            if (gid) CK(cudaMemcpyAsync(b->in_gid.p, gid, sizeof(uint32_t) * n_rows, cudaMemcpyHostToDevice, st));
        }
        rs = dnni_batch_run_device(b, (const int32_t*)b->in_xyz.p, gid ? (const uint32_t*)b->in_gid.p : nullptr,
                                   (float*)b->out_h.p, out_site ? (uint32_t*)b->out_site.p : nullptr, st, stats);
        if (rs) return rs;
        CK(cudaMemcpyAsync(out_h, b->out_h.p, sizeof(float) * b->hb.out_end, cudaMemcpyDeviceToHost, st));
        if (out_site && b->hb.site_end > 0)
            CK(cudaMemcpyAsync(out_site, b->out_site.p, sizeof(uint32_t) * b->hb.site_end, cudaMemcpyDeviceToHost,
                               st));
        CK(cudaMemcpyAsync(c->h_ctr, b->arr.ctr, sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c->h_ctr->err & kErrRange)
            return set_err(c, DNNI_E_RANGE, "a point lies beyond its tile's declared extent or the coordinate range");
    } else {
        // pipelined: slice s uploads on s_in while the slices before it
        // compute, alternately on the context stream and on s_cmp (each in its
        // own part of the scratch, so one slice's kernels fill the SMs that
        // the other's leave idle), and finished slices download on s_out
        if (stats) {
            memset(stats, 0, sizeof(*stats));
            CK(cudaEventRecord(c->ev[0], st));
            CK(cudaStreamWaitEvent(b->s_in, c->ev[0], 0));
        }
        int32_t* dx = (int32_t*)b->in_xyz.p;
        uint32_t* dg = gid ? (uint32_t*)b->in_gid.p : nullptr;
        for (size_t s = 0; s < b->slices.size(); ++s) {
            const BatchSlice& sl = b->slices[s];
            const size_t r0 = (size_t)sl.row0, nr = (size_t)(sl.row1 - sl.row0);
            if (nr) {
                CK(cudaMemcpyAsync(dx + 3 * r0, xyz + 3 * r0, 12 * nr, cudaMemcpyHostToDevice, b->s_in));
                if (gid) CK(cudaMemcpyAsync(dg + r0, gid + r0, 4 * nr, cudaMemcpyHostToDevice, b->s_in));
            }
            CK(cudaEventRecord(b->ev_in[s], b->s_in));
            cudaStream_t cs = (s & 1) ? b->s_cmp : st;
            CK(cudaStreamWaitEvent(cs, b->ev_in[s], 0));
            const DevArrays& a = sl.arr;
            launch_prologue(sl.hb, sl.bt, a, dx, cs, false);
            launch_body(sl.hb, sl.bt, a, dx, dg, (float*)b->out_h.p, out_site ? (uint32_t*)b->out_site.p : nullptr,
                        c->sm_count, cs, nullptr, true);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(&b->h_ctrs[s], a.ctr, sizeof(BatchCounters), cudaMemcpyDeviceToHost, cs));
            CK(cudaEventRecord(b->ev_done[s], cs));
            CK(cudaStreamWaitEvent(b->s_out, b->ev_done[s], 0));
            CK(cudaMemcpyAsync(out_h + sl.out0, (const float*)b->out_h.p + sl.out0, 4 * (size_t)(sl.out1 - sl.out0),
                               cudaMemcpyDeviceToHost, b->s_out));
            if (out_site && sl.site1 > sl.site0)
                CK(cudaMemcpyAsync(out_site + sl.site0, (const uint32_t*)b->out_site.p + sl.site0,
                                   4 * (size_t)(sl.site1 - sl.site0), cudaMemcpyDeviceToHost, b->s_out));
        }
        if (stats) CK(cudaEventRecord(c->ev[1], b->s_out));
        CK(cudaStreamSynchronize(b->s_out));
        CK(cudaStreamSynchronize(st));
        CK(cudaStreamSynchronize(b->s_cmp));
        for (size_t s = 0; s < b->slices.size(); ++s)
            if (b->h_ctrs[s].err & kErrRange)
                return set_err(c, DNNI_E_RANGE,
                               "a point lies beyond its tile's declared extent or the coordinate range");
        if (stats) {
            float ms = 0;
            cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
            stats->ms_total = ms;
            for (const TileParams& t : b->hb.tiles) stats->n_points += t.npts;
            stats->n_cells = b->hb.n_cells;
            stats->n_pixels = b->hb.n_pix;
        }
    }
    if (stats) {
        stats->h2d_bytes = (int64_t)(sizeof(int32_t) * 3 * n_rows + (gid ? sizeof(uint32_t) * n_rows : 0));
        stats->d2h_bytes =
            (int64_t)(sizeof(float) * b->hb.out_end + (out_site ? sizeof(uint32_t) * b->hb.site_end : 0));
    }
    return DNNI_OK;
}

dnni_status dnni_batch_destroy(dnni_batch* b) {
    if (!b) return DNNI_E_INVAL;
    dnni_ctx* c = b->ctx;
    {
        DeviceGuard g(c->device);
        cudaDeviceSynchronize();
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->graph) cudaGraphDestroy(b->graph);
        for (BatchSlice& sl : b->slices) dnni_release(sl.tables, c);
        for (cudaEvent_t e : b->ev_in)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : b->ev_done)
            if (e) cudaEventDestroy(e);
        if (b->s_in) cudaStreamDestroy(b->s_in);
        if (b->s_out) cudaStreamDestroy(b->s_out);
        if (b->s_cmp) cudaStreamDestroy(b->s_cmp);
        dnni_release(b->slice_ctrs, c);
        if (b->h_ctrs) cudaFreeHost(b->h_ctrs);
        release_scratch(c, b->scr);
        dnni_release(b->in_xyz, c);
        dnni_release(b->in_gid, c);
        dnni_release(b->out_h, c);
        dnni_release(b->out_site, c);
    }
    delete b;
    return DNNI_OK;
}

// ---- autotuner -------------------------------------------------------------

dnni_status dnni_batch_autotune(dnni_ctx* c, const dnni_tile* tiles, int32_t ntiles, const int32_t* d_xyz,
                                const uint32_t* d_gid, int32_t sample_tiles, dnni_batch_options* options,
                                dnni_tune_report* report) {
    if (!c || !tiles || ntiles <= 0 || !options) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    const dnni_batch_options given = *options;
    // sample: tiles evenly spaced in cost order, so that it spans the sizes
    std::vector<int> idx(ntiles);
    std::iota(idx.begin(), idx.end(), 0);
    auto cost = [&](int k) { return (int64_t)tiles[k].wp.ncols * tiles[k].wp.nrows + tiles[k].pt_count; };
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return cost(x) > cost(y); });
    const int m = sample_tiles > 0 && sample_tiles < ntiles ? sample_tiles : ntiles;
    std::vector<dnni_tile> smp(m);
    int64_t out = 0;
    for (int k = 0; k < m; ++k) {
        smp[k] = tiles[idx[(int64_t)k * ntiles / m]];
        smp[k].out_offset = out;
        smp[k].site_offset = -1;
        out += (int64_t)smp[k].wp.ncols * smp[k].wp.nrows;
    }
    DevBuf hbuf;
    Scratch tscr;
    DevArrays a;
    HostBatch hb;
    std::vector<int> order;
    std::vector<dnni_tune_trial> trials;
    cudaStream_t st = c->stream;
    auto trial = [&](int rs_, int bt_, int ww_, int fg_, int db_, float* ms) -> dnni_status {
        dnni_batch_options o = given;
        o.small_radius = rs_;
        o.bin_target = bt_;
        o.span_window = ww_;
        o.far_group = fg_;
        o.dense_band = db_;
        dnni_status rs = plan_batch(c, smp.data(), m, o, hb, order);
        if (rs) return rs;
        if ((rs = ensure_scratch(c, tscr, scratch_sizes(hb), a))) return rs;
        const BatchTables bt = device_tables(a.tables, m);
        if ((rs = stage_tables(c, hb, a.tables, st))) return rs;
        for (int r = 0; r < 3; ++r) {            // one warm-up run, two timed
            if (r == 1) CK(cudaEventRecord(c->ev[0], st));
            launch_prologue(hb, bt, a, d_xyz, st, false);
            launch_body(hb, bt, a, d_xyz, d_gid, (float*)hbuf.p, nullptr, c->sm_count, st, nullptr, true);
        }
        CK(cudaEventRecord(c->ev[1], st));
        CK(cudaGetLastError());
        CK(cudaEventSynchronize(c->ev[1]));
        float t = 0;
        CK(cudaEventElapsedTime(&t, c->ev[0], c->ev[1]));
        *ms = t / 2;
        trials.push_back(dnni_tune_trial{rs_, bt_, *ms, ww_, fg_, db_});
        return DNNI_OK;
    };
    dnni_status rs = dnni_ensure(c, hbuf, sizeof(float) * std::max<int64_t>(out, 1));
    const int rs0 = given.small_radius ? given.small_radius : c->s.small_radius;
    const int bt0 = given.bin_target ? given.bin_target : (c->s.bin_target ? c->s.bin_target : 4);
    const int ww0 = given.span_window ? given.span_window : kSpanWindowWords;
    const int fg0 = given.far_group ? given.far_group : kFarBlocksDefault + 1;
    const int db0 = given.dense_band ? given.dense_band : kTileY;
    float ms_default = 0, best_ms = 0;
    int best_rs = rs0, best_bt = bt0, best_ww = ww0, best_fg = fg0, best_db = db0;
    if (!rs) rs = trial(rs0, bt0, ww0, fg0, db0, &ms_default);
    best_ms = ms_default;
    // coordinate search: the bin size first, then the stencil/span split,
    // the span path's shared-memory window, the far pass's pixel groups and
    // the ring search's pixel-block shape
    static const int kBinTargets[] = {1, 2, 3, 4, 6, 8, 12};
    static const int kRadii[] = {1, 2, 3, 4, 5, 6};
    static const int kWindows[] = {1, 2048, 4096, 8192, 12288};   // 1: no window
    static const int kBands[] = {16, 32, 64};
    for (int bt_ : kBinTargets) {
        if (rs || bt_ == bt0) continue;
        float ms = 0;
        rs = trial(rs0, bt_, ww0, fg0, db0, &ms);
        if (!rs && ms < best_ms) { best_ms = ms; best_bt = bt_; }
    }
    for (int r_ : kRadii) {
        if (rs || r_ == rs0 || r_ > kMaxSmallRadius) continue;
        float ms = 0;
        rs = trial(r_, best_bt, ww0, fg0, db0, &ms);
        if (!rs && ms < best_ms) { best_ms = ms; best_rs = r_; }
    }
    for (int w_ : kWindows) {
        if (rs || w_ == ww0) continue;
        float ms = 0;
        rs = trial(best_rs, best_bt, w_, fg0, db0, &ms);
        if (!rs && ms < best_ms) { best_ms = ms; best_ww = w_; }
    }
    for (int f_ = 1; f_ <= 2; ++f_) {
        if (rs || f_ == fg0) continue;
        float ms = 0;
        rs = trial(best_rs, best_bt, best_ww, f_, db0, &ms);
        if (!rs && ms < best_ms) { best_ms = ms; best_fg = f_; }
    }
    for (int d_ : kBands) {
        if (rs || d_ == db0) continue;
        float ms = 0;
        rs = trial(best_rs, best_bt, best_ww, best_fg, d_, &ms);
        if (!rs && ms < best_ms) { best_ms = ms; best_db = d_; }
    }
    release_scratch(c, tscr);
    dnni_release(hbuf, c);
    if (rs) return rs;
    options->small_radius = best_rs;
    options->bin_target = best_bt;
    options->span_window = best_ww;
    options->far_group = best_fg;
    options->dense_band = best_db;
    if (report) {
        memset(report, 0, sizeof(*report));
        report->ntrials = (int32_t)std::min<size_t>(trials.size(), 32);
        report->sample_tiles = m;
        report->ms_default = ms_default;
        for (int k = 0; k < report->ntrials; ++k) {
            report->trial[k] = trials[k];
            if (trials[k].small_radius == best_rs && trials[k].bin_target == best_bt &&
                trials[k].span_window == best_ww && trials[k].far_group == best_fg &&
                trials[k].dense_band == best_db)
                report->best = k;
        }
    }
    return DNNI_OK;
}

}  // extern "C"

void SegBufs::release(dnni_ctx* c) {
    DevBuf* all[] = {&xin, &sxyz, &sgid, &part, &cur, &cnt, &start, &bbox, &occ, &gxyz, &ggid, &gout[0], &gout[1],
                     &gsite[0], &gsite[1], &chunks, &ring};
    for (DevBuf* b : all) dnni_release(*b, c);
}

void dnni_free_all(dnni_ctx* c) {
    release_scratch(c, c->scr);
    release_scratch(c, c->seg_scr);
    c->seg.release(c);
    release_scratch(c, c->st.scr);
    DevBuf* bufs[] = {&c->in_xyz, &c->in_gid, &c->out_h, &c->out_site, &c->st.xin, &c->st.tin, &c->st.xyz,
                      &c->st.idx, &c->st.gs, &c->st.site, &c->st.pix};
    for (DevBuf* b : bufs) dnni_release(*b, c);
}

// ---------------------------------------------------------------------------
// Entry point that allocates nothing (no counterpart in the reference).
//
// Some callers cannot let a library call cudaMalloc: a host application that
// manages all device memory through its own pool and forbids libraries from
// allocating behind its back (a GIS or database plug-in host with a fixed
// device budget), or a latency-critical caller that cannot absorb the implicit
// device-wide synchronisation of cudaMalloc/cudaFree.  For them,
// dnni_interpolate_segment_device_noalloc runs the same kernels as
// dnni_interpolate_segment_device with every byte of scratch taken from the
// file-scope device array below.  The module that holds the array is loaded on
// every GPU that uses this library, and that GPU keeps the 32 MiB until the
// process exits.
// ---------------------------------------------------------------------------

constexpr size_t kNoAllocScratchBytes = 32u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_base[kNoAllocMaxDevices] = {};

// In host code g_noalloc_scratch is only a host-side stand-in for the array,
// not a device address: a kernel given it would fault or, where the GPU can
// reach host memory, silently use the wrong memory.  The device address is
// looked up once per device, with that device current, on the first call,
// and kept for the life of the process (a cudaDeviceReset of the device
// would leave it stale; the header tells callers not to mix the two).
dnni_status noalloc_base(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices) return DNNI_E_INVAL;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return DNNI_E_CUDA;
        }
        g_noalloc_base[dev] = (unsigned char*)p;
    }
    *out = g_noalloc_base[dev];
    return DNNI_OK;
}

// Carves one work package's scratch out of the array; false when it does
// not fit.
bool carve_noalloc(unsigned char* base, const ScratchSizes& z, DevArrays& a) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + off;
        off = (off + bytes + 255) & ~(size_t)255;
        return p;
    };
    a.tables = take(z.tables);
    a.sc = (Scalars*)take(z.sc);
    a.ctr = (BatchCounters*)take(z.ctr);
    a.pix = (int2*)take(z.pix);
    a.far = (FarSlot*)take(z.far);
    a.D = (unsigned long long*)take(z.D);
    a.Dc = (int*)take(z.Dc);
    a.sorted = (int4*)take(z.sorted);
    a.cnt = (int*)take(z.cnt);
    a.start = (int*)take(z.cnt);
    a.bsum = (int*)take(z.bsum);
    a.bmask = (uint64_t*)take(z.bmask);
    a.smask = (uint64_t*)take(z.smask);
    a.rownear = (int*)take(z.rownear);
    a.near = (int64_t*)take(z.near);
    return off <= kNoAllocScratchBytes;
}

}  // namespace

extern "C" dnni_status dnni_interpolate_segment_device_noalloc(const dnni_workpackage* wp, const int32_t* d_xyz,
                                                               const uint32_t* d_gid, int64_t n, float* d_h,
                                                               uint32_t* d_site, void* stream) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return DNNI_E_CUDA;
    }
    unsigned char* base = nullptr;
    dnni_status rs = noalloc_base(dev, &base);
    if (rs) return rs;
    TileParams t;
    const char* msg = "";
    rs = plan_geometry(wp, n, 3, t, &msg);
    if (rs) return rs;
    if (!d_h || (n > 0 && !d_xyz)) return DNNI_E_INVAL;
    t.has_gid = d_gid ? 1 : 0;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    set_dense_smem_attr();
    cudaStream_t st = (cudaStream_t)stream;
    // provisional one-tile plan for the bounding-box pass
    int32_t bb[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN};
    plan_bins(bb, 0, 0.0, t);
    HostBatch hb;
    batch_add(hb, t, 0, 0, d_site ? 0 : -1);
    DevArrays a;
    if (!carve_noalloc(base, scratch_sizes(hb), a)) return DNNI_E_SCRATCH;
    // the one-tile tables go up from pageable host memory: the copy has
    // taken the bytes when cudaMemcpyAsync returns, so the buffer can be
    // repacked at once
    std::vector<unsigned char> tbl(TableLayout(1).total);
    pack_tables(hb, tbl.data());
    if (cudaMemcpyAsync(a.tables, tbl.data(), tbl.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
        return DNNI_E_CUDA;
    BatchTables bt = device_tables(a.tables, 1);
    // the array keeps the previous call's contents: the scalars, bin counts
    // and span words are cleared by the launch sequence itself
    launch_prologue(hb, bt, a, d_xyz, st);
    if (n > 0) {
        Scalars hsc;
        if (cudaMemcpyAsync(&hsc, a.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return DNNI_E_CUDA;
        }
        if (hsc.err & kErrRange) return DNNI_E_RANGE;
        plan_bins(hsc.bbox, n, 0.0, t);
        hb = HostBatch();
        batch_add(hb, t, 0, 0, d_site ? 0 : -1);
        if (!carve_noalloc(base, scratch_sizes(hb), a)) return DNNI_E_SCRATCH;
        pack_tables(hb, tbl.data());
        if (cudaMemcpyAsync(a.tables, tbl.data(), tbl.size(), cudaMemcpyHostToDevice, st) != cudaSuccess)
            return DNNI_E_CUDA;
        bt = device_tables(a.tables, 1);
    }
    launch_body(hb, bt, a, d_xyz, d_gid, d_h, d_site, sms, st, nullptr);
    if (cudaGetLastError() != cudaSuccess) return DNNI_E_CUDA;
    return DNNI_OK;
}

#include "dnni_segment.cuh"
#include "dnni_server.cuh"
#include "dnni_compat.cuh"
#include "dnni_spacetime.cuh"
#include "dnni_calibrate.cuh"
