// dnni_server.cuh -- serving DEM requests against a resident point cloud with
// continuous batching (dnni_server_*).  Included by dnni_engine.cu after the
// segment driver, whose bucketing, bound and gather pieces it reuses.
//
// No counterpart in the reference, whose CLI interpolates one dataset per run
// (terranni.cpp:544-700); each request is one work package of nni::performNNI
// (nni.cpp:870-944) cut from the resident cloud.
#pragma once

#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct SrvReq {
    dnni_request r{};
    double t_submit = 0, t_launch = 0, t_done = 0;
    int status = DNNI_OK;
    int hr_force = 0;          // raster halo to use (cells), 0 = from the bound
    int halo = 0, batch = 0, runs = 0;
    int64_t points = 0;
    bool done = false;
};

// One request of a batch under construction or in flight.
struct SrvItem {
    uint64_t ticket;
    int hr;                    // raster halo (cells)
    bool all_raster, all_buckets;
    int rx0, ry0, rw;          // raster origin (request cells) and width
    dnni_tile tile;
    size_t nchunks;
};

struct SrvSlot {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;   // device start and end of the slot's batch
    DevBuf arena;
    unsigned char* h_out = nullptr;   // pinned landing area for results bound for pageable buffers
    size_t h_out_cap = 0;
    std::vector<std::pair<size_t, size_t>> landing;   // per item: offset of heights, of site map (or SIZE_MAX)
    unsigned char* h_tab = nullptr;
    size_t h_tab_cap = 0;
    Scalars* h_sc = nullptr;
    int h_sc_cap = 0;
    BatchCounters* h_ctr = nullptr;
    std::vector<SrvItem> items;
    bool busy = false;
};

}  // namespace

struct dnni_server {
    dnni_ctx* ctx = nullptr;
    dnni_server_options o{};
    // the resident cloud
    SegGrid G{};
    SegBufs B;
    std::vector<long long> start;
    std::vector<int4> bbox;
    long long wx0 = 0, wy0 = 0, wx1 = -1, wy1 = -1;   // world box (LAS, inclusive)
    long long fw = 1;
    int nfx = 0, nfy = 0;
    std::vector<double> edt2;
    int64_t n = 0;
    double ms_build = 0;
    // requests
    std::mutex mu;
    std::condition_variable cv;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, SrvReq> reqs;
    uint64_t next = 1;
    bool stop = false;
    std::vector<SrvSlot> slots;
    std::thread th;
    int64_t submitted = 0, completed = 0, failed = 0, batches = 0, cells = 0, points = 0;
    // device time line of the batches: [start, end] in ms after `epoch`
    cudaEvent_t epoch = nullptr;
    std::vector<std::pair<double, double>> busy;
};

namespace {

// Upper bound (LAS units) of the nearest-site distance of any position in the
// LAS box [x0,x1] x [y0,y1]; < 0 when the cloud has no points.
double srv_bound(const dnni_server* s, long long x0, long long y0, long long x1, long long y1) {
    if (s->n == 0) return -1.0;
    const long long gx1 = s->G.ox + (long long)s->nfx * s->fw - 1, gy1 = s->G.oy + (long long)s->nfy * s->fw - 1;
    const double ox = (double)std::max<long long>({0, s->G.ox - x0, x1 - gx1});
    const double oy = (double)std::max<long long>({0, s->G.oy - y0, y1 - gy1});
    auto clampf = [](long long v, int hi) { return (int)std::min<long long>(std::max<long long>(v, 0), hi); };
    const int fx0 = clampf(floor_div_ll(x0 - s->G.ox, s->fw), s->nfx - 1);
    const int fx1 = clampf(floor_div_ll(x1 - s->G.ox, s->fw), s->nfx - 1);
    const int fy0 = clampf(floor_div_ll(y0 - s->G.oy, s->fw), s->nfy - 1);
    const int fy1 = clampf(floor_div_ll(y1 - s->G.oy, s->fw), s->nfy - 1);
    double m = 0;
    for (int fy = fy0; fy <= fy1; ++fy)
        for (int fx = fx0; fx <= fx1; ++fx) m = std::max(m, s->edt2[(size_t)fy * s->nfx + fx]);
    return (double)s->fw * (std::sqrt(m) + 1.4143) + std::sqrt(ox * ox + oy * oy);
}

// Plans one request: raster (its grid +- hr, clipped to the world box on its
// cell lattice), point box, gather chunks.  false: the request cannot run
// (status in *why).
bool srv_plan(dnni_server* s, uint64_t ticket, const SrvReq& q, std::vector<SegChunk>& chunks, int64_t& pt,
              int64_t& out, int64_t& site, SrvItem& it, int* why) {
    const dnni_request& r = q.r;
    const long long cs = r.cell_size;
    // lattice indices of the world box on the request's cell lattice
    const long long wi0 = -floor_div_ll(r.x0 - s->wx0, cs), wi1 = floor_div_ll(s->wx1 - r.x0, cs);
    const long long wj0 = -floor_div_ll(r.y0 - s->wy0, cs), wj1 = floor_div_ll(s->wy1 - r.y0, cs);
    auto raster_of = [&](int hr, long long& a0, long long& b0, long long& a1, long long& b1) {
        a0 = std::max<long long>(-hr, wi0);
        b0 = std::max<long long>(-hr, wj0);
        a1 = std::min<long long>((long long)r.ncols - 1 + hr, wi1);
        b1 = std::min<long long>((long long)r.nrows - 1 + hr, wj1);
    };
    int hr = q.hr_force;
    long long a0, b0, a1, b1;
    if (hr == 0) {
        hr = 2;
        for (int iter = 0; iter < 24; ++iter) {
            raster_of(hr, a0, b0, a1, b1);
            if (a0 > a1 || b0 > b1) break;
            const double ub = srv_bound(s, r.x0 + a0 * cs, r.y0 + b0 * cs, r.x0 + a1 * cs, r.y0 + b1 * cs);
            const int h2 = ub < 0 ? 2 : (int)std::min<double>(std::ceil(ub / cs) + 3, 1 << 20);
            if (h2 <= hr) break;
            hr = h2;
        }
    }
    raster_of(hr, a0, b0, a1, b1);
    it = SrvItem{};
    it.ticket = ticket;
    it.hr = hr;
    dnni_tile& t = it.tile;
    t.wp.ncols = r.ncols;
    t.wp.nrows = r.nrows;
    t.wp.cell_size = r.cell_size;
    t.wp.origin_x = r.x0;
    t.wp.origin_y = r.y0;
    t.wp.z_scale = r.z_scale;
    t.wp.z_offset = r.z_offset;
    t.wp.nodata = r.nodata;
    if (a0 > a1 || b0 > b1) {   // the request lies off the world box: no pixel at all
        it.rw = 0;
        t.pt_count = 0;
        t.out_offset = out;
        out += (int64_t)r.ncols * r.nrows;
        it.nchunks = 0;
        return true;
    }
    if (a1 - a0 + 1 > 32767 || b1 - b0 + 1 > 32767 || std::max<long long>(a1, r.ncols - 1) - std::min<long long>(a0, 0) >= 32767 ||
        std::max<long long>(b1, r.nrows - 1) - std::min<long long>(b0, 0) >= 32767) {
        *why = DNNI_E_INVAL;    // halo beyond the largest raster
        return false;
    }
    it.all_raster = a0 == wi0 && b0 == wj0 && a1 == wi1 && b1 == wj1;
    it.rx0 = (int)a0;
    it.ry0 = (int)b0;
    it.rw = (int)(a1 - a0 + 1);
    t.wp.raster_x0 = (int32_t)a0;
    t.wp.raster_y0 = (int32_t)b0;
    t.wp.raster_x1 = (int32_t)(a1 + 1);
    t.wp.raster_y1 = (int32_t)(b1 + 1);
    // point box: the raster +- hr, as bucket rows
    const long long px0 = r.x0 + (a0 - hr) * cs, px1 = r.x0 + (a1 + hr) * cs;
    const long long py0 = r.y0 + (b0 - hr) * cs, py1 = r.y0 + (b1 + hr) * cs;
    auto bclamp = [](long long v, int hi) { return (int)std::min<long long>(std::max<long long>(v, 0), hi); };
    const int bx0 = bclamp(floor_div_ll(px0 - s->G.ox, s->G.w), s->G.nbx - 1);
    const int bx1 = bclamp(floor_div_ll(px1 - s->G.ox, s->G.w), s->G.nbx - 1);
    const int by0 = bclamp(floor_div_ll(py0 - s->G.oy, s->G.w), s->G.nby - 1);
    const int by1 = bclamp(floor_div_ll(py1 - s->G.oy, s->G.w), s->G.nby - 1);
    it.all_buckets = bx0 == 0 && by0 == 0 && bx1 == s->G.nbx - 1 && by1 == s->G.nby - 1;
    const int64_t p0 = pt;
    const size_t c0 = chunks.size();
    int4 ext = make_int4(INT_MAX, INT_MAX, INT_MIN, INT_MIN);
    for (int by = by0; by <= by1; ++by) {
        const long long s0 = s->start[(size_t)by * s->G.nbx + bx0], s1 = s->start[(size_t)by * s->G.nbx + bx1 + 1];
        for (long long o = s0; o < s1; o += kSegGatherChunk) {
            const int m = (int)std::min<long long>(kSegGatherChunk, s1 - o);
            chunks.push_back(SegChunk{o, pt, m, 0});
            pt += m;
        }
        for (int bx = bx0; bx <= bx1; ++bx) {
            const int4 bb = s->bbox[(size_t)by * s->G.nbx + bx];
            if (bb.x > bb.z) continue;
            ext.x = std::min(ext.x, bb.x); ext.y = std::min(ext.y, bb.y);
            ext.z = std::max(ext.z, bb.z); ext.w = std::max(ext.w, bb.w);
        }
    }
    t.pt_offset = p0;
    t.pt_count = pt - p0;
    if (pt > p0) {
        t.ext_x0 = ext.x;
        t.ext_y0 = ext.y;
        t.ext_x1 = ext.z;
        t.ext_y1 = ext.w;
    }
    t.out_offset = out;
    out += (int64_t)r.ncols * r.nrows;
    t.site_offset = r.out_site ? site : -1;
    if (r.out_site) site += (int64_t)it.rw * (b1 - b0 + 1);
    it.nchunks = chunks.size() - c0;
    return true;
}

size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device bytes a batch needs in a slot arena: staging plus scratch.
size_t srv_footprint(const HostBatch& hb, int64_t pts, int64_t out, int64_t site, size_t nchunks) {
    const ScratchSizes z = scratch_sizes(hb);
    size_t b = al256(12 * (size_t)pts) + al256(4 * (size_t)pts) + al256(4 * (size_t)out) + al256(4 * (size_t)site) +
               al256(sizeof(SegChunk) * nchunks);
    const size_t parts[] = {z.tables, z.sc, z.ctr, z.pix, z.far, z.D, z.Dc, z.sorted, z.cnt, z.cnt, z.bsum,
                            z.bmask, z.smask, z.rownear, z.near};
    for (size_t p : parts) b += al256(p);
    return b;
}

// Launches a batch of planned requests on a free slot.
dnni_status srv_launch(dnni_server* s, SrvSlot& sl, std::vector<SrvItem>& items, const std::vector<SegChunk>& chunks,
                       int64_t pts, int64_t out, int64_t site) {
    dnni_ctx* c = s->ctx;
    const int ng = (int)items.size();
    std::vector<dnni_tile> tl(ng);
    std::vector<int> run;                       // items that have pixels
    for (int k = 0; k < ng; ++k) tl[k] = items[k].tile;
    for (int k = 0; k < ng; ++k)
        if (items[k].rw > 0) run.push_back(k);
    std::vector<dnni_tile> tr;
    for (int k : run) tr.push_back(tl[k]);
    HostBatch hb;
    std::vector<int> order;
    dnni_batch_options bo{};
    bo.small_radius = s->o.small_radius;
    bo.bin_target = s->o.bin_target;
    dnni_status rs = DNNI_OK;
    if (!tr.empty() && (rs = plan_batch(c, tr.data(), (int)tr.size(), bo, hb, order))) return rs;
    // carve the arena
    unsigned char* base = (unsigned char*)sl.arena.p;
    size_t off = 0;
    auto take = [&](size_t bytes) { unsigned char* p = base + off; off += al256(bytes); return p; };
    int32_t* gxyz = (int32_t*)take(12 * (size_t)pts);
    uint32_t* ggid = (uint32_t*)take(4 * (size_t)pts);
    float* gout = (float*)take(4 * (size_t)out);
    uint32_t* gsite = (uint32_t*)take(4 * (size_t)site);
    SegChunk* dch = (SegChunk*)take(sizeof(SegChunk) * chunks.size());
    DevArrays a;
    const ScratchSizes z = scratch_sizes(hb);
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
    if (off > sl.arena.cap) return set_err(c, DNNI_E_NOMEM, "batch exceeds the slot arena");
    cudaStream_t st = sl.st;
    // host staging of the tables and the chunk list (pinned, reused once the slot is free)
    const int nt = (int)tr.size();
    const size_t tbytes = nt ? TableLayout(nt).total : 0;
    const size_t need = tbytes + sizeof(SegChunk) * chunks.size();
    if (need > sl.h_tab_cap) {
        if (sl.h_tab) cudaFreeHost(sl.h_tab);
        sl.h_tab = nullptr;
        sl.h_tab_cap = 0;
        if (cudaMallocHost((void**)&sl.h_tab, need + need / 2) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, DNNI_E_NOMEM, "pinned staging of a slot");
        }
        sl.h_tab_cap = need + need / 2;
    }
    if (nt > sl.h_sc_cap) {
        if (sl.h_sc) cudaFreeHost(sl.h_sc);
        sl.h_sc = nullptr;
        if (cudaMallocHost((void**)&sl.h_sc, sizeof(Scalars) * (nt + 16)) != cudaSuccess) {
            cudaGetLastError();
            sl.h_sc_cap = 0;
            return set_err(c, DNNI_E_NOMEM, "pinned scalars of a slot");
        }
        sl.h_sc_cap = nt + 16;
    }
    if (nt) pack_tables(hb, sl.h_tab);
    if (!chunks.empty()) memcpy(sl.h_tab + tbytes, chunks.data(), sizeof(SegChunk) * chunks.size());
    CK(cudaEventRecord(sl.ev_t0, st));
    if (nt) CK(cudaMemcpyAsync(a.tables, sl.h_tab, tbytes, cudaMemcpyHostToDevice, st));
    if (!chunks.empty()) {
        CK(cudaMemcpyAsync(dch, sl.h_tab + tbytes, sizeof(SegChunk) * chunks.size(), cudaMemcpyHostToDevice, st));
        k_seg_gather<<<(int)chunks.size(), 256, 0, st>>>(dch, (const int32_t*)s->B.sxyz.p, (const uint32_t*)s->B.sgid.p,
                                                         gxyz, ggid);
    }
    if (nt) {
        const BatchTables bt = device_tables(a.tables, nt);
        launch_prologue(hb, bt, a, gxyz, st, false);
        launch_body(hb, bt, a, gxyz, ggid, gout, site ? gsite : nullptr, c->sm_count, st, nullptr, true);
        CK(cudaMemcpyAsync(sl.h_sc, a.sc, sizeof(Scalars) * nt, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(sl.h_ctr, a.ctr, sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
    }
    CK(cudaGetLastError());
    // results to the callers' host buffers: straight into pinned ones, via the
    // slot's pinned landing area otherwise (copied out when the batch ends),
    // so that no copy blocks this thread
    auto pinned = [](const void* p) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    size_t land = 0;
    std::vector<char> direct_h(ng, 0), direct_s(ng, 0);
    for (int k : run) {
        const SrvReq& q = s->reqs[items[k].ticket];
        const size_t cellsk = (size_t)q.r.ncols * q.r.nrows;
        direct_h[k] = pinned(q.r.out_h);
        if (!direct_h[k]) land += al256(4 * cellsk);
        if (q.r.out_site) {
            direct_s[k] = pinned(q.r.out_site);
            if (!direct_s[k]) land += al256(4 * cellsk);
        }
    }
    if (land > sl.h_out_cap) {
        if (sl.h_out) cudaFreeHost(sl.h_out);
        sl.h_out = nullptr;
        sl.h_out_cap = 0;
        if (cudaMallocHost((void**)&sl.h_out, land) != cudaSuccess) {
            cudaGetLastError();
            return set_err(c, DNNI_E_NOMEM, "pinned landing area of a slot");
        }
        sl.h_out_cap = land;
    }
    sl.landing.assign(ng, {SIZE_MAX, SIZE_MAX});
    size_t lo = 0;
    for (int k : run) {
        const SrvItem& it = items[k];
        const SrvReq& q = s->reqs[it.ticket];
        const size_t cellsk = (size_t)q.r.ncols * q.r.nrows;
        float* dh = q.r.out_h;
        if (!direct_h[k]) {
            sl.landing[k].first = lo;
            dh = (float*)(sl.h_out + lo);
            lo += al256(4 * cellsk);
        }
        CK(cudaMemcpyAsync(dh, gout + it.tile.out_offset, 4 * cellsk, cudaMemcpyDeviceToHost, st));
        if (q.r.out_site) {
            uint32_t* ds = q.r.out_site;
            if (!direct_s[k]) {
                sl.landing[k].second = lo;
                ds = (uint32_t*)(sl.h_out + lo);
                lo += al256(4 * cellsk);
            }
            // core cells inside the raster come from the site map, the rest
            // (off the cloud's box) have no site
            const int ci0 = std::max(0, it.rx0), cj0 = std::max(0, it.ry0);
            const int ci1 = std::min(q.r.ncols, it.rx0 + it.rw);
            const int cj1 = std::min(q.r.nrows, it.ry0 + (int)(it.tile.wp.raster_y1 - it.tile.wp.raster_y0));
            if (ci0 > 0 || cj0 > 0 || ci1 < q.r.ncols || cj1 < q.r.nrows)
                for (size_t m = 0; m < cellsk; ++m) ds[m] = 0xFFFFFFFFu;
            if (ci0 < ci1 && cj0 < cj1) {
                const uint32_t* src = gsite + it.tile.site_offset + (size_t)(cj0 - it.ry0) * it.rw + (ci0 - it.rx0);
                CK(cudaMemcpy2DAsync(ds + (size_t)cj0 * q.r.ncols + ci0, 4 * (size_t)q.r.ncols, src, 4 * (size_t)it.rw,
                                     4 * (size_t)(ci1 - ci0), cj1 - cj0, cudaMemcpyDeviceToHost, st));
            }
        }
    }
    CK(cudaEventRecord(sl.ev_t1, st));
    CK(cudaEventRecord(sl.ev, st));
    // batch position of each running item (no cost order: position = index in tr)
    sl.items = items;
    return DNNI_OK;
}

// Completion of a slot's batch: halo checks, results, requeues.
void srv_finish(dnni_server* s, SrvSlot& sl, cudaError_t e) {
    if (e == cudaSuccess && s->epoch) {
        float a = 0, b = 0;
        if (cudaEventElapsedTime(&a, s->epoch, sl.ev_t0) == cudaSuccess &&
            cudaEventElapsedTime(&b, s->epoch, sl.ev_t1) == cudaSuccess)
            s->busy.emplace_back(a, b);
        cudaGetLastError();
    }
    int pos = 0;
    for (const SrvItem& it : sl.items) {
        SrvReq& q = s->reqs[it.ticket];
        if (e != cudaSuccess) {
            q.status = DNNI_E_CUDA;
        } else if (it.rw == 0) {
            const size_t cellsk = (size_t)q.r.ncols * q.r.nrows;
            for (size_t k = 0; k < cellsk; ++k) q.r.out_h[k] = q.r.nodata;
            if (q.r.out_site)
                for (size_t k = 0; k < cellsk; ++k) q.r.out_site[k] = 0xFFFFFFFFu;
        } else {
            const Scalars& sc = sl.h_sc[pos++];
            int mr2 = -1;
            for (int l = 0; l < kStatSlots; ++l) mr2 = std::max(mr2, sc.max_r2[l]);
            // no site found (mr2 < 0): the box held no point, so unless it
            // covers every bucket the sites lie beyond it (the occupancy bound
            // rules this out; the check keeps it from being accepted anyway)
            const bool none = mr2 < 0;
            const double R = std::sqrt((double)std::max(mr2, 0) + 1.0);
            const bool okA = it.all_raster || none || R <= it.hr - 2;
            const bool okB = it.all_buckets || (!none && R <= it.hr);
            if (sl.h_ctr->err & kErrRange) {
                q.status = DNNI_E_RANGE;
            } else if (!(okA && okB)) {
                q.hr_force = none ? std::max(2 * it.hr, 8) : std::max(2 * it.hr, (int)std::ceil(R) + 3);
                q.runs++;
                s->queue.push_front(it.ticket);
                continue;
            }
        }
        if (!q.status && it.rw > 0) {
            const size_t k = &it - sl.items.data();
            const size_t cellsk = (size_t)q.r.ncols * q.r.nrows;
            if (k < sl.landing.size() && sl.landing[k].first != SIZE_MAX)
                memcpy(q.r.out_h, sl.h_out + sl.landing[k].first, 4 * cellsk);
            if (k < sl.landing.size() && q.r.out_site && sl.landing[k].second != SIZE_MAX)
                memcpy(q.r.out_site, sl.h_out + sl.landing[k].second, 4 * cellsk);
        }
        q.done = true;
        q.t_done = now_s();
        q.halo = it.hr;
        q.batch = (int)sl.items.size();
        q.runs++;
        if (q.status) {
            s->failed++;
        } else {
            s->completed++;
            s->cells += (int64_t)q.r.ncols * q.r.nrows;
            s->points += it.tile.pt_count;
            q.points = it.tile.pt_count;
        }
    }
    sl.items.clear();
    sl.busy = false;
}

void srv_fail(dnni_server* s, uint64_t ticket, int status) {
    SrvReq& q = s->reqs[ticket];
    q.status = status;
    q.done = true;
    q.t_done = now_s();
    s->failed++;
}

void srv_loop(dnni_server* s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    std::vector<SegChunk> chunks;
    for (;;) {
        bool any_busy = false, progressed = false;
        for (SrvSlot& sl : s->slots) {
            if (!sl.busy) continue;
            const cudaError_t e = cudaEventQuery(sl.ev);
            if (e == cudaErrorNotReady) {
                any_busy = true;
                continue;
            }
            if (e != cudaSuccess) cudaGetLastError();
            srv_finish(s, sl, e);
            progressed = true;
        }
        if (progressed) s->cv.notify_all();
        // fill free slots from the queue, in arrival order
        for (SrvSlot& sl : s->slots) {
            if (sl.busy || s->queue.empty()) continue;
            std::vector<SrvItem> items;
            chunks.clear();
            int64_t pt = 0, out = 0, site = 0;
            while (!s->queue.empty() && (int)items.size() < s->o.max_batch) {
                const uint64_t tk = s->queue.front();
                SrvReq& q = s->reqs[tk];
                const size_t ch0 = chunks.size();
                const int64_t pt0 = pt, out0 = out, site0 = site;
                SrvItem it;
                int why = DNNI_OK;
                if (!srv_plan(s, tk, q, chunks, pt, out, site, it, &why)) {
                    s->queue.pop_front();
                    srv_fail(s, tk, why);
                    progressed = true;
                    continue;
                }
                items.push_back(it);
                // footprint of the batch with this request
                std::vector<dnni_tile> tr;
                for (const SrvItem& x : items)
                    if (x.rw > 0) tr.push_back(x.tile);
                HostBatch hb;
                std::vector<int> order;
                dnni_batch_options bo{};
                bo.small_radius = s->o.small_radius;
                bo.bin_target = s->o.bin_target;
                if (!tr.empty() && plan_batch(s->ctx, tr.data(), (int)tr.size(), bo, hb, order)) {
                    items.pop_back();
                    chunks.resize(ch0);
                    pt = pt0; out = out0; site = site0;
                    s->queue.pop_front();
                    srv_fail(s, tk, DNNI_E_INVAL);
                    progressed = true;
                    continue;
                }
                if (srv_footprint(hb, pt, out, site, chunks.size()) > sl.arena.cap) {
                    items.pop_back();
                    chunks.resize(ch0);
                    pt = pt0; out = out0; site = site0;
                    if (items.empty()) {          // alone it does not fit either
                        s->queue.pop_front();
                        srv_fail(s, tk, DNNI_E_NOMEM);
                        progressed = true;
                        continue;
                    }
                    break;
                }
                s->queue.pop_front();
            }
            if (items.empty()) continue;
            const double t = now_s();
            for (const SrvItem& it : items) s->reqs[it.ticket].t_launch = t;
            const dnni_status rs = srv_launch(s, sl, items, chunks, pt, out, site);
            if (rs) {
                for (const SrvItem& it : items) srv_fail(s, it.ticket, rs);
            } else {
                sl.busy = true;
                any_busy = true;
                s->batches++;
            }
            progressed = true;
        }
        if (progressed) s->cv.notify_all();
        if (s->stop && s->queue.empty() && !any_busy) break;
        if (any_busy)
            s->cv.wait_for(lk, std::chrono::microseconds(50));
        else if (s->queue.empty())
            s->cv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
    }
}

}  // namespace

extern "C" {

dnni_status dnni_server_create(dnni_ctx* c, const int32_t* h_xyz, int64_t n, const dnni_server_options* opt,
                               dnni_server** out) {
    if (!c || !out || n < 0 || (n > 0 && !h_xyz)) return DNNI_E_INVAL;
    *out = nullptr;
    c->err.clear();
    DeviceGuard g(c->device);
    if ((uint64_t)n >= 0xFFFFFFFFull) return set_err(c, DNNI_E_INVAL, "more points than 32-bit site ids can name");
    dnni_server_options o{};
    if (opt) o = *opt;
    if (!o.bucket) o.bucket = 25600;
    if (!o.slots) o.slots = 2;
    if (!o.max_batch) o.max_batch = 64;
    if (!o.slot_bytes) o.slot_bytes = 16ull << 30;
    if (!o.small_radius) o.small_radius = c->s.small_radius;
    if (!o.bin_target) o.bin_target = c->s.bin_target;
    if (o.bucket < 1 || o.fine < 0 || o.slots < 1 || o.slots > 8 || o.max_batch < 1 || o.max_batch > 4096 ||
        o.small_radius < 1 || o.small_radius > kMaxSmallRadius || o.bin_target < 0)
        return set_err(c, DNNI_E_INVAL, "bad server options");
    const double t0 = now_s();
    dnni_server* s = new dnni_server();
    s->ctx = c;
    s->o = o;
    s->n = n;
    cudaStream_t st = c->stream;
    dnni_status rs = upload_points(c, st, h_xyz, n, s->B);
    int ext[4] = {INT_MAX, INT_MAX, INT_MIN, INT_MIN};
    DevBuf ext_d;
    if (!rs) rs = dnni_ensure(c, ext_d, sizeof(ext));
    if (!rs) {
        cudaError_t e = cudaMemcpyAsync(ext_d.p, ext, sizeof(ext), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && n > 0)
            k_seg_extent<<<c->sm_count * 8, 256, 0, st>>>((const int32_t*)s->B.xin.p, n, (int*)ext_d.p);
        if (e == cudaSuccess) e = cudaMemcpyAsync(ext, ext_d.p, sizeof(ext), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rs = cuda_err(c, e, "cloud extent");
    }
    dnni_release(ext_d, c);
    if (!rs) {
        if (n == 0) ext[0] = ext[1] = ext[2] = ext[3] = 0;
        s->wx0 = ext[0];
        s->wy0 = ext[1];
        s->wx1 = ext[2];
        s->wy1 = ext[3];
        s->G.ox = ext[0];
        s->G.oy = ext[1];
        s->G.w = o.bucket;
        s->G.nbx = (int)((s->wx1 - s->wx0) / o.bucket + 1);
        s->G.nby = (int)((s->wy1 - s->wy0) / o.bucket + 1);
        if ((int64_t)s->G.nbx * s->G.nby > (1 << 26)) rs = set_err(c, DNNI_E_INVAL, "bucket side too small for the cloud");
    }
    float ms_up = 0, ms_bk = 0;
    if (!rs) rs = bucket_uploaded(c, st, s->G, n, s->B, s->start, s->bbox, &ms_up, &ms_bk);
    if (!rs) {
        const long long span = std::max(s->wx1 - s->wx0, s->wy1 - s->wy0) + 1;
        s->fw = o.fine ? o.fine : std::max<long long>(1600, (span + 4095) / 4096);
        s->nfx = (int)((s->wx1 - s->wx0) / s->fw + 1);
        s->nfy = (int)((s->wy1 - s->wy0) / s->fw + 1);
        rs = occupancy_edt(c, st, s->G, s->fw, s->nfx, s->nfy, s->B, n, s->edt2);
    }
    if (!rs) {
        s->slots.resize(o.slots);
        for (SrvSlot& sl : s->slots) {
            if (cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking) != cudaSuccess ||
                cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreate(&sl.ev_t0) != cudaSuccess || cudaEventCreate(&sl.ev_t1) != cudaSuccess ||
                cudaMallocHost((void**)&sl.h_ctr, sizeof(BatchCounters)) != cudaSuccess) {
                cudaGetLastError();
                rs = set_err(c, DNNI_E_CUDA, "slot streams");
                break;
            }
            if ((rs = dnni_ensure(c, sl.arena, o.slot_bytes))) break;
        }
    }
    if (rs) {
        for (SrvSlot& sl : s->slots) {
            dnni_release(sl.arena, c);
            if (sl.st) cudaStreamDestroy(sl.st);
            if (sl.ev) cudaEventDestroy(sl.ev);
            if (sl.ev_t0) cudaEventDestroy(sl.ev_t0);
            if (sl.ev_t1) cudaEventDestroy(sl.ev_t1);
            if (sl.h_ctr) cudaFreeHost(sl.h_ctr);
        }
        s->B.release(c);
        delete s;
        return rs;
    }
    if (cudaEventCreate(&s->epoch) != cudaSuccess || cudaEventRecord(s->epoch, st) != cudaSuccess) {
        cudaGetLastError();
        if (s->epoch) cudaEventDestroy(s->epoch);
        s->epoch = nullptr;                      // no device time line, nothing else lost
    }
    s->ms_build = 1000.0 * (now_s() - t0);
    s->th = std::thread(srv_loop, s);
    *out = s;
    return DNNI_OK;
}

dnni_status dnni_server_submit(dnni_server* s, const dnni_request* r, uint64_t* ticket) {
    if (!s || !r || !ticket) return DNNI_E_INVAL;
    if (r->ncols <= 0 || r->nrows <= 0 || r->ncols > 32767 || r->nrows > 32767 || r->cell_size <= 0 || !r->out_h)
        return DNNI_E_INVAL;
    // every point and raster pixel must lie within +-2^30 LAS units of the
    // request origin
    const long long lim = (1LL << 30) - 1;
    const long long far_x = std::max(std::llabs(s->wx0 - r->x0), std::llabs(s->wx1 - r->x0));
    const long long far_y = std::max(std::llabs(s->wy0 - r->y0), std::llabs(s->wy1 - r->y0));
    if (far_x + (long long)r->cell_size > lim || far_y + (long long)r->cell_size > lim ||
        (long long)r->ncols * r->cell_size > lim || (long long)r->nrows * r->cell_size > lim)
        return DNNI_E_RANGE;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return DNNI_E_STATE;
    const uint64_t t = s->next++;
    SrvReq& q = s->reqs[t];
    q.r = *r;
    q.t_submit = now_s();
    s->queue.push_back(t);
    s->submitted++;
    *ticket = t;
    s->cv.notify_all();
    return DNNI_OK;
}

dnni_status dnni_server_wait(dnni_server* s, uint64_t ticket, double timeout_s, dnni_request_result* res) {
    if (!s) return DNNI_E_INVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return DNNI_E_INVAL;
    auto ready = [&] { return s->reqs[ticket].done; };
    if (timeout_s < 0) {
        s->cv.wait(lk, ready);
    } else if (!s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
        return DNNI_E_TIMEOUT;
    }
    const SrvReq q = s->reqs[ticket];
    s->reqs.erase(ticket);
    if (res) {
        memset(res, 0, sizeof(*res));
        res->status = q.status;
        res->halo = q.halo;
        res->ms_queue = 1000.0 * (q.t_launch - q.t_submit);
        res->ms_latency = 1000.0 * (q.t_done - q.t_submit);
        res->points = q.points;
        res->cells = (int64_t)q.r.ncols * q.r.nrows;
        res->batch_size = q.batch;
        res->runs = q.runs;
    }
    return (dnni_status)q.status;
}

dnni_status dnni_server_get_stats(dnni_server* s, dnni_server_stats* st) {
    if (!s || !st) return DNNI_E_INVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->batches = s->batches;
    st->cells = s->cells;
    st->points = s->points;
    st->resident_bytes = (int64_t)(s->B.sxyz.cap + s->B.sgid.cap);
    st->ms_build = s->ms_build;
    // the batches' device time line: time with any slot busy, with two or
    // more busy at once, and the span from the first start to the last end
    std::vector<std::pair<double, int>> ends;
    for (const auto& iv : s->busy) {
        ends.emplace_back(iv.first, +1);
        ends.emplace_back(iv.second, -1);
    }
    std::sort(ends.begin(), ends.end(), [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
        return x.first < y.first || (x.first == y.first && x.second < y.second);
    });
    int depth = 0;
    double prev = 0;
    for (const auto& e : ends) {
        if (depth >= 1) st->ms_device_busy += e.first - prev;
        if (depth >= 2) st->ms_device_overlap += e.first - prev;
        depth += e.second;
        prev = e.first;
    }
    if (!ends.empty()) st->ms_device_span = ends.back().first - ends.front().first;
    return DNNI_OK;
}

dnni_status dnni_server_destroy(dnni_server* s) {
    if (!s) return DNNI_E_INVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->th.joinable()) s->th.join();
    dnni_ctx* c = s->ctx;
    {
        DeviceGuard g(c->device);
        for (SrvSlot& sl : s->slots) {
            if (sl.st) cudaStreamSynchronize(sl.st);
            dnni_release(sl.arena, c);
            if (sl.st) cudaStreamDestroy(sl.st);
            if (sl.ev) cudaEventDestroy(sl.ev);
            if (sl.ev_t0) cudaEventDestroy(sl.ev_t0);
            if (sl.ev_t1) cudaEventDestroy(sl.ev_t1);
            if (sl.h_tab) cudaFreeHost(sl.h_tab);
            if (sl.h_out) cudaFreeHost(sl.h_out);
            if (sl.h_sc) cudaFreeHost(sl.h_sc);
            if (sl.h_ctr) cudaFreeHost(sl.h_ctr);
        }
        if (s->epoch) cudaEventDestroy(s->epoch);
        s->B.release(c);
    }
    delete s;
    return DNNI_OK;
}

}  // extern "C"
