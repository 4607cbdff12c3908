// dnni_engine.cu -- context, device scratch and the per-work-package pipeline
// behind the C ABI in include/dnni.h.
//
// Reference counterparts:
//   nni::init / cuda_nni::init          nni.cpp:569-598, cuda_nni.cu:641-669
//   nni::setupRun / cuda_nni::setup_run nni.cpp:601-668, cuda_nni.cu:110-126
//   nni::performNNI                     nni.cpp:870-944
//   nni::clearRenderbuffers / cleanup   nni.cpp:362-379, 563-566
//   nni::printTimes                     nni.cpp:554-560
// The GL context, framebuffers, renderbuffers and GL/CUDA interop of the
// reference have no counterpart: the engine works on plain device buffers.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dnni.h"
#include "dnni_internal.h"
#include "dnni_kernels.cuh"
#include "dnni_plan.h"

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

int grid_for(int64_t n, int threads, int cap) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    return (int)(b < cap ? b : cap);
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

dnni_status dnni_tile_geometry(dnni_ctx* c, const dnni_workpackage* wp, int64_t n, TileParams& t) {
    const char* msg = "";
    dnni_status st = plan_geometry(wp, n, c->s.small_radius, t, &msg);
    if (st) return set_err(c, st, msg);
    return DNNI_OK;
}

void dnni_bin_grid(const dnni_ctx* c, const int32_t bbox[6], int64_t n, TileParams& t) {
    plan_bins(bbox, n, (double)c->s.bin_target, t);
}

// Worklist capacity: every dense warp (32 pixels of a tile row, the raster
// padded to whole tiles) may append one group of 32 slots.
static int64_t far_slots(const TileParams& t) {
    return (int64_t)((t.rw + kTileX - 1) / kTileX * kTileX) * ((t.rh + kTileY - 1) / kTileY * kTileY);
}

// Nearest-site passes: dense tiles, then the far worklist.
static void launch_nearest(const TileParams& t, const int4* sorted, const int* start, const uint64_t* bmask,
                           const uint64_t* smask, int* rownear, int64_t* near, int2* pix, uint32_t* site, int2* far,
                           Scalars* sc, int sms, cudaStream_t st) {
    static thread_local int attr_dev = -1;
    int dev = 0;
    cudaGetDevice(&dev);
    if (attr_dev != dev) {
        cudaFuncSetAttribute(k_near_dense, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDenseSmem);
        attr_dev = dev;
    }
    dim3 blk(32, 8), grd((t.rw + kTileX - 1) / kTileX, (t.rh + kTileY - 1) / kTileY);
    k_near_dense<<<grd, blk, kDenseSmem, st>>>(t, sorted, start, pix, site, far, sc);
    if (t.npts > 0) {
        const int n1x = t.bg.nbx >> 3, n1y = t.bg.nby >> 3;
        k_block_rows<<<(n1y + 127) / 128, 128, 0, st>>>(t.bg, bmask, rownear);
        k_block_near<<<(int)(((int64_t)n1x * n1y + 255) / 256), 256, 0, st>>>(t.bg, rownear, near);
        k_near_far<<<sms * 6, 256, 0, st>>>(t, sorted, start, bmask, smask, near, far, pix, site, sc);
    }
}

static void launch_final(const TileParams& t, const int2* pix, Scalars* sc, const unsigned long long* S,
                         const int* Sc, float* h, cudaStream_t st) {
    dim3 blk(32, 16), grd((t.ncols + 31) / 32, (t.nrows + 15) / 16);
    switch (t.rs) {
        case 1: k_final<1><<<grd, blk, 0, st>>>(t, pix, sc, S, Sc, h); break;
        case 2: k_final<2><<<grd, blk, 0, st>>>(t, pix, sc, S, Sc, h); break;
        case 4: k_final<4><<<grd, blk, 0, st>>>(t, pix, sc, S, Sc, h); break;
        case 5: k_final<5><<<grd, blk, 0, st>>>(t, pix, sc, S, Sc, h); break;
        case 6: k_final<6><<<grd, blk, 0, st>>>(t, pix, sc, S, Sc, h); break;
        default: k_final<3><<<grd, blk, 0, st>>>(t, pix, sc, S, Sc, h); break;
    }
}

// The plain per-work-package pipeline on device buffers.
dnni_status dnni_run_device(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* d_xyz, const uint32_t* d_gid,
                            int64_t n, float* d_h, uint32_t* d_site, cudaStream_t st, dnni_stats* stats) {
    TileParams t;
    dnni_status rs = dnni_tile_geometry(c, wp, n, t);
    if (rs) return rs;
    if (!d_h) return set_err(c, DNNI_E_INVAL, "output grid pointer is NULL");
    if (n > 0 && !d_xyz) return set_err(c, DNNI_E_INVAL, "point pointer is NULL");
    t.has_gid = d_gid ? 1 : 0;
    const int64_t npix = (int64_t)t.rw * t.rh;
    const int64_t cells = (int64_t)t.ncols * t.nrows;
    const bool timing = stats || (c->s.flags & DNNI_F_TIMING);

    if ((rs = dnni_ensure(c, c->pix, sizeof(int2) * npix))) return rs;
    if ((rs = dnni_ensure(c, c->D, sizeof(unsigned long long) * cells))) return rs;
    if ((rs = dnni_ensure(c, c->Dc, sizeof(int) * cells))) return rs;
    if (n > 0) {
        if ((rs = dnni_ensure(c, c->rank, sizeof(int) * n))) return rs;
        if ((rs = dnni_ensure(c, c->sorted, sizeof(int4) * n))) return rs;
    }
    Scalars* sc = c->d_sc;
    if (timing) CK(cudaEventRecord(c->ev[0], st));
    k_init_scalars<<<1, 32, 0, st>>>(sc);
    if (n > 0) {
        k_bbox<<<grid_for(n, 256, c->sm_count * 8), 256, 0, st>>>(d_xyz, n, t.ox, t.oy, sc);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(c->h_sc, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c->h_sc->err & kErrRange)
            return set_err(c, DNNI_E_RANGE, "a point lies beyond +-2^30 LAS units of the work-package origin");
    }
    dnni_bin_grid(c, c->h_sc->bbox, n, t);
    if (n > 0) {
        const int64_t m = t.bg.nbins + 1;
        const int nb = (int)((m + kScanTile - 1) / kScanTile);
        if ((rs = dnni_ensure(c, c->cnt, sizeof(int) * m))) return rs;
        if ((rs = dnni_ensure(c, c->start, sizeof(int) * m))) return rs;
        if ((rs = dnni_ensure(c, c->bsum, sizeof(int) * nb))) return rs;
        int* cnt = (int*)c->cnt.p;
        int* start = (int*)c->start.p;
        int* bsum = (int*)c->bsum.p;
        CK(cudaMemsetAsync(cnt, 0, sizeof(int) * m, st));
        const int g = grid_for(n, 256, c->sm_count * 16);
        k_bin_count<<<g, 256, 0, st>>>(d_xyz, n, t.ox, t.oy, t.bg, cnt, (int*)c->rank.p);
        k_scan_partial<<<nb, kScanThreads, 0, st>>>(cnt, m, bsum);
        k_scan_bsum<<<1, 1024, 0, st>>>(bsum, nb);
        k_scan_final<<<nb, kScanThreads, 0, st>>>(cnt, m, bsum, start);
        k_bin_scatter<<<g, 256, 0, st>>>(d_xyz, d_gid, n, t.ox, t.oy, t.bg, start, (int*)c->rank.p,
                                         (int4*)c->sorted.p);
        const int64_t nblk = t.bg.nbins / kBinsPerBlock, nsup = t.bg.nbins / kBinsPerSuper;
        if ((rs = dnni_ensure(c, c->bmask, sizeof(uint64_t) * nblk))) return rs;
        if ((rs = dnni_ensure(c, c->smask, sizeof(uint64_t) * nsup))) return rs;
        k_block_masks<<<(int)((nblk * 32 + 255) / 256), 256, 0, st>>>(start, nblk, (uint64_t*)c->bmask.p);
        k_super_masks<<<(int)((nsup * 32 + 255) / 256), 256, 0, st>>>((const uint64_t*)c->bmask.p, nsup,
                                                                      (uint64_t*)c->smask.p);
        CK(cudaGetLastError());
    }
    if (timing) CK(cudaEventRecord(c->ev[1], st));
    {
        if ((rs = dnni_ensure(c, c->far, sizeof(int2) * far_slots(t)))) return rs;
        const int64_t nblk = n > 0 ? t.bg.nbins / kBinsPerBlock : 1;
        if ((rs = dnni_ensure(c, c->rownear, sizeof(int) * nblk))) return rs;
        if ((rs = dnni_ensure(c, c->near, sizeof(int64_t) * nblk))) return rs;
        launch_nearest(t, (const int4*)c->sorted.p, (const int*)c->start.p, (const uint64_t*)c->bmask.p,
                       (const uint64_t*)c->smask.p, (int*)c->rownear.p, (int64_t*)c->near.p, (int2*)c->pix.p, d_site,
                       (int2*)c->far.p, sc, c->sm_count, st);
        k_decide<<<1, 32, 0, st>>>(sc, npix);
        CK(cudaGetLastError());
    }
    if (timing) CK(cudaEventRecord(c->ev[2], st));
    {
        CK(cudaMemsetAsync(c->D.p, 0, sizeof(unsigned long long) * cells, st));
        CK(cudaMemsetAsync(c->Dc.p, 0, sizeof(int) * cells, st));
        dim3 blk(32, 8), grd((t.rw + 31) / 32, (t.rh + 7) / 8);
        k_scatter_spans<<<grd, blk, 0, st>>>(t, (const int2*)c->pix.p, sc, (unsigned long long*)c->D.p, (int*)c->Dc.p);
        CK(cudaGetLastError());
    }
    if (timing) CK(cudaEventRecord(c->ev[3], st));
    {
        k_rowscan<unsigned long long><<<t.nrows, kScanThreads, 0, st>>>((unsigned long long*)c->D.p, t.ncols, sc, 0);
        k_rowscan<int><<<t.nrows, kScanThreads, 0, st>>>((int*)c->Dc.p, t.ncols, sc, 1);
        launch_final(t, (const int2*)c->pix.p, sc, (const unsigned long long*)c->D.p, (const int*)c->Dc.p, d_h, st);
        CK(cudaGetLastError());
    }
    if (timing) CK(cudaEventRecord(c->ev[4], st));
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
        }
    }
    if (stats) {
        CK(cudaMemcpyAsync(c->h_sc, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const Scalars& h = *c->h_sc;
        stats->n_points = n;
        stats->n_cells = cells;
        stats->n_pixels = npix;
        int64_t big = 0, sp = 0, nod = 0;
        int mx = -1;
        for (int k = 0; k < kStatSlots; ++k) {
            big += (int64_t)h.big_pixels[k];
            sp += (int64_t)h.spans[k];
            nod += (int64_t)h.nodata[k];
            mx = std::max(mx, h.max_r2[k]);
        }
        stats->big_pixels = big;
        stats->spans = sp;
        stats->nodata_cells = nod;
        stats->max_r2 = mx;
        stats->packed = h.packed;
        stats->bin_size = t.bg.bs;
    }
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
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) { delete c; return DNNI_E_CUDA; }
    for (auto& e : c->ev)
        if (cudaEventCreate(&e) != cudaSuccess) { dnni_destroy(c); return DNNI_E_CUDA; }
    if (cudaMalloc(&c->d_sc, sizeof(Scalars)) != cudaSuccess ||
        cudaMallocHost(&c->h_sc, sizeof(Scalars)) != cudaSuccess) {
        dnni_destroy(c);
        return DNNI_E_NOMEM;
    }
    memset(c->h_sc, 0, sizeof(Scalars));
    *out = c;
    return DNNI_OK;
}

dnni_status dnni_destroy(dnni_ctx* c) {
    if (!c) return DNNI_E_INVAL;
    {
        DeviceGuard g(c->device);
        if (c->stream) cudaStreamSynchronize(c->stream);
        dnni_free_all(c);
        if (c->d_sc) cudaFree(c->d_sc);
        if (c->h_sc) cudaFreeHost(c->h_sc);
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
    dnni_status rs = dnni_tile_geometry(c, wp, max_points, t);
    if (rs) return rs;
    const int64_t npix = (int64_t)t.rw * t.rh, cells = (int64_t)t.ncols * t.nrows;
    if ((rs = dnni_ensure(c, c->pix, sizeof(int2) * npix))) return rs;
    if ((rs = dnni_ensure(c, c->D, sizeof(unsigned long long) * cells))) return rs;
    if ((rs = dnni_ensure(c, c->Dc, sizeof(int) * cells))) return rs;
    if (max_points > 0) {
        if ((rs = dnni_ensure(c, c->rank, sizeof(int) * max_points))) return rs;
        if ((rs = dnni_ensure(c, c->sorted, sizeof(int4) * max_points))) return rs;
        // bins are sized from the points; reserve for the densest grid allowed
        int32_t bb[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, 0, 0};
        dnni_bin_grid(c, bb, max_points, t);
        const int64_t m = t.bg.nbins + 1;
        if ((rs = dnni_ensure(c, c->cnt, sizeof(int) * m))) return rs;
        if ((rs = dnni_ensure(c, c->start, sizeof(int) * m))) return rs;
        if ((rs = dnni_ensure(c, c->bsum, sizeof(int) * ((m + kScanTile - 1) / kScanTile)))) return rs;
    }
    return DNNI_OK;
}

dnni_status dnni_interpolate_segment_device(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* d_xyz,
                                            const uint32_t* d_gid, int64_t n, float* d_h, uint32_t* d_site,
                                            void* stream, dnni_stats* stats) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    if (stats) memset(stats, 0, sizeof(*stats));
    return dnni_run_device(c, wp, d_xyz, d_gid, n, d_h, d_site, st, stats);
}

dnni_status dnni_interpolate_segment(dnni_ctx* c, const dnni_workpackage* wp, const int32_t* xyz, const uint32_t* gid,
                                     int64_t n, float* out_h, uint32_t* out_site, dnni_stats* stats) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    if (!out_h) return set_err(c, DNNI_E_INVAL, "output grid pointer is NULL");
    if (n > 0 && !xyz) return set_err(c, DNNI_E_INVAL, "point pointer is NULL");
    DeviceGuard g(c->device);
    TileParams t;
    dnni_status rs = dnni_tile_geometry(c, wp, n, t);
    if (rs) return rs;
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
    rs = dnni_run_device(c, wp, (const int32_t*)c->in_xyz.p, gid ? (const uint32_t*)c->in_gid.p : nullptr, n,
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

}  // extern "C"

void dnni_free_all(dnni_ctx* c) {
    DevBuf* bufs[] = {&c->rank, &c->sorted, &c->cnt, &c->start, &c->bsum, &c->pix, &c->D, &c->Dc,
                      &c->bmask, &c->smask, &c->far, &c->rownear, &c->near,
                      &c->in_xyz, &c->in_gid, &c->out_h, &c->out_site};
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
// looked up once per device, with that device current, on the first call.
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

struct ArenaCursor {
    size_t off = 0;
    size_t take(size_t bytes) {
        const size_t o = off;
        off = (off + bytes + 255) & ~(size_t)255;
        return o;
    }
    bool fits() const { return off <= kNoAllocScratchBytes; }
};

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
    const int64_t npix = (int64_t)t.rw * t.rh, cells = (int64_t)t.ncols * t.nrows;
    ArenaCursor a;
    const size_t o_sc = a.take(sizeof(Scalars));
    const size_t o_pix = a.take(sizeof(int2) * npix);
    const size_t o_D = a.take(sizeof(unsigned long long) * cells);
    const size_t o_Dc = a.take(sizeof(int) * cells);
    const size_t o_rank = n > 0 ? a.take(sizeof(int) * n) : 0;
    const size_t o_sorted = n > 0 ? a.take(sizeof(int4) * n) : 0;
    const size_t o_far = a.take(sizeof(int2) * far_slots(t));
    if (!a.fits()) return DNNI_E_SCRATCH;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st = (cudaStream_t)stream;
    Scalars* sc = (Scalars*)(base + o_sc);
    int2* pix = (int2*)(base + o_pix);
    unsigned long long* D = (unsigned long long*)(base + o_D);
    int* Dc = (int*)(base + o_Dc);
    int* rank = (int*)(base + o_rank);
    int4* sorted = (int4*)(base + o_sorted);
    // the array keeps the previous call's contents: every region that must
    // start at zero (scalars, bin counts, span words) is cleared below
    k_init_scalars<<<1, 32, 0, st>>>(sc);
    Scalars hsc;
    memset(&hsc, 0, sizeof(hsc));
    if (n > 0) {
        k_bbox<<<grid_for(n, 256, sms * 8), 256, 0, st>>>(d_xyz, n, t.ox, t.oy, sc);
        if (cudaMemcpyAsync(&hsc, sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return DNNI_E_CUDA;
        }
        if (hsc.err & kErrRange) return DNNI_E_RANGE;
    }
    plan_bins(hsc.bbox, n, 0.0, t);
    int* start = nullptr;
    uint64_t* bmask = nullptr;
    uint64_t* smask = nullptr;
    int* rownear = nullptr;
    int64_t* nearb = nullptr;
    if (n > 0) {
        const int64_t m = t.bg.nbins + 1;
        const int nb = (int)((m + kScanTile - 1) / kScanTile);
        int* cnt = (int*)(base + a.take(sizeof(int) * m));
        start = (int*)(base + a.take(sizeof(int) * m));
        int* bsum = (int*)(base + a.take(sizeof(int) * nb));
        if (!a.fits()) return DNNI_E_SCRATCH;
        if (cudaMemsetAsync(cnt, 0, sizeof(int) * m, st) != cudaSuccess) return DNNI_E_CUDA;
        const int g = grid_for(n, 256, sms * 16);
        k_bin_count<<<g, 256, 0, st>>>(d_xyz, n, t.ox, t.oy, t.bg, cnt, rank);
        k_scan_partial<<<nb, kScanThreads, 0, st>>>(cnt, m, bsum);
        k_scan_bsum<<<1, 1024, 0, st>>>(bsum, nb);
        k_scan_final<<<nb, kScanThreads, 0, st>>>(cnt, m, bsum, start);
        k_bin_scatter<<<g, 256, 0, st>>>(d_xyz, d_gid, n, t.ox, t.oy, t.bg, start, rank, sorted);
        const int64_t nblk = t.bg.nbins / kBinsPerBlock, nsup = t.bg.nbins / kBinsPerSuper;
        bmask = (uint64_t*)(base + a.take(sizeof(uint64_t) * nblk));
        smask = (uint64_t*)(base + a.take(sizeof(uint64_t) * nsup));
        if (!a.fits()) return DNNI_E_SCRATCH;
        k_block_masks<<<(int)((nblk * 32 + 255) / 256), 256, 0, st>>>(start, nblk, bmask);
        k_super_masks<<<(int)((nsup * 32 + 255) / 256), 256, 0, st>>>(bmask, nsup, smask);
        rownear = (int*)(base + a.take(sizeof(int) * nblk));
        nearb = (int64_t*)(base + a.take(sizeof(int64_t) * nblk));
        if (!a.fits()) return DNNI_E_SCRATCH;
    }
    {
        dim3 blk(32, 8), grd((t.rw + 31) / 32, (t.rh + 7) / 8);
        launch_nearest(t, sorted, start, bmask, smask, rownear, nearb, pix, d_site, (int2*)(base + o_far), sc, sms, st);
        k_decide<<<1, 32, 0, st>>>(sc, npix);
        if (cudaMemsetAsync(D, 0, sizeof(unsigned long long) * cells, st) != cudaSuccess ||
            cudaMemsetAsync(Dc, 0, sizeof(int) * cells, st) != cudaSuccess)
            return DNNI_E_CUDA;
        k_scatter_spans<<<grd, blk, 0, st>>>(t, pix, sc, D, Dc);
    }
    k_rowscan<unsigned long long><<<t.nrows, kScanThreads, 0, st>>>(D, t.ncols, sc, 0);
    k_rowscan<int><<<t.nrows, kScanThreads, 0, st>>>(Dc, t.ncols, sc, 1);
    launch_final(t, pix, sc, D, Dc, d_h, st);
    if (cudaGetLastError() != cudaSuccess) return DNNI_E_CUDA;
    return DNNI_OK;
}
