// dnni_compat.cuh -- the reference's own default semantics on the GPU
// (dnni_interpolate_compat): square site regions, a pixel lattice `scale`
// times finer than the cells, float32 lifted-plane depths with the
// later-drawn site winning equal depths, square query regions, int32 z-codes
// summed with wrap-around and a truncating divide.  Included by
// dnni_engine.cu.
//
// Follows nni::performNNI for timeRadius == 0 with the plane algorithm:
//   pixel_offset and raster size                   nni.cpp:879-886
//   site squares, z-code, depth test (LEQUAL)      nni.cpp:171-230, 470-479, 538-549, 733-737
//   query squares tested against the stored depth  nni.cpp:483-534, 803-807
//   int32 numer/denom, truncating divide           cuda_nni.cu:423-448, 491-503
//   dequantisation                                 nni.cpp:836-848
// evaluating each plane at pixel centres over the half-open square
// [x - r, x + r) x [y - r, y + r); the GL rasteriser's fill rule and its
// depth interpolation are not reproduced.  Every floating-point operation is
// written with an explicit rounding intrinsic, in the order the formulas
// give, so that no multiply-add is fused and the results are those of the
// same formulas evaluated in IEEE single and double precision on the host.
#pragma once

namespace dnni {

struct CompatGeom {
    double pixel_size, left, bottom, rs, rq, qspacing;
    float hw;
    int32_t xp, yp, ncols, nrows, z_offset, z_mult;
    float ox, oy;
};

// A site's (or query's) lifted plane: its slopes and offset depend on the
// point only, so they are formed once per point, as drawPlane forms them
// (nni.cpp:186-200): the point's offset (dx, dy) from the work-package
// origin stays in double, zpx = (dx + halfwidth) / halfwidth and the slopes
// a = -2.0 * zpx / halfwidth are evaluated in double and rounded to float
// once each, and the offset is the float sum of the float squares (the time
// term is zero in 2-D).
struct CompatPlane {
    float a, b, zoff;
};

__device__ __forceinline__ CompatPlane compat_plane(float hw, double dx, double dy) {
    const double h = (double)hw;
    const float zpx = __double2float_rn(__ddiv_rn(__dadd_rn(dx, h), h));
    const float zpy = __double2float_rn(__ddiv_rn(__dadd_rn(dy, h), h));
    CompatPlane P;
    P.zoff = __fadd_rn(__fmul_rn(zpx, zpx), __fmul_rn(zpy, zpy));
    P.a = __double2float_rn(__ddiv_rn(__dmul_rn(-2.0, (double)zpx), h));
    P.b = __double2float_rn(__ddiv_rn(__dmul_rn(-2.0, (double)zpy), h));
    return P;
}

// The plane's depth at a pixel centre (px, py).
__device__ __forceinline__ float compat_depth(const CompatPlane& P, float hw, float px, float py) {
    const float zx = __fadd_rn(px, hw), zy = __fadd_rn(py, hw);
    return __fadd_rn(__fadd_rn(__fmul_rn(P.a, zx), __fmul_rn(P.b, zy)), P.zoff);
}

// Pixel index range [i0, i1] whose centres fall in [x0, x1) (one axis).
__device__ __forceinline__ void compat_span(float x0, float x1, double left, double ps, long long n, long long& i0,
                                            long long& i1) {
    i0 = (long long)ceil(__dsub_rn(__ddiv_rn(__dsub_rn((double)x0, left), ps), 0.5));
    i1 = (long long)ceil(__dsub_rn(__ddiv_rn(__dsub_rn((double)x1, left), ps), 0.5)) - 1;
    if (i0 < 0) i0 = 0;
    if (i1 > n - 1) i1 = n - 1;
}

__device__ __forceinline__ float compat_centre(long long p, double base, double ps) {
    return __double2float_rn(__dadd_rn(base, __dmul_rn((double)p + 0.5, ps)));
}

// Order-preserving map of a float's bits to an unsigned integer.
__device__ __forceinline__ uint32_t compat_order(float d) {
    const uint32_t u = __float_as_uint(d);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float compat_unorder(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

// A point's square of site influence: its offset from the work package
// (double, and rounded to float as drawPlane's px, py) and the pixels
// [i0,i1] x [j0,j1] whose centres the square covers (empty when i0 > i1 or
// j0 > j1).
struct CompatSquare {
    double dx, dy;
    float sx, sy;
    long long i0, i1, j0, j1;
};

__device__ __forceinline__ CompatSquare compat_square(const CompatGeom& G, const double* __restrict__ xyz, int64_t k) {
    CompatSquare q;
    q.dx = __dsub_rn(xyz[3 * k], (double)G.ox);
    q.dy = __dsub_rn(xyz[3 * k + 1], (double)G.oy);
    q.sx = __double2float_rn(q.dx);
    q.sy = __double2float_rn(q.dy);
    const float x0 = __double2float_rn(__dsub_rn((double)q.sx, G.rs)), x1 = __double2float_rn(__dadd_rn((double)q.sx, G.rs));
    const float y0 = __double2float_rn(__dsub_rn((double)q.sy, G.rs)), y1 = __double2float_rn(__dadd_rn((double)q.sy, G.rs));
    compat_span(x0, x1, G.left, G.pixel_size, G.xp, q.i0, q.i1);
    compat_span(y0, y1, G.bottom, G.pixel_size, G.yp, q.j0, q.j1);
    return q;
}

// The site pass runs per raster tile of kCpTile x kCpTile pixels whose keys
// sit in shared memory: the points are first listed per tile they reach
// (k_compat_count, k_compat_offsets, k_compat_fill), then one CTA per tile
// takes the minimum key of its points per pixel and writes the tile out once.
constexpr int kCpTile = 96;
constexpr size_t kCpTileSmem = sizeof(unsigned long long) * kCpTile * kCpTile;

__global__ void __launch_bounds__(256) k_compat_count(CompatGeom G, const double* __restrict__ xyz, int64_t n,
                                                      int ntx, int* __restrict__ tcnt) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const CompatSquare q = compat_square(G, xyz, k);
        if (q.i0 > q.i1 || q.j0 > q.j1) continue;
        for (long long ty = q.j0 / kCpTile; ty <= q.j1 / kCpTile; ++ty)
            for (long long tx = q.i0 / kCpTile; tx <= q.i1 / kCpTile; ++tx) atomicAdd(&tcnt[ty * ntx + tx], 1);
    }
}

// One CTA of 1024 threads: exclusive prefix of the nt tile counts into
// toff[0..nt] and zeroed fill cursors.
__global__ void __launch_bounds__(1024) k_compat_offsets(const int* __restrict__ tcnt, int nt, long long* __restrict__ toff,
                                                         int* __restrict__ tcur) {
    __shared__ long long wsum[32];
    const int per = (nt + 1023) / 1024;
    const int b0 = threadIdx.x * per;
    long long s = 0;
    for (int k = 0; k < per; ++k) if (b0 + k < nt) s += tcnt[b0 + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long x = s;
    for (int o = 1; o < 32; o <<= 1) { const long long y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        long long w = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) { const long long y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
        wsum[lane] = w;
    }
    __syncthreads();
    long long run = x - s + (warp ? wsum[warp - 1] : 0);
    for (int k = 0; k < per; ++k)
        if (b0 + k < nt) { toff[b0 + k] = run; run += tcnt[b0 + k]; tcur[b0 + k] = 0; }
    if (threadIdx.x == 1023) toff[nt] = run;
}

// (cap: the list's capacity, a bound on the squares' tile counts that the
// host derives from the site radius; entries past it are dropped, never written)
__global__ void __launch_bounds__(256) k_compat_fill(CompatGeom G, const double* __restrict__ xyz, int64_t n, int ntx,
                                                     const long long* __restrict__ toff, int* __restrict__ tcur,
                                                     uint32_t* __restrict__ list, int64_t cap) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const CompatSquare q = compat_square(G, xyz, k);
        if (q.i0 > q.i1 || q.j0 > q.j1) continue;
        for (long long ty = q.j0 / kCpTile; ty <= q.j1 / kCpTile; ++ty)
            for (long long tx = q.i0 / kCpTile; tx <= q.i1 / kCpTile; ++tx) {
                const long long t = ty * ntx + tx;
                const long long e = toff[t] + atomicAdd(&tcur[t], 1);
                if (e < cap) list[e] = (uint32_t)k;
            }
    }
}

// Site pass, one CTA per tile: every pixel keeps the smallest depth of the
// points whose squares cover it, the largest draw order k among equal depths
// (the depth test's later-draw-wins), as the 64-bit key order(d) << 32 | ~k;
// ~0 where no square reaches.
__global__ void __launch_bounds__(256) k_compat_sites(CompatGeom G, const double* __restrict__ xyz, int ntx,
                                                      const long long* __restrict__ toff,
                                                      const uint32_t* __restrict__ list, int64_t cap,
                                                      unsigned long long* __restrict__ key) {
    extern __shared__ unsigned long long sk[];
    const int t = blockIdx.x;
    const long long px0 = (long long)(t % ntx) * kCpTile, py0 = (long long)(t / ntx) * kCpTile;
    const int pw = (int)min((long long)kCpTile, (long long)G.xp - px0);
    const int ph = (int)min((long long)kCpTile, (long long)G.yp - py0);
    for (int e = threadIdx.x; e < kCpTile * kCpTile; e += blockDim.x) sk[e] = ~0ull;
    __syncthreads();
    const long long e1 = toff[t + 1] < cap ? toff[t + 1] : (long long)cap;
    for (long long e = toff[t] + threadIdx.x; e < e1; e += blockDim.x) {
        const int64_t k = list[e];
        const CompatSquare q = compat_square(G, xyz, k);
        const long long i0 = max(q.i0, px0), i1 = min(q.i1, px0 + pw - 1);
        const long long j0 = max(q.j0, py0), j1 = min(q.j1, py0 + ph - 1);
        const unsigned long long low = 0xFFFFFFFFull - (unsigned long long)k;
        const CompatPlane P = compat_plane(G.hw, q.dx, q.dy);
        for (long long pj = j0; pj <= j1; ++pj) {
            const float cy = compat_centre(pj, G.bottom, G.pixel_size);
            for (long long pi = i0; pi <= i1; ++pi) {
                const float cx = compat_centre(pi, G.left, G.pixel_size);
                const float d = compat_depth(P, G.hw, cx, cy);
                atomicMin(&sk[(pj - py0) * kCpTile + (pi - px0)], ((unsigned long long)compat_order(d) << 32) | low);
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kCpTile * kCpTile; e += blockDim.x) {
        const int r = e / kCpTile, c = e - r * kCpTile;
        if (r < ph && c < pw) key[(py0 + r) * G.xp + px0 + c] = sk[e];
    }
}

// z-code of a point: floor((z + zOffset + 1) * zMult) (nni.cpp:538-549).
__device__ __forceinline__ uint32_t compat_zcode(double z, int z_offset, int z_mult) {
    return (uint32_t)(long long)floor(__dmul_rn(__dadd_rn(__dadd_rn(z, (double)z_offset), 1.0), (double)z_mult));
}

// Query pass and divide: one thread per cell, over the pixels of its square;
// a pixel counts when it holds a site with a non-zero z-code and the cell's
// own plane is no deeper there (cuda_nni.cu:423-448).
__global__ void __launch_bounds__(256) k_compat_cells(CompatGeom G, const double* __restrict__ xyz,
                                                      const unsigned long long* __restrict__ key,
                                                      float* __restrict__ h, int32_t* __restrict__ res) {
    const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (w >= (int64_t)G.ncols * G.nrows) return;
    const int i = (int)(w % G.ncols), j = (int)(w / G.ncols);
    const double qdx = __dmul_rn((double)i, G.qspacing), qdy = __dmul_rn((double)j, G.qspacing);
    const float qx = __double2float_rn(qdx);
    const float qy = __double2float_rn(qdy);
    const float x0 = __double2float_rn(__dsub_rn((double)qx, G.rq)), x1 = __double2float_rn(__dadd_rn((double)qx, G.rq));
    const float y0 = __double2float_rn(__dsub_rn((double)qy, G.rq)), y1 = __double2float_rn(__dadd_rn((double)qy, G.rq));
    long long i0, i1, j0, j1;
    compat_span(x0, x1, G.left, G.pixel_size, G.xp, i0, i1);
    compat_span(y0, y1, G.bottom, G.pixel_size, G.yp, j0, j1);
    uint32_t numer = 0;
    int32_t denom = 0;
    const CompatPlane Q = compat_plane(G.hw, qdx, qdy);
    for (long long pj = j0; pj <= j1; ++pj) {
        const float cy = compat_centre(pj, G.bottom, G.pixel_size);
        for (long long pi = i0; pi <= i1; ++pi) {
            const unsigned long long kk = key[pj * G.xp + pi];
            if (kk == ~0ull) continue;                        // no site drew here
            const int64_t k = (int64_t)(0xFFFFFFFFull - (kk & 0xFFFFFFFFull));
            const uint32_t zc = compat_zcode(xyz[3 * k + 2], G.z_offset, G.z_mult);
            if (zc == 0) continue;
            const float cx = compat_centre(pi, G.left, G.pixel_size);
            const float d = compat_depth(Q, G.hw, cx, cy);
            if (d <= compat_unorder((uint32_t)(kk >> 32))) {
                numer += zc;                                  // int32 sum with wrap, as the atomicAdd
                denom += 1;
            }
        }
    }
    const int32_t r = denom == 0 ? -9999 * G.z_mult : (int32_t)numer / denom;
    if (res) res[w] = r;
    double z = __ddiv_rn((double)r, (double)G.z_mult);
    if (z != -9999.0) z = __dsub_rn(__dsub_rn(z, (double)G.z_offset), 1.0);
    h[w] = __double2float_rn(z);
}

}  // namespace dnni

// Both entry points: host buffers (device = false: points copied in,
// heights and quotients copied out, the call waits) or device buffers
// (queued on st; the call returns with the work queued).
static dnni_status compat_run(dnni_ctx* c, const dnni_compat_settings* s, const dnni_compat_wp* wp, const double* xyz,
                              int64_t n, float* h_out, int32_t* res_out, bool device, cudaStream_t st) {
    if (s->scale <= 0 || !(s->cell_size > 0) || wp->nrows <= 0 || wp->ncols <= 0 || s->multiplier <= 0)
        return set_err(c, DNNI_E_INVAL, "scale, cell size, grid sides and multiplier must be positive");
    if ((uint64_t)n >= 0xFFFFFFFFull) return set_err(c, DNNI_E_INVAL, "too many points for 32-bit draw order");
    // geometry as nni::performNNI derives it (nni.cpp:879-886, 186-189)
    CompatGeom G;
    G.qspacing = s->cell_size;
    G.pixel_size = G.qspacing / s->scale;
    const float qr = (float)s->query_radius;
    const int pixel_offset = (int)std::ceil((qr - std::floor(s->scale / 2.0) * G.pixel_size) / G.pixel_size) + 1;
    const long long xp = (long long)wp->ncols * s->scale + 2LL * pixel_offset;
    const long long yp = (long long)wp->nrows * s->scale + 2LL * pixel_offset;
    if (xp <= 0 || yp <= 0 || xp > 65535 || yp > 65535 || xp * yp > (1LL << 31))
        return set_err(c, DNNI_E_INVAL, "raster of the work package too large");
    G.xp = (int32_t)xp;
    G.yp = (int32_t)yp;
    G.left = 0 - (G.qspacing / 2.0) - (pixel_offset * G.pixel_size);
    G.bottom = G.left;
    G.hw = (float)(((wp->nrows - 1) * G.qspacing) / 2.0);
    G.rs = s->site_radius / std::sqrt(2.0);
    G.rq = qr / std::sqrt(2.0);
    G.ncols = wp->ncols;
    G.nrows = wp->nrows;
    G.z_offset = -1 * s->point_min;
    G.z_mult = s->multiplier;
    G.ox = wp->origin_x;
    G.oy = wp->origin_y;
    const int64_t cells = (int64_t)wp->ncols * wp->nrows;
    const int ntx = (int)((xp + kCpTile - 1) / kCpTile), nty = (int)((yp + kCpTile - 1) / kCpTile);
    const int nt = ntx * nty;
    // tiles one square can reach: its pixel span is at most 2 rs / ps + 1
    // (plus rounding) wide
    const long long span = (long long)std::ceil(2.0 * G.rs / G.pixel_size) + 3;
    const long long per = (span / kCpTile + 2) * (span / kCpTile + 2);
    const int64_t list_n = std::max<int64_t>(n * per, 1);
    dnni_status rs;
    // scratch: the pixel keys in the context's span-word buffer, the tile
    // counts, offsets and cursors in its bin-count buffer, the per-tile point
    // lists in its rank buffer; points and outputs in its staging buffers
    const size_t tbytes = sizeof(long long) * (size_t)(nt + 1) + 2 * sizeof(int) * (size_t)nt;
    if ((rs = dnni_ensure(c, c->scr.D, sizeof(unsigned long long) * (size_t)(xp * yp))) ||
        (rs = dnni_ensure(c, c->scr.cnt, tbytes)) ||
        (rs = dnni_ensure(c, c->scr.list, sizeof(uint32_t) * (size_t)list_n)) ||
        (!device && ((rs = dnni_ensure(c, c->in_xyz, sizeof(double) * 3 * (size_t)std::max<int64_t>(n, 1))) ||
                     (rs = dnni_ensure(c, c->out_h, sizeof(float) * (size_t)cells)) ||
                     (res_out && (rs = dnni_ensure(c, c->out_site, sizeof(int32_t) * (size_t)cells))))))
        return rs;
    const double* dxyz = device ? xyz : (const double*)c->in_xyz.p;
    float* dh = device ? h_out : (float*)c->out_h.p;
    int32_t* dres = res_out ? (device ? res_out : (int32_t*)c->out_site.p) : nullptr;
    unsigned long long* key = (unsigned long long*)c->scr.D.p;
    long long* toff = (long long*)c->scr.cnt.p;
    int* tcnt = (int*)(toff + nt + 1);
    int* tcur = tcnt + nt;
    CK(cudaMemsetAsync(tcnt, 0, sizeof(int) * (size_t)nt, st));
    if (n > 0) {
        if (!device) CK(cudaMemcpyAsync(c->in_xyz.p, xyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, st));
        k_compat_count<<<c->sm_count * 8, 256, 0, st>>>(G, dxyz, n, ntx, tcnt);
    }
    k_compat_offsets<<<1, 1024, 0, st>>>(tcnt, nt, toff, tcur);
    if (n > 0)
        k_compat_fill<<<c->sm_count * 8, 256, 0, st>>>(G, dxyz, n, ntx, toff, tcur, (uint32_t*)c->scr.list.p, list_n);
    CK(cudaFuncSetAttribute(k_compat_sites, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCpTileSmem));
    k_compat_sites<<<nt, 256, kCpTileSmem, st>>>(G, dxyz, ntx, toff, (const uint32_t*)c->scr.list.p, list_n, key);
    k_compat_cells<<<(int)((cells + 255) / 256), 256, 0, st>>>(G, dxyz, key, dh, dres);
    CK(cudaGetLastError());
    if (!device) {
        CK(cudaMemcpyAsync(h_out, c->out_h.p, sizeof(float) * (size_t)cells, cudaMemcpyDeviceToHost, st));
        if (res_out)
            CK(cudaMemcpyAsync(res_out, c->out_site.p, sizeof(int32_t) * (size_t)cells, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return DNNI_OK;
}

extern "C" dnni_status dnni_interpolate_compat(dnni_ctx* c, const dnni_compat_settings* s, const dnni_compat_wp* wp,
                                               const double* xyz, int64_t n, float* h_out, int32_t* res_out) {
    if (!c || !s || !wp || !h_out || n < 0 || (n > 0 && !xyz)) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    return compat_run(c, s, wp, xyz, n, h_out, res_out, false, c->stream);
}

extern "C" dnni_status dnni_interpolate_compat_device(dnni_ctx* c, const dnni_compat_settings* s,
                                                      const dnni_compat_wp* wp, const double* d_xyz, int64_t n,
                                                      float* d_h, int32_t* d_res, void* stream) {
    if (!c || !s || !wp || !d_h || n < 0 || (n > 0 && !d_xyz)) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    return compat_run(c, s, wp, d_xyz, n, d_h, d_res, true, stream ? (cudaStream_t)stream : c->stream);
}
