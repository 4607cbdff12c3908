// dnni_segment.cuh -- the segment driver: one large grid interpolated as
// tiles with halos (dnni_segment_run).  Included by dnni_engine.cu, whose
// scratch, planning and launch helpers it uses.
//
// Replaces the reference's out-of-core pipeline around performNNI for one
// grid: TPIE binning of the points into work packages with duplicated borders
// (terranni.cpp:203-368, border copies terranni.cpp:271-302), the loop over
// work packages (binRun, terranni.cpp:394-426) and the grid assembly
// (terranni.cpp:430-488).  Here the points go to HBM once and are bucketed
// there (buckets of 256 x 256 cells, row-major, so one row of buckets is one
// contiguous range of the bucketed points); each tile gathers the buckets of
// its point box into a staging area and a batch of tiles runs through the
// ordinary launch sequence.
#pragma once

namespace dnni {

constexpr int kSegBucketCells = 256;        // bucket side in cells
constexpr int kSegGatherChunk = 1 << 16;    // points per gather block

struct SegGrid {
    long long ox, oy;   // LAS origin of cell (0,0)
    long long w;        // bucket side in LAS units
    int nbx, nby;
};

// Bucket of a point; points beyond the grid fall into the edge buckets.
__device__ __forceinline__ int seg_bucket(const SegGrid& g, int x, int y) {
    const long long rx = (long long)x - g.ox, ry = (long long)y - g.oy;
    long long bx = rx >= 0 ? rx / g.w : 0, by = ry >= 0 ? ry / g.w : 0;
    bx = bx < g.nbx - 1 ? bx : g.nbx - 1;
    by = by < g.nby - 1 ? by : g.nby - 1;
    return (int)(by * g.nbx + bx);
}

__global__ void __launch_bounds__(256) k_seg_count(SegGrid g, const int32_t* __restrict__ xyz, int64_t n,
                                                   unsigned* __restrict__ cnt) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[seg_bucket(g, xyz[3 * i], xyz[3 * i + 1])], 1u);
}

// Bucketing by partition in two passes, each staged in shared memory: a CTA
// takes kSegPart points, counts them per key, places them in key order in
// shared memory, reserves one range per key with a global cursor and writes
// each key's points as one contiguous run (the input order is random in
// space, so writing point by point would scatter every store).  Pass 1 keys
// by group of rstep bucket rows into `part` ({x, y, z, input index}); pass 2,
// over part, keys by bucket within the rows a CTA's points span (point by
// point with global cursors when they span more than kSegKeys buckets).  The
// order of points inside a bucket is free: the input index travels with
// each point.
constexpr int kSegPart = 2048;              // points per CTA
constexpr int kSegPer = kSegPart / 256;     // per thread
constexpr int kSegKeys = 2048;              // most keys one pass-2 CTA stages
constexpr int kSegRowKeys = 4096;           // most row groups of pass 1

__device__ __forceinline__ int seg_row(const SegGrid& g, int x, int y) { return seg_bucket(g, x, y) / g.nbx; }

// Exclusive prefix of cnt[0..nk) into off[] by 256 threads (each sums a run
// of consecutive keys); reserves each non-empty key's range from cur[key0 +
// k] into base[k].
__device__ __forceinline__ void seg_part_offsets(const int* cnt, int* off, unsigned long long* base, int nk,
                                                 unsigned long long* __restrict__ cur, long long key0) {
    __shared__ int wsum[8];
    const int per = (nk + 255) / 256, k0 = threadIdx.x * per;
    int s = 0;
    for (int k = k0; k < k0 + per && k < nk; ++k) s += cnt[k];
    int total;
    int run = block_exclusive_sum(s, wsum, total, (int)threadIdx.x);
    for (int k = k0; k < k0 + per && k < nk; ++k) {
        off[k] = run;
        run += cnt[k];
        base[k] = cnt[k] ? atomicAdd(&cur[key0 + k], (unsigned long long)cnt[k]) : 0ull;
    }
}

__global__ void __launch_bounds__(256) k_seg_part_rows(SegGrid g, int rstep, int ngrp,
                                                       const int32_t* __restrict__ xyz, int64_t n,
                                                       unsigned long long* __restrict__ rowcur,
                                                       int4* __restrict__ part) {
    extern __shared__ int4 stage[];                        // kSegPart points, then the per-group tables
    unsigned long long* base = (unsigned long long*)(stage + kSegPart);
    int* cnt = (int*)(base + ngrp);
    int* off = cnt + ngrp;
    const int64_t c0 = (int64_t)blockIdx.x * kSegPart;
    const int m = (int)(n - c0 < kSegPart ? n - c0 : kSegPart);
    for (int r = threadIdx.x; r < ngrp; r += blockDim.x) cnt[r] = 0;
    __syncthreads();
    int4 p[kSegPer];
    int key[kSegPer], lr[kSegPer];
#pragma unroll
    for (int k = 0; k < kSegPer; ++k) {
        const int j = k * 256 + threadIdx.x;
        if (j < m) {
            const int64_t i = c0 + j;
            p[k] = make_int4(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], (int)i);
            key[k] = seg_row(g, p[k].x, p[k].y) / rstep;
            lr[k] = atomicAdd(&cnt[key[k]], 1);
        }
    }
    __syncthreads();
    seg_part_offsets(cnt, off, base, ngrp, rowcur, 0);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSegPer; ++k)
        if (k * 256 + (int)threadIdx.x < m) stage[off[key[k]] + lr[k]] = p[k];
    __syncthreads();
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
        const int4 q = stage[j];
        const int r = seg_row(g, q.x, q.y) / rstep;
        part[base[r] + (unsigned long long)(j - off[r])] = q;
    }
}

__global__ void __launch_bounds__(256) k_seg_part_buckets(SegGrid g, const int4* __restrict__ part, int64_t n,
                                                          unsigned long long* __restrict__ bcur,
                                                          int32_t* __restrict__ oxyz, uint32_t* __restrict__ ogid) {
    extern __shared__ int4 stage[];                        // kSegPart points, then the per-bucket tables
    unsigned long long* base = (unsigned long long*)(stage + kSegPart);
    int* cnt = (int*)(base + kSegKeys);
    int* off = cnt + kSegKeys;
    const int64_t c0 = (int64_t)blockIdx.x * kSegPart;
    const int m = (int)(n - c0 < kSegPart ? n - c0 : kSegPart);
    // the rows r0 .. r1 that the CTA's points span
    __shared__ int rmin, rmax;
    if (threadIdx.x == 0) {
        rmin = INT_MAX;
        rmax = INT_MIN;
    }
    __syncthreads();
    {
        int lo = INT_MAX, hi = INT_MIN;
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const int4 q = part[c0 + j];
            const int r = seg_row(g, q.x, q.y);
            lo = r < lo ? r : lo;
            hi = r > hi ? r : hi;
        }
        atomicMin(&rmin, lo);
        atomicMax(&rmax, hi);
    }
    __syncthreads();
    const int r0 = rmin, r1 = rmax;
    const long long key0 = (long long)r0 * g.nbx;
    const long long nk = (long long)(r1 - r0 + 1) * g.nbx;
    if (nk > kSegKeys) {
        // sparse rows: too many buckets to stage, place point by point
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const int4 q = part[c0 + j];
            const unsigned long long pos = atomicAdd(&bcur[seg_bucket(g, q.x, q.y)], 1ull);
            oxyz[3 * pos] = q.x;
            oxyz[3 * pos + 1] = q.y;
            oxyz[3 * pos + 2] = q.z;
            ogid[pos] = (uint32_t)q.w;
        }
        return;
    }
    for (int k = threadIdx.x; k < (int)nk; k += blockDim.x) cnt[k] = 0;
    __syncthreads();
    int4 p[kSegPer];
    int key[kSegPer], lr[kSegPer];
#pragma unroll
    for (int k = 0; k < kSegPer; ++k) {
        const int j = k * 256 + threadIdx.x;
        if (j < m) {
            p[k] = part[c0 + j];
            key[k] = (int)(seg_bucket(g, p[k].x, p[k].y) - key0);
            lr[k] = atomicAdd(&cnt[key[k]], 1);
        }
    }
    __syncthreads();
    seg_part_offsets(cnt, off, base, (int)nk, bcur, key0);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSegPer; ++k)
        if (k * 256 + (int)threadIdx.x < m) stage[off[key[k]] + lr[k]] = p[k];
    __syncthreads();
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
        const int4 q = stage[j];
        const int b = (int)(seg_bucket(g, q.x, q.y) - key0);
        const unsigned long long pos = base[b] + (unsigned long long)(j - off[b]);
        oxyz[3 * pos] = q.x;
        oxyz[3 * pos + 1] = q.y;
        oxyz[3 * pos + 2] = q.z;
        ogid[pos] = (uint32_t)q.w;
    }
}

// One block per bucket: bounding box {minx, miny, maxx, maxy} of its points
// (INT_MAX, INT_MAX, INT_MIN, INT_MIN when empty).
__global__ void __launch_bounds__(256) k_seg_bbox(const int32_t* __restrict__ sxyz, const long long* __restrict__ start,
                                                  int4* __restrict__ bbox) {
    __shared__ int red[4][8];
    const long long s0 = start[blockIdx.x], s1 = start[blockIdx.x + 1];
    int mnx = INT_MAX, mny = INT_MAX, mxx = INT_MIN, mxy = INT_MIN;
    for (long long i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
        const int x = sxyz[3 * i], y = sxyz[3 * i + 1];
        mnx = min(mnx, x); mxx = max(mxx, x);
        mny = min(mny, y); mxy = max(mxy, y);
    }
    mnx = __reduce_min_sync(0xffffffffu, mnx); mny = __reduce_min_sync(0xffffffffu, mny);
    mxx = __reduce_max_sync(0xffffffffu, mxx); mxy = __reduce_max_sync(0xffffffffu, mxy);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = mnx; red[1][w] = mny; red[2][w] = mxx; red[3][w] = mxy; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int4 b = make_int4(INT_MAX, INT_MAX, INT_MIN, INT_MIN);
        for (int k = 0; k < 8; ++k) {
            b.x = min(b.x, red[0][k]); b.y = min(b.y, red[1][k]);
            b.z = max(b.z, red[2][k]); b.w = max(b.w, red[3][k]);
        }
        bbox[blockIdx.x] = b;
    }
}

// Occupancy of the fine blocks (fw LAS units square) that partition the
// grid; points beyond the grid are left out.
__global__ void __launch_bounds__(256) k_seg_occ(SegGrid g, long long fw, int nfx, int nfy,
                                                 const int32_t* __restrict__ xyz, int64_t n,
                                                 unsigned char* __restrict__ occ) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const long long rx = (long long)xyz[3 * i] - g.ox, ry = (long long)xyz[3 * i + 1] - g.oy;
        if (rx < 0 || ry < 0) continue;
        const long long fx = rx / fw, fy = ry / fw;
        if (fx < nfx && fy < nfy) occ[fy * nfx + fx] = 1;
    }
}

// Bounding box {minx, miny, maxx, maxy} of n points (ext pre-set to empty).
__global__ void __launch_bounds__(256) k_seg_extent(const int32_t* __restrict__ xyz, int64_t n, int* __restrict__ ext) {
    int mnx = INT_MAX, mny = INT_MAX, mxx = INT_MIN, mxy = INT_MIN;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = xyz[3 * i], y = xyz[3 * i + 1];
        mnx = min(mnx, x); mxx = max(mxx, x);
        mny = min(mny, y); mxy = max(mxy, y);
    }
    mnx = __reduce_min_sync(0xffffffffu, mnx); mny = __reduce_min_sync(0xffffffffu, mny);
    mxx = __reduce_max_sync(0xffffffffu, mxx); mxy = __reduce_max_sync(0xffffffffu, mxy);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&ext[0], mnx); atomicMin(&ext[1], mny);
        atomicMax(&ext[2], mxx); atomicMax(&ext[3], mxy);
    }
}

// Per tile of a batch, the largest R2 over the two outermost pixel columns
// or rows on each side of its raster: rm[4t + 0..3] = left, right, bottom,
// top (-1 without sites).
__global__ void __launch_bounds__(256) k_ring_max(BatchTables bt, const int2* __restrict__ pix, int* __restrict__ rm) {
    __shared__ int red[4][8];
    const TileParams& T = bt.tiles[blockIdx.x];
    const int2* P = pix + T.pix_off;
    int m[4] = {-1, -1, -1, -1};
    for (int k = threadIdx.x; k < 2 * T.rh; k += blockDim.x) {
        const int j = k >> 1, c = min(k & 1, T.rw - 1);
        m[0] = max(m[0], P[(int64_t)j * T.rw + c].y);
        m[1] = max(m[1], P[(int64_t)j * T.rw + (T.rw - 1 - c)].y);
    }
    for (int k = threadIdx.x; k < 2 * T.rw; k += blockDim.x) {
        const int i = k >> 1, r = min(k & 1, T.rh - 1);
        m[2] = max(m[2], P[(int64_t)r * T.rw + i].y);
        m[3] = max(m[3], P[(int64_t)(T.rh - 1 - r) * T.rw + i].y);
    }
    for (int s = 0; s < 4; ++s) {
        const int v = __reduce_max_sync(0xffffffffu, m[s]);
        if ((threadIdx.x & 31) == 0) red[s][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        int v = -1;
        for (int w = 0; w < 8; ++w) v = max(v, red[threadIdx.x][w]);
        rm[4 * blockIdx.x + threadIdx.x] = v;
    }
}

// Gather of bucket ranges into a tile's staging rows: one block per chunk.
struct SegChunk {
    long long src, dst;
    int count, pad;
};

__global__ void __launch_bounds__(256) k_seg_gather(const SegChunk* __restrict__ ch, const int32_t* __restrict__ sxyz,
                                                    const uint32_t* __restrict__ sgid, int32_t* __restrict__ dxyz,
                                                    uint32_t* __restrict__ dgid) {
    const SegChunk c = ch[blockIdx.x];
    const int32_t* s = sxyz + 3 * c.src;
    int32_t* d = dxyz + 3 * c.dst;
    for (int k = threadIdx.x; k < 3 * c.count; k += blockDim.x) d[k] = s[k];
    for (int k = threadIdx.x; k < c.count; k += blockDim.x) dgid[c.dst + k] = sgid[c.src + k];
}

}  // namespace dnni

namespace {

struct SegTile {
    int x0, y0, x1, y1;   // core cells [x0,x1) x [y0,y1)
    int h[4];             // raster halo (cells) on the left, right, bottom, top
    int hp;               // point halo: the point box is the raster +- hp
};

long long floor_div_ll(long long a, long long b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Uploads n points (chunks of 64 Mi) and buckets them on the device by G:
// afterwards B.sxyz / B.sgid hold the points in bucket order (gid = input
// index), start / bbox the bucket ranges and bounding boxes; B.xin and
// B.part are released again.
dnni_status upload_points(dnni_ctx* c, cudaStream_t st, const int32_t* h_xyz, int64_t n, SegBufs& B) {
    dnni_status rs;
    if ((rs = dnni_ensure(c, B.xin, 12 * (size_t)std::max<int64_t>(n, 1)))) return rs;
    CK(cudaEventRecord(c->ev[0], st));
    const int64_t kUp = 64ll << 20;
    for (int64_t o = 0; o < n; o += kUp) {
        const int64_t m = std::min(kUp, n - o);
        CK(cudaMemcpyAsync((int32_t*)B.xin.p + 3 * o, h_xyz + 3 * o, 12 * (size_t)m, cudaMemcpyHostToDevice, st));
    }
    CK(cudaEventRecord(c->ev[1], st));
    return DNNI_OK;
}

// Buckets the n points already uploaded to B.xin (see bucket_points);
// keep_staging leaves B.xin and B.part allocated for the next call.
dnni_status bucket_uploaded(dnni_ctx* c, cudaStream_t st, const SegGrid& G, int64_t n, SegBufs& B,
                            std::vector<long long>& start, std::vector<int4>& bbox, float* ms_up, float* ms_bk,
                            bool keep_staging = false) {
    const int nb = G.nbx * G.nby;
    dnni_status rs;
    const size_t npts = (size_t)std::max<int64_t>(n, 1);
    if ((rs = dnni_ensure(c, B.sxyz, 12 * npts)) || (rs = dnni_ensure(c, B.sgid, 4 * npts)) ||
        (rs = dnni_ensure(c, B.part, 16 * npts)) || (rs = dnni_ensure(c, B.cnt, 4 * (size_t)nb)) ||
        (rs = dnni_ensure(c, B.cur, 8 * (size_t)nb)) || (rs = dnni_ensure(c, B.start, 8 * (size_t)(nb + 1))) ||
        (rs = dnni_ensure(c, B.bbox, 16 * (size_t)nb)))
        return rs;
    CK(cudaMemsetAsync(B.cnt.p, 0, 4 * (size_t)nb, st));
    const int grid = c->sm_count * 8;
    if (n > 0) k_seg_count<<<grid, 256, 0, st>>>(G, (const int32_t*)B.xin.p, n, (unsigned*)B.cnt.p);
    std::vector<unsigned> cnt(nb);
    start.assign(nb + 1, 0);
    CK(cudaMemcpyAsync(cnt.data(), B.cnt.p, 4 * (size_t)nb, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int b = 0; b < nb; ++b) start[b + 1] = start[b] + cnt[b];
    CK(cudaMemcpyAsync(B.start.p, start.data(), 8 * (size_t)(nb + 1), cudaMemcpyHostToDevice, st));
    if (n > 0) {
        // pass 1 by bucket row (cursors: the rows' first positions), pass 2
        // by bucket (cursors: the buckets' first positions)
        const int rstep = (G.nby + kSegRowKeys - 1) / kSegRowKeys;
        const int ngrp = (G.nby + rstep - 1) / rstep;
        std::vector<long long> rowcur(ngrp);
        for (int r = 0; r < ngrp; ++r) rowcur[r] = start[(size_t)r * rstep * G.nbx];
        CK(cudaMemcpyAsync(B.cur.p, rowcur.data(), 8 * (size_t)ngrp, cudaMemcpyHostToDevice, st));
        const int nblk = (int)((n + kSegPart - 1) / kSegPart);
        const size_t sm1 = sizeof(int4) * kSegPart + 16 * (size_t)ngrp;
        const size_t sm2 = sizeof(int4) * kSegPart + 16 * (size_t)kSegKeys;
        CK(cudaFuncSetAttribute(k_seg_part_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
        CK(cudaFuncSetAttribute(k_seg_part_buckets, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
        k_seg_part_rows<<<nblk, 256, sm1, st>>>(G, rstep, ngrp, (const int32_t*)B.xin.p, n,
                                                (unsigned long long*)B.cur.p, (int4*)B.part.p);
        CK(cudaMemcpyAsync(B.cur.p, B.start.p, 8 * (size_t)nb, cudaMemcpyDeviceToDevice, st));
        k_seg_part_buckets<<<nblk, 256, sm2, st>>>(G, (const int4*)B.part.p, n, (unsigned long long*)B.cur.p,
                                                   (int32_t*)B.sxyz.p, (uint32_t*)B.sgid.p);
    }
    k_seg_bbox<<<nb, 256, 0, st>>>((const int32_t*)B.sxyz.p, (const long long*)B.start.p, (int4*)B.bbox.p);
    bbox.resize(nb);
    CK(cudaMemcpyAsync(bbox.data(), B.bbox.p, 16 * (size_t)nb, cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(c->ev[2], st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    cudaEventElapsedTime(ms_up, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(ms_bk, c->ev[1], c->ev[2]);
    if (!keep_staging) {
        dnni_release(B.xin, c);
        dnni_release(B.part, c);
    }
    return DNNI_OK;
}

dnni_status bucket_points(dnni_ctx* c, cudaStream_t st, const SegGrid& G, const int32_t* h_xyz, int64_t n, SegBufs& B,
                          std::vector<long long>& start, std::vector<int4>& bbox, float* ms_up, float* ms_bk,
                          bool keep_staging = false) {
    dnni_status rs = upload_points(c, st, h_xyz, n, B);
    if (rs) return rs;
    return bucket_uploaded(c, st, G, n, B, start, bbox, ms_up, ms_bk, keep_staging);
}

// Squared distance, in fine blocks (fw LAS units square, nfx x nfy from the
// grid origin), from every fine block to the nearest one holding a point.
dnni_status occupancy_edt(dnni_ctx* c, cudaStream_t st, const SegGrid& G, long long fw, int nfx, int nfy,
                          SegBufs& B, int64_t n, std::vector<double>& edt2) {
    DevBuf& occ_d = B.occ;                   // kept between calls: no allocation, no implicit synchronisation
    dnni_status rs;
    if ((rs = dnni_ensure(c, occ_d, (size_t)nfx * nfy))) return rs;
    std::vector<unsigned char> occ((size_t)nfx * nfy);
    cudaError_t e = cudaMemsetAsync(occ_d.p, 0, occ.size(), st);
    if (e == cudaSuccess && n > 0)
        k_seg_occ<<<c->sm_count * 8, 256, 0, st>>>(G, fw, nfx, nfy, (const int32_t*)B.sxyz.p, n,
                                                   (unsigned char*)occ_d.p);
    if (e == cudaSuccess) e = cudaMemcpyAsync(occ.data(), occ_d.p, occ.size(), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_err(c, e, "occupancy");
    edt2 = edt_2d(occ.data(), nfx, nfy);
    return DNNI_OK;
}

dnni_status segment_run(dnni_ctx* c, const dnni_segment& s, const int32_t* h_xyz, int64_t n, float* h_out,
                        uint32_t* h_site, dnni_segment_stats* stats, SegBufs& B, Scratch& scr) {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    cudaStream_t st = c->stream;
    const int nbx = (s.ncols + kSegBucketCells - 1) / kSegBucketCells;
    const int nby = (s.nrows + kSegBucketCells - 1) / kSegBucketCells;
    const SegGrid G{s.origin_x, s.origin_y, (long long)kSegBucketCells * s.cell_size, nbx, nby};
    dnni_status rs;
    std::vector<long long> start;
    std::vector<int4> bbox;
    float ms_up = 0, ms_bk = 0;
    if ((rs = bucket_points(c, st, G, h_xyz, n, B, start, bbox, &ms_up, &ms_bk, true))) return rs;

    // 3. first halo of each tile: unless the caller fixed it, an upper bound
    // of the nearest-site distance from the occupancy of fine blocks (fb
    // cells square, at most 4096 per side): a pixel in block b has a site
    // within fb * (sqrt(edt2(b)) + sqrt(2)) cells, and a halo of that + 3 over
    // the whole raster passes the exactness check below.
    const auto t_bound = clk::now();
    const int fb = std::max(16, (std::max(s.ncols, s.nrows) + 4095) / 4096);
    const int nfx = (s.ncols + fb - 1) / fb, nfy = (s.nrows + fb - 1) / fb;
    std::vector<double> edt2;
    if (s.halo == 0 && (rs = occupancy_edt(c, st, G, (long long)fb * s.cell_size, nfx, nfy, B, n, edt2))) return rs;
    const int hmax = std::max(s.ncols, s.nrows) + 4;
    auto bound_halo = [&](int x0, int y0, int x1, int y1) {   // cells [x0,x1) x [y0,y1), clipped
        double m = 0;
        for (int fy = y0 / fb; fy <= (y1 - 1) / fb; ++fy)
            for (int fx = x0 / fb; fx <= (x1 - 1) / fb; ++fx) m = std::max(m, edt2[(size_t)fy * nfx + fx]);
        if (m >= kEdtFar / 2) return hmax;
        return std::min(hmax, (int)std::ceil(fb * (std::sqrt(m) + 1.4143)) + 3);
    };
    // Halos per side: a pixel outside the raster whose disc reaches a core
    // cell forces, on the side where the segment to that cell leaves the
    // raster, a pixel among the two outermost columns (rows) with distance
    // to its nearest site >= halo - 1.21 (see the check below); so each
    // side's halo need only exceed the bound over its own two outer lines,
    // while the point halo must exceed the bound over the whole raster.
    auto raster_of = [&](const SegTile& T, int& ax0, int& ay0, int& ax1, int& ay1) {
        ax0 = std::max(0, T.x0 - T.h[0]);
        ax1 = std::min(s.ncols, T.x1 + T.h[1]);
        ay0 = std::max(0, T.y0 - T.h[2]);
        ay1 = std::min(s.nrows, T.y1 + T.h[3]);
    };
    // the grid's tiles in row-major order, each with a cost (its cells and the
    // points of the buckets its core touches); a call with parts > 1 runs
    // the contiguous, cost-balanced range of tiles of its part
    std::vector<SegTile> cores;
    std::vector<int64_t> cost;
    for (int y = 0; y < s.nrows; y += s.tile)
        for (int x = 0; x < s.ncols; x += s.tile) {
            const SegTile T{x, y, std::min(x + s.tile, s.ncols), std::min(y + s.tile, s.nrows),
                            {s.halo, s.halo, s.halo, s.halo}, s.halo};
            const int cbx0 = T.x0 / kSegBucketCells, cbx1 = (T.x1 - 1) / kSegBucketCells;
            int64_t pts = 0;
            for (int by = T.y0 / kSegBucketCells; by <= (T.y1 - 1) / kSegBucketCells; ++by)
                pts += start[(size_t)by * nbx + cbx1 + 1] - start[(size_t)by * nbx + cbx0];
            cores.push_back(T);
            cost.push_back((int64_t)(T.x1 - T.x0) * (T.y1 - T.y0) + pts);
        }
    int k0 = 0, k1 = (int)cores.size();
    if (s.parts > 1) {
        std::vector<int32_t> first((size_t)s.parts + 1);
        if ((rs = dnni_partition_contiguous(cost.data(), (int32_t)cost.size(), s.parts, first.data())))
            return set_err(c, rs, "tile partition");
        k0 = first[s.part];
        k1 = first[s.part + 1];
    }
    std::vector<SegTile> queue;
    for (int kq = k0; kq < k1; ++kq) {
        SegTile T = cores[kq];
        if (s.halo == 0) {
            for (int k = 0; k < 4; ++k) T.h[k] = 2;
            for (int it = 0; it < 32; ++it) {
                int ax0, ay0, ax1, ay1;
                raster_of(T, ax0, ay0, ax1, ay1);
                const int hs[4] = {bound_halo(ax0, ay0, std::min(ax0 + 2, ax1), ay1),
                                   bound_halo(std::max(ax1 - 2, ax0), ay0, ax1, ay1),
                                   bound_halo(ax0, ay0, ax1, std::min(ay0 + 2, ay1)),
                                   bound_halo(ax0, std::max(ay1 - 2, ay0), ax1, ay1)};
                bool grew = false;
                for (int k = 0; k < 4; ++k)
                    if (hs[k] > T.h[k]) { T.h[k] = hs[k]; grew = true; }
                if (!grew) break;
            }
            int ax0, ay0, ax1, ay1;
            raster_of(T, ax0, ay0, ax1, ay1);
            T.hp = bound_halo(ax0, ay0, ax1, ay1);
        }
        queue.push_back(T);
    }
    const int64_t ntiles = (int64_t)queue.size();
    const auto t_tiles = clk::now();
    int64_t runs = 0, d2h = 0;
    int batches = 0;
    int max_halo = 0;
    size_t qi = 0;
    dnni_batch_options bo{};
    bo.small_radius = s.small_radius;
    std::vector<dnni_tile> tl;
    std::vector<SegChunk> chunks;
    std::vector<int> order;
    std::vector<Scalars> hsc;
    std::vector<int> ring;
    HostBatch hb;
    DevArrays a;
    // a batch's accepted tiles download on so while the next batch computes
    // into the other of two output buffers (done[b]: buffer b's downloads)
    cudaStream_t so = nullptr;
    cudaEvent_t done[2] = {nullptr, nullptr};
    struct Release {
        cudaStream_t& so;
        cudaEvent_t* done;
        ~Release() {
            if (so) { cudaStreamSynchronize(so); cudaStreamDestroy(so); }
            for (int b = 0; b < 2; ++b) if (done[b]) cudaEventDestroy(done[b]);
        }
    } release_on_exit{so, done};
    if (cudaStreamCreateWithFlags(&so, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming) != cudaSuccess)
        return cuda_err(c, cudaGetLastError(), "segment download stream");
    int ob = 0;
    while (qi < queue.size()) {
        const size_t q1 = std::min(queue.size(), qi + (size_t)s.tiles_per_batch);
        const int ng = (int)(q1 - qi);
        tl.assign(ng, dnni_tile{});
        chunks.clear();
        std::vector<int> rx0(ng), ry0(ng), rw(ng);
        std::vector<char> all_buckets(ng), clipped(4 * ng);
        int64_t pt = 0, out = 0, site = 0;
        for (int k = 0; k < ng; ++k) {
            const SegTile& T = queue[qi + k];
            int ax0, ay0, ax1, ay1;
            raster_of(T, ax0, ay0, ax1, ay1);
            clipped[4 * k + 0] = ax0 == 0;
            clipped[4 * k + 1] = ax1 == s.ncols;
            clipped[4 * k + 2] = ay0 == 0;
            clipped[4 * k + 3] = ay1 == s.nrows;
            rx0[k] = ax0;
            ry0[k] = ay0;
            rw[k] = ax1 - ax0;
            // point box: the raster +- hp, as a range of buckets
            const int bx0 = (int)std::min<long long>(std::max<long long>(floor_div_ll(ax0 - T.hp, kSegBucketCells), 0), nbx - 1);
            const int bx1 = (int)std::min<long long>(std::max<long long>(floor_div_ll(ax1 + T.hp - 1, kSegBucketCells), 0), nbx - 1);
            const int by0 = (int)std::min<long long>(std::max<long long>(floor_div_ll(ay0 - T.hp, kSegBucketCells), 0), nby - 1);
            const int by1 = (int)std::min<long long>(std::max<long long>(floor_div_ll(ay1 + T.hp - 1, kSegBucketCells), 0), nby - 1);
            all_buckets[k] = bx0 == 0 && by0 == 0 && bx1 == nbx - 1 && by1 == nby - 1;
            const int64_t p0 = pt;
            int4 ext = make_int4(INT_MAX, INT_MAX, INT_MIN, INT_MIN);
            for (int by = by0; by <= by1; ++by) {
                const long long a0 = start[(size_t)by * nbx + bx0], a1 = start[(size_t)by * nbx + bx1 + 1];
                for (long long o = a0; o < a1; o += kSegGatherChunk) {
                    const int m = (int)std::min<long long>(kSegGatherChunk, a1 - o);
                    chunks.push_back(SegChunk{o, pt, m, 0});
                    pt += m;
                }
                for (int bx = bx0; bx <= bx1; ++bx) {
                    const int4 bb = bbox[(size_t)by * nbx + bx];
                    if (bb.x > bb.z) continue;
                    ext.x = std::min(ext.x, bb.x); ext.y = std::min(ext.y, bb.y);
                    ext.z = std::max(ext.z, bb.z); ext.w = std::max(ext.w, bb.w);
                }
            }
            dnni_tile& t = tl[k];
            t.wp.ncols = T.x1 - T.x0;
            t.wp.nrows = T.y1 - T.y0;
            t.wp.cell_size = s.cell_size;
            t.wp.origin_x = (int32_t)(s.origin_x + (long long)T.x0 * s.cell_size);
            t.wp.origin_y = (int32_t)(s.origin_y + (long long)T.y0 * s.cell_size);
            t.wp.raster_x0 = ax0 - T.x0;
            t.wp.raster_y0 = ay0 - T.y0;
            t.wp.raster_x1 = ax1 - T.x0;
            t.wp.raster_y1 = ay1 - T.y0;
            t.wp.z_scale = s.z_scale;
            t.wp.z_offset = s.z_offset;
            t.wp.nodata = s.nodata;
            t.pt_offset = p0;
            t.pt_count = pt - p0;
            if (pt > p0) {
                t.ext_x0 = ext.x;
                t.ext_y0 = ext.y;
                t.ext_x1 = ext.z;
                t.ext_y1 = ext.w;
            }
            t.out_offset = out;
            t.site_offset = h_site ? site : -1;
            out += (int64_t)t.wp.ncols * t.wp.nrows;
            site += (int64_t)(ax1 - ax0) * (ay1 - ay0);
        }
        const size_t gp = (size_t)std::max<int64_t>(pt, 1);
        // this buffer's downloads from two batches ago must be over before
        // it is written (or reallocated) again
        CK(cudaEventSynchronize(done[ob]));
        if ((rs = dnni_ensure(c, B.gxyz, 12 * gp)) || (rs = dnni_ensure(c, B.ggid, 4 * gp)) ||
            (rs = dnni_ensure(c, B.gout[ob], 4 * (size_t)std::max<int64_t>(out, 1))) ||
            (h_site && (rs = dnni_ensure(c, B.gsite[ob], 4 * (size_t)std::max<int64_t>(site, 1)))) ||
            (rs = dnni_ensure(c, B.chunks, sizeof(SegChunk) * std::max<size_t>(chunks.size(), 1))))
            return rs;
        float* gout = (float*)B.gout[ob].p;
        uint32_t* gsite = h_site ? (uint32_t*)B.gsite[ob].p : nullptr;
        if (!chunks.empty()) {
            CK(cudaMemcpyAsync(B.chunks.p, chunks.data(), sizeof(SegChunk) * chunks.size(), cudaMemcpyHostToDevice, st));
            k_seg_gather<<<(int)chunks.size(), 256, 0, st>>>((const SegChunk*)B.chunks.p, (const int32_t*)B.sxyz.p,
                                                             (const uint32_t*)B.sgid.p, (int32_t*)B.gxyz.p,
                                                             (uint32_t*)B.ggid.p);
        }
        if ((rs = plan_batch(c, tl.data(), ng, bo, hb, order))) return rs;
        if ((rs = ensure_scratch(c, scr, scratch_sizes(hb), a))) return rs;
        const BatchTables bt = device_tables(a.tables, ng);
        if ((rs = stage_tables(c, hb, a.tables, st))) return rs;
        launch_prologue(hb, bt, a, (const int32_t*)B.gxyz.p, st, false);
        launch_body(hb, bt, a, (const int32_t*)B.gxyz.p, (const uint32_t*)B.ggid.p, gout, gsite, c->sm_count, st,
                    nullptr, true);
        CK(cudaGetLastError());
        hsc.resize(ng);
        ring.resize(4 * (size_t)ng);
        if ((rs = dnni_ensure(c, B.ring, sizeof(int) * 4 * (size_t)ng))) return rs;
        k_ring_max<<<ng, 256, 0, st>>>(bt, a.pix, (int*)B.ring.p);
        CK(cudaMemcpyAsync(ring.data(), B.ring.p, sizeof(int) * 4 * (size_t)ng, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hsc.data(), a.sc, sizeof(Scalars) * ng, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(c->h_ctr, a.ctr, sizeof(BatchCounters), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (c->h_ctr->err & kErrRange)
            return set_err(c, DNNI_E_RANGE, "a point lies beyond +-2^30 LAS units of a tile origin");
        runs += ng;
        ++batches;
        // accept or rerun each tile (batch position k is tile k: no cost order)
        for (int k = 0; k < ng; ++k) {
            const SegTile T = queue[qi + k];
            int mr2 = -1;
            for (int l = 0; l < kStatSlots; ++l) mr2 = std::max(mr2, hsc[k].max_r2[l]);
            // Every raster pixel's nearest-site distance d is below
            // R = sqrt(R2 + 1) cells.  (B) With R <= hp over the whole raster,
            // no point outside the point box (the raster +- hp) is as near as
            // the site found, so the found sites are exact.  (A) A pixel p
            // outside the raster whose disc reaches a core cell q has
            // d(p) >= |p - q|.  Let the segment p-q leave the raster through
            // side s, and c be the point of the segment half a pixel inside
            // that side's outermost line: |c - q| >= h_s - 1/2, and the pixel
            // p' nearest c lies in the side's two outermost lines, within
            // sqrt(2)/2 of c.  d is 1-Lipschitz, so d(p') >= |c - q| -
            // sqrt(2)/2 > h_s - 1.21; R <= h_s - 2 over those two lines rules
            // p out.  A side on the grid's edge has no pixel beyond it.
            // A tile whose point box held no point found no site at all
            // (mr2 < 0): unless its box already covers every bucket (there is
            // no point anywhere), the nearest sites lie beyond the box at a
            // distance nothing here bounds, so the point halo doubles.
            const bool none = mr2 < 0;
            const double R = std::sqrt((double)std::max(mr2, 0) + 1.0);
            const bool okB = all_buckets[k] || (!none && R <= T.hp);
            SegTile U = T;
            bool again = !okB;
            if (!okB) U.hp = none ? std::max(2 * T.hp, 8) : std::max(2 * T.hp, (int)std::ceil(R) + 3);
            for (int sd = 0; sd < 4; ++sd) {
                if (clipped[4 * k + sd]) continue;
                const double Rs = std::sqrt((double)ring[4 * k + sd] + 1.0);
                if (Rs > T.h[sd] - 2) {
                    U.h[sd] = std::max(2 * T.h[sd], (int)std::ceil(Rs) + 3);
                    again = true;
                }
            }
            if (again) {
                queue.push_back(U);
                continue;
            }
            for (int sd = 0; sd < 4; ++sd) max_halo = std::max(max_halo, T.h[sd]);
            const dnni_tile& t = tl[k];
            const size_t w = (size_t)t.wp.ncols, h = (size_t)t.wp.nrows;
            CK(cudaMemcpy2DAsync(h_out + (size_t)T.y0 * s.ncols + T.x0, 4 * (size_t)s.ncols, gout + t.out_offset,
                                 4 * w, 4 * w, h, cudaMemcpyDeviceToHost, so));
            d2h += (int64_t)(4 * w * h);
            if (h_site) {
                const uint32_t* src = gsite + t.site_offset + (size_t)(T.y0 - ry0[k]) * rw[k] + (T.x0 - rx0[k]);
                CK(cudaMemcpy2DAsync(h_site + (size_t)T.y0 * s.ncols + T.x0, 4 * (size_t)s.ncols, src,
                                     4 * (size_t)rw[k], 4 * w, h, cudaMemcpyDeviceToHost, so));
                d2h += (int64_t)(4 * w * h);
            }
        }
        CK(cudaEventRecord(done[ob], so));
        ob ^= 1;
        qi = q1;
    }
    CK(cudaStreamSynchronize(so));
    if (stats) {
        stats->ms_total = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        stats->ms_upload = ms_up;
        stats->ms_bucket = ms_bk;
        stats->ms_bound = std::chrono::duration<double, std::milli>(t_tiles - t_bound).count();
        stats->ms_tiles = std::chrono::duration<double, std::milli>(clk::now() - t_tiles).count();
        stats->points = n;
        stats->cells = (int64_t)s.ncols * s.nrows;
        stats->tiles = ntiles;
        stats->tile_runs = runs;
        stats->h2d_bytes = 12 * n;
        stats->d2h_bytes = d2h;
        stats->max_halo = max_halo;
        stats->batches = batches;
    }
    return DNNI_OK;
}

}  // namespace

extern "C" dnni_status dnni_segment_run(dnni_ctx* c, const dnni_segment* sp, const int32_t* h_xyz, int64_t n,
                                        float* h_out, uint32_t* h_site, dnni_segment_stats* stats) {
    if (!c || !sp || !h_out || n < 0 || (n > 0 && !h_xyz)) return DNNI_E_INVAL;
    c->err.clear();
    DeviceGuard g(c->device);
    dnni_segment s = *sp;
    if (!s.tile) s.tile = 2048;
    if (!s.tiles_per_batch) s.tiles_per_batch = 64;
    if (!s.small_radius) s.small_radius = c->s.small_radius;
    if (s.ncols <= 0 || s.nrows <= 0 || s.ncols > (1 << 20) || s.nrows > (1 << 20))
        return set_err(c, DNNI_E_INVAL, "grid sides must be in [1, 2^20]");
    if (s.cell_size <= 0) return set_err(c, DNNI_E_INVAL, "cell_size must be positive");
    if (s.tile < 32 || s.tile > 16384) return set_err(c, DNNI_E_INVAL, "tile side must be in [32, 16384]");
    if (s.halo < 0 || s.halo == 1 || s.tiles_per_batch < 1 || s.tiles_per_batch > 4096)
        return set_err(c, DNNI_E_INVAL, "bad halo or tiles_per_batch");
    if (s.small_radius < 1 || s.small_radius > kMaxSmallRadius) return set_err(c, DNNI_E_INVAL, "bad small_radius");
    if ((long long)s.ncols * s.cell_size >= (1LL << 30) || (long long)s.nrows * s.cell_size >= (1LL << 30))
        return set_err(c, DNNI_E_RANGE, "grid extent must stay below 2^30 LAS units");
    if ((uint64_t)n >= 0xFFFFFFFFull) return set_err(c, DNNI_E_INVAL, "more points than 32-bit site ids can name");
    if (s.parts < 0 || s.parts > 65536 || (s.parts > 1 && (s.part < 0 || s.part >= s.parts)))
        return set_err(c, DNNI_E_INVAL, "part must lie in [0, parts)");
    // buffers stay with the context (grow-only) for the next call; dnni_clear
    // and dnni_destroy free them
    const dnni_status rs = segment_run(c, s, h_xyz, n, h_out, h_site, stats, c->seg, c->seg_scr);
    if (c->stream) cudaStreamSynchronize(c->stream);
    return rs;
}
