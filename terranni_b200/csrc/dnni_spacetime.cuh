// dnni_spacetime.cuh -- space-time (3-D) interpolation, nni::performNNI with
// timeRadius > 0 (dnni_interpolate_spacetime).  Included by dnni_engine.cu.
//
// The reference loops over the slices ts = curTime + j, j = -timeRadius ..
// timeRadius (nni.cpp:902-933).  Per slice it draws every point within
// timeRadius of ts as a plane whose offset carries the squared time distance
// (drawPlane's timeOffset term, nni.cpp:171-230, 722-790), then draws the
// query planes lifted by j^2 (nni.cpp:483-493) and accumulates into the same
// numer/denom buffers over all slices (cuda_nni.cu:516-548 clears them once per
// call).  Here, in the engine's exact form:
//
//   1. the points are grouped by time value v in [cur - 2rt, cur + 2rt] on
//      the device, each keeping its input index as its gid (ties go to the
//      lower index, the earlier point of the stream);
//   2. one batch of the 2-D engine's nearest-site kernels, one tile per time
//      value, gives every raster pixel its nearest site among that value's
//      points (the site map; the batch stops there);
//   3. k_st_lift: for slice s and pixel p the lifted-nearest site is the
//      minimum over the 2rt + 1 values v within rt of ts of
//      (2-D distance^2 to v's nearest site + ((ts - v) * tau)^2, input index,
//      z) -- the time term is constant within a value, so v's 2-D nearest site
//      is also its lifted-nearest one; the pixel record gets
//      R2 = floor((d_l^2 - (j tau)^2) / cell^2), none when negative;
//   4. the span scatter of the 2-D path runs once per slice into the same
//      per-row difference words, one row scan follows, and k_st_final gathers
//      the small discs of every slice before dividing.
#pragma once

namespace dnni {

constexpr int kStMaxRadius = 16;
constexpr int kStMaxValues = 4 * kStMaxRadius + 1;

constexpr int kStChunk = 4096;          // points per block in the grouping passes

struct StParams {
    int32_t rt, tau, nv, pad;
    int64_t npix;                        // raster pixels of one slice
    int64_t t0;                          // time of value 0 (cur - 2 rt)
    int64_t off[kStMaxValues + 1];       // first grouped row of each time value
};

// Per time value: point count, box (absolute x0, y0, x1, y1, then z0, z1) and
// the scatter cursors; err: a point beyond the coordinate range.
struct StGroupStats {
    int cnt[kStMaxValues];
    int cursor[kStMaxValues];
    int bb[kStMaxValues][6];
    int err;
};

__global__ void k_st_init(StGroupStats* gs) {
    for (int v = threadIdx.x; v < kStMaxValues; v += blockDim.x) {
        gs->cnt[v] = 0;
        gs->cursor[v] = 0;
        gs->bb[v][0] = INT_MAX; gs->bb[v][1] = INT_MAX; gs->bb[v][2] = INT_MIN;
        gs->bb[v][3] = INT_MIN; gs->bb[v][4] = INT_MAX; gs->bb[v][5] = INT_MIN;
    }
    if (threadIdx.x == 0) gs->err = 0;
}

// Time value of point i (-1: in no slice's reach or past the end).
__device__ __forceinline__ int st_value(const int32_t* __restrict__ tt, int64_t i, int64_t n, int64_t t0, int nv) {
    if (i >= n) return -1;
    const int64_t dv = (int64_t)__ldg(&tt[i]) - t0;
    return (dv >= 0 && dv < nv) ? (int)dv : -1;
}

// Grouping pass 1: counts and boxes per time value.  The lanes of a warp
// that hold the same value reduce together; their leader updates the block's
// shared copy, and each block folds its copy into the global one.
__global__ void __launch_bounds__(256) k_st_count(const int32_t* __restrict__ xyz, const int32_t* __restrict__ tt,
                                                  int64_t n, int64_t t0, int nv, int32_t ox, int32_t oy,
                                                  StGroupStats* gs) {
    __shared__ int cnt[kStMaxValues];
    __shared__ int bb[kStMaxValues][6];
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        cnt[v] = 0;
        bb[v][0] = INT_MAX; bb[v][1] = INT_MAX; bb[v][2] = INT_MIN;
        bb[v][3] = INT_MIN; bb[v][4] = INT_MAX; bb[v][5] = INT_MIN;
    }
    __syncthreads();
    const int64_t c0 = (int64_t)blockIdx.x * kStChunk;
    const int64_t c1 = c0 + kStChunk < n ? c0 + kStChunk : n;
    const unsigned lane = threadIdx.x & 31;
    unsigned bad = 0;
    for (int64_t b = c0; b < c1; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const int v = st_value(tt, i, c1, t0, nv);
        int x = 0, y = 0, z = 0;
        if (v >= 0) {
            x = __ldg(&xyz[3 * i]);
            y = __ldg(&xyz[3 * i + 1]);
            z = __ldg(&xyz[3 * i + 2]);
            const int64_t rx = (int64_t)x - ox, ry = (int64_t)y - oy;
            if (rx <= -kCoordLimit || rx >= kCoordLimit || ry <= -kCoordLimit || ry >= kCoordLimit) bad = 1;
        }
        const unsigned grp = __match_any_sync(0xffffffffu, v);
        if (v >= 0) {
            const int x0 = __reduce_min_sync(grp, x), x1 = __reduce_max_sync(grp, x);
            const int y0 = __reduce_min_sync(grp, y), y1 = __reduce_max_sync(grp, y);
            const int z0 = __reduce_min_sync(grp, z), z1 = __reduce_max_sync(grp, z);
            if (lane == (unsigned)(__ffs(grp) - 1)) {
                atomicAdd(&cnt[v], __popc(grp));
                atomicMin(&bb[v][0], x0); atomicMin(&bb[v][1], y0); atomicMax(&bb[v][2], x1);
                atomicMax(&bb[v][3], y1); atomicMin(&bb[v][4], z0); atomicMax(&bb[v][5], z1);
            }
        }
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&gs->err, 1);
    __syncthreads();
    for (int v = threadIdx.x; v < nv; v += blockDim.x) {
        if (!cnt[v]) continue;
        atomicAdd(&gs->cnt[v], cnt[v]);
        atomicMin(&gs->bb[v][0], bb[v][0]); atomicMin(&gs->bb[v][1], bb[v][1]);
        atomicMax(&gs->bb[v][2], bb[v][2]); atomicMax(&gs->bb[v][3], bb[v][3]);
        atomicMin(&gs->bb[v][4], bb[v][4]); atomicMax(&gs->bb[v][5], bb[v][5]);
    }
}

// Grouping pass 2: every point of a value to its group (rows off[v] ..),
// with its input index as the gid that breaks ties.  A block counts its
// points per value, reserves one range per value with a global cursor, then
// places them (order inside a group is free: the gid carries the input order).
__global__ void __launch_bounds__(256) k_st_scatter(const int32_t* __restrict__ xyz, const int32_t* __restrict__ tt,
                                                    int64_t n, StParams P, StGroupStats* gs,
                                                    int32_t* __restrict__ gxyz, uint32_t* __restrict__ gidx) {
    __shared__ int cnt[kStMaxValues];
    __shared__ int base[kStMaxValues];
    for (int v = threadIdx.x; v < P.nv; v += blockDim.x) cnt[v] = 0;
    __syncthreads();
    const int64_t c0 = (int64_t)blockIdx.x * kStChunk;
    const int64_t c1 = c0 + kStChunk < n ? c0 + kStChunk : n;
    const unsigned lane = threadIdx.x & 31, below = (1u << lane) - 1u;
    for (int64_t b = c0; b < c1; b += blockDim.x) {
        const int v = st_value(tt, b + threadIdx.x, c1, P.t0, P.nv);
        const unsigned grp = __match_any_sync(0xffffffffu, v);
        if (v >= 0 && lane == (unsigned)(__ffs(grp) - 1)) atomicAdd(&cnt[v], __popc(grp));
    }
    __syncthreads();
    for (int v = threadIdx.x; v < P.nv; v += blockDim.x) {
        base[v] = cnt[v] ? atomicAdd(&gs->cursor[v], cnt[v]) : 0;
        cnt[v] = 0;
    }
    __syncthreads();
    for (int64_t b = c0; b < c1; b += blockDim.x) {
        const int64_t i = b + threadIdx.x;
        const int v = st_value(tt, i, c1, P.t0, P.nv);
        const unsigned grp = __match_any_sync(0xffffffffu, v);
        const int leader = __ffs(grp) - 1;
        int first = 0;
        if (v >= 0 && (int)lane == leader) first = atomicAdd(&cnt[v], __popc(grp));
        first = __shfl_sync(0xffffffffu, first, leader);
        if (v >= 0) {
            const int64_t q = P.off[v] + base[v] + first + __popc(grp & below);
            gxyz[3 * q] = __ldg(&xyz[3 * i]);
            gxyz[3 * q + 1] = __ldg(&xyz[3 * i + 1]);
            gxyz[3 * q + 2] = __ldg(&xyz[3 * i + 2]);
            gidx[q] = (uint32_t)i;
        }
    }
}

// One thread per (slice, raster pixel); see step 3 above.
// The site maps hold input indices (the batch's gids); xyz is the input.
__global__ void __launch_bounds__(256) k_st_lift(TileParams T, StParams P, const uint32_t* __restrict__ site,
                                                 const int32_t* __restrict__ xyz, int2* __restrict__ pix,
                                                 Scalars* __restrict__ sc) {
    const int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int R2 = -1;
    if (w < (2LL * P.rt + 1) * P.npix) {
        const int s = (int)(w / P.npix);
        const int64_t p = w - (int64_t)s * P.npix;
        const int i = (int)(p % T.rw), j = (int)(p / T.rw);
        const long long px = (long long)(T.rx0 + i) * T.cs, py = (long long)(T.ry0 + j) * T.cs;
        unsigned long long bd = ~0ull;
        uint32_t bg = 0xFFFFFFFFu;
        int bz = INT_MAX;
        for (int k = 0; k <= 2 * P.rt; ++k) {
            const int vi = s + k;                        // time value cur - 2rt + vi, ts - v = rt - k
            const uint32_t g = __ldg(&site[(int64_t)vi * P.npix + p]);
            if (g == 0xFFFFFFFFu) continue;
            const int64_t q = g;
            const long long dx = (long long)rel_coord(__ldg(&xyz[3 * q]), T.ox) - px;
            const long long dy = (long long)rel_coord(__ldg(&xyz[3 * q + 1]), T.oy) - py;
            const long long dt = (long long)(P.rt - k) * P.tau;
            const unsigned long long d2 =
                (unsigned long long)(dx * dx) + (unsigned long long)(dy * dy) + (unsigned long long)(dt * dt);
            const int z = __ldg(&xyz[3 * q + 2]);
            if (d2 < bd || (d2 == bd && (g < bg || (g == bg && z < bz)))) {
                bd = d2;
                bg = g;
                bz = z;
            }
        }
        if (bg != 0xFFFFFFFFu) {
            const long long jt = (long long)(s - P.rt) * P.tau;
            const unsigned long long q2 = (unsigned long long)(jt * jt);
            if (bd >= q2) {
                const unsigned long long e = bd - q2;
                R2 = e > (unsigned long long)LLONG_MAX ? T.r2cap
                                                       : r2_of((long long)e, (long long)T.cs * T.cs, T.r2cap);
            }
        }
        pix[w] = make_int2(R2 >= 0 ? bz : 0, R2);
    }
    const int m = __reduce_max_sync(0xffffffffu, R2);
    if ((threadIdx.x & 31) == 0 && m >= 0)
        atomicMax(&sc->max_r2[(blockIdx.x * 8 + (threadIdx.x >> 5)) & (kStatSlots - 1)], m);
}

// Accumulator form for `layers` stacked slices (decide_packing with the
// per-cell count bound multiplied by the slice count).
__global__ void k_st_decide(Scalars* sc, int zmin, int zmax, long long npix, int layers) {
    int mx = sc->max_r2[threadIdx.x];
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (threadIdx.x == 0) {
        int packed, K;
        long long zbase;
        decide_packing(mx, npix, zmin, zmax, packed, K, zbase, layers);
        sc->packed = packed;
        sc->kbits = K;
        sc->zbase = zbase;
    }
}

// Stencil and divide over `layers` stacked pixel rasters (layer stride lstride): each
// cell gathers the small discs of every slice, adds the prefix-summed span
// words and divides.  One CTA per 32 x 16 cell tile.
template <int H>
__global__ void __launch_bounds__(512) k_st_final(BatchTables bt, const int2* __restrict__ pix, int layers,
                                                  int64_t lstride, Scalars* __restrict__ sc,
                                                  const unsigned long long* __restrict__ S_all,
                                                  const int* __restrict__ Sc_all, float* __restrict__ h_all) {
    constexpr int TX = 32, TY = 16, SW = TX + 2 * H, SH = TY + 2 * H;
    __shared__ int2 tile[SH][SW];
    const int t = find_tile(bt.ct_base, bt.ntiles, blockIdx.x);
    const TileParams& T = bt.tiles[t];
    const int lt = blockIdx.x - __ldg(&bt.ct_base[t]);
    const int nctx = (T.ncols + TX - 1) / TX;
    const int cx0 = (lt % nctx) * TX, cy0 = (lt / nctx) * TY;
    long long Z = 0, C = 0;
    for (int layer = 0; layer < layers; ++layer) {
        const int2* P = pix + T.pix_off + (int64_t)layer * lstride;
        __syncthreads();
        for (int idx = threadIdx.y * TX + threadIdx.x; idx < SW * SH; idx += TX * TY) {
            const int ly = idx / SW, lx = idx - ly * SW;
            const int rxi = cx0 - H + lx - T.rx0, ryi = cy0 - H + ly - T.ry0;
            int2 v = make_int2(0, -1);
            if (rxi >= 0 && rxi < T.rw && ryi >= 0 && ryi < T.rh) v = P[(int64_t)ryi * T.rw + rxi];
            tile[ly][lx] = v;
        }
        __syncthreads();
#pragma unroll
        for (int dy = -H; dy <= H; ++dy)
#pragma unroll
            for (int dx = -H; dx <= H; ++dx) {
                if (dx * dx + dy * dy > H * H) continue;
                const int2 p = tile[threadIdx.y + H + dy][threadIdx.x + H + dx];
                if (p.y >= dx * dx + dy * dy && p.y <= H * H) { Z += p.x; C += 1; }
            }
    }
    const int qx = cx0 + threadIdx.x, qy = cy0 + threadIdx.y;
    unsigned nod = 0;
    Scalars* s = sc + t;
    if (qx < T.ncols && qy < T.nrows) {
        const int64_t q = (int64_t)qy * T.ncols + qx;
        const unsigned long long w = S_all[T.cell_off + q];
        if (s->packed) {
            long long zb, cb;
            decode_span_word(w, s->kbits, s->zbase, zb, cb);
            Z += zb;
            C += cb;
        } else {
            Z += (long long)w;
            C += Sc_all[T.cell_off + q];
        }
        h_all[T.out_off + q] = finalize_height(Z, C, T.z_scale, T.z_offset, T.nodata);
        nod = C <= 0 ? 1u : 0u;
    }
    nod = __reduce_add_sync(0xffffffffu, nod);
    if ((threadIdx.x & 31) == 0 && nod) {
        const int slot = (blockIdx.x + threadIdx.y) & (kStatSlots - 1);
        atomicAdd(&s->nodata[slot], (unsigned long long)nod);
    }
}

void launch_st_final(const BatchTables& bt, int ncta, int rs, const int2* pix, int layers, int64_t lstride,
                     Scalars* sc, const unsigned long long* S, const int* Sc, float* h, cudaStream_t st) {
    dim3 blk(32, 16);
    switch (rs) {
        case 1: k_st_final<1><<<ncta, blk, 0, st>>>(bt, pix, layers, lstride, sc, S, Sc, h); break;
        case 2: k_st_final<2><<<ncta, blk, 0, st>>>(bt, pix, layers, lstride, sc, S, Sc, h); break;
        case 4: k_st_final<4><<<ncta, blk, 0, st>>>(bt, pix, layers, lstride, sc, S, Sc, h); break;
        case 5: k_st_final<5><<<ncta, blk, 0, st>>>(bt, pix, layers, lstride, sc, S, Sc, h); break;
        case 6: k_st_final<6><<<ncta, blk, 0, st>>>(bt, pix, layers, lstride, sc, S, Sc, h); break;
        default: k_st_final<3><<<ncta, blk, 0, st>>>(bt, pix, layers, lstride, sc, S, Sc, h); break;
    }
}

}  // namespace dnni

// Both entry points: host buffers (device = false: points and times copied
// in, heights copied out, the call waits) or device buffers (queued on st;
// it waits once, for the per-value counts, and at the end only for stats).
static dnni_status spacetime_run(dnni_ctx* c, const dnni_workpackage* wp, const dnni_st_options* o,
                                 const int32_t* xyz, const int32_t* tt, int64_t n, float* h_out, bool device,
                                 cudaStream_t st, dnni_stats* stats) {
    const int rt = o->time_radius, tau = o->time_scale;
    if (rt < 0 || rt > kStMaxRadius || tau <= 0 || (int64_t)rt * tau > (1LL << 30))
        return set_err(c, DNNI_E_INVAL, "time_radius must be in [0, 16], time_scale > 0, their product <= 2^30");
    TileParams T;
    const char* msg = "";
    dnni_status rs = plan_geometry(wp, 0, c->s.small_radius, T, &msg);
    if (rs) return set_err(c, rs, msg);
    const int S = 2 * rt + 1, V = 4 * rt + 1;
    const int64_t npix = (int64_t)T.rw * T.rh, cells = (int64_t)T.ncols * T.nrows;
    if (npix * V >= (int64_t)INT32_MAX) return set_err(c, DNNI_E_INVAL, "raster pixels x time values exceed 2^31");

    if (n > (int64_t)INT32_MAX - 1) return set_err(c, DNNI_E_INVAL, "more than 2^31 - 2 points");
    const int64_t t0 = (int64_t)o->cur_time - 2 * rt;
    const int64_t nb = std::max<int64_t>(n, 1);
    if ((!device && ((rs = dnni_ensure(c, c->st.xin, sizeof(int32_t) * 3 * (size_t)nb)) ||
                     (rs = dnni_ensure(c, c->st.tin, sizeof(int32_t) * (size_t)nb)) ||
                     (rs = dnni_ensure(c, c->out_h, sizeof(float) * (size_t)cells)))) ||
        (rs = dnni_ensure(c, c->st.xyz, sizeof(int32_t) * 3 * (size_t)nb)) ||
        (rs = dnni_ensure(c, c->st.idx, sizeof(uint32_t) * (size_t)nb)) ||
        (rs = dnni_ensure(c, c->st.gs, sizeof(StGroupStats))) ||
        (rs = dnni_ensure(c, c->st.site, sizeof(uint32_t) * (size_t)(V * npix))) ||
        (rs = dnni_ensure(c, c->st.pix, sizeof(int2) * (size_t)(S * npix))))
        return rs;
    const int32_t* dxyz = device ? xyz : (const int32_t*)c->st.xin.p;
    const int32_t* dt = device ? tt : (const int32_t*)c->st.tin.p;
    float* dh = device ? h_out : (float*)c->out_h.p;
    const bool timing = stats || (c->s.flags & DNNI_F_TIMING);
    if (timing) CK(cudaEventRecord(c->ev[0], st));

    // 1. upload, then group the points of the 4rt + 1 time values on the device
    StGroupStats* gs = (StGroupStats*)c->st.gs.p;
    k_st_init<<<1, 128, 0, st>>>(gs);
    const int nchunk = (int)((n + kStChunk - 1) / kStChunk);
    if (n > 0) {
        if (!device) {
            CK(cudaMemcpyAsync(c->st.xin.p, xyz, sizeof(int32_t) * 3 * (size_t)n, cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(c->st.tin.p, tt, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
        }
        k_st_count<<<nchunk, 256, 0, st>>>(dxyz, dt, n, t0, V, wp->origin_x, wp->origin_y, gs);
    }
    StGroupStats hg;
    CK(cudaMemcpyAsync(&hg, gs, sizeof(StGroupStats), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hg.err) return set_err(c, DNNI_E_RANGE, "a point lies beyond +-2^30 LAS units of the work-package origin");
    StParams P;
    memset(&P, 0, sizeof(P));
    P.rt = rt;
    P.tau = tau;
    P.nv = V;
    P.npix = npix;
    P.t0 = t0;
    for (int v = 0; v < V; ++v) P.off[v + 1] = P.off[v] + hg.cnt[v];
    const int64_t m = P.off[V];
    int zmin = INT_MAX, zmax = INT_MIN;
    for (int v = 0; v < V; ++v)
        if (hg.cnt[v]) {
            zmin = std::min(zmin, hg.bb[v][4]);
            zmax = std::max(zmax, hg.bb[v][5]);
        }
    if (m > 0)
        k_st_scatter<<<nchunk, 256, 0, st>>>(dxyz, dt, n, P, gs, (int32_t*)c->st.xyz.p, (uint32_t*)c->st.idx.p);

    // 2. nearest site per time value: one 2-D batch, one tile per value
    std::vector<dnni_tile> tiles((size_t)V);
    for (int v = 0; v < V; ++v) {
        dnni_tile& d = tiles[v];
        memset(&d, 0, sizeof(d));
        d.wp = *wp;
        d.pt_offset = P.off[v];
        d.pt_count = P.off[v + 1] - P.off[v];
        d.out_offset = (int64_t)v * cells;
        d.site_offset = (int64_t)v * npix;
        if (d.pt_count > 0) {
            d.ext_x0 = hg.bb[v][0];
            d.ext_y0 = hg.bb[v][1];
            d.ext_x1 = hg.bb[v][2];
            d.ext_y1 = hg.bb[v][3];
            if (!(d.ext_x0 || d.ext_y0 || d.ext_x1 || d.ext_y1)) d.ext_x1 = 1;   // all zero reads as "the raster"
        }
    }
    {
        dnni_batch_options bo{};
        HostBatch vb;
        std::vector<int> order;
        if ((rs = plan_batch(c, tiles.data(), V, bo, vb, order))) return rs;
        DevArrays va;
        if ((rs = ensure_scratch(c, c->st.scr, scratch_sizes(vb), va))) return rs;
        const BatchTables vbt = device_tables(va.tables, V);
        if ((rs = stage_tables(c, vb, va.tables, st))) return rs;
        const int32_t* dx = m > 0 ? (const int32_t*)c->st.xyz.p : nullptr;
        launch_prologue(vb, vbt, va, dx, st, false);
        launch_body(vb, vbt, va, dx, (const uint32_t*)c->st.idx.p, nullptr, (uint32_t*)c->st.site.p, c->sm_count, st,
                    nullptr, true, true);
        CK(cudaGetLastError());
    }
    if (timing) CK(cudaEventRecord(c->ev[1], st));

    // 3-4. lift the site maps into per-slice pixel records, scatter, finalize
    int32_t nobb[6] = {INT_MAX, INT_MIN, INT_MAX, INT_MIN, INT_MAX, INT_MIN};
    plan_bins(nobb, 0, c->s.bin_target, T);
    HostBatch hb;
    hb.rs = c->s.small_radius;
    batch_add(hb, T, 0, 0, -1);
    DevArrays a;
    if ((rs = ensure_scratch(c, c->scr, scratch_sizes(hb), a))) return rs;
    BatchTables bt = device_tables(a.tables, 1);
    if ((rs = stage_tables(c, hb, a.tables, st))) return rs;
    k_init_scalars<<<1, 32, 0, st>>>(bt, a.sc, a.ctr);
    int2* pix = (int2*)c->st.pix.p;
    const int64_t lifts = (int64_t)S * npix;
    k_st_lift<<<(unsigned)((lifts + 255) / 256), 256, 0, st>>>(T, P, (const uint32_t*)c->st.site.p, dxyz, pix,
                                                               a.sc);
    k_st_decide<<<1, 32, 0, st>>>(a.sc, m > 0 ? zmin : 1, m > 0 ? zmax : 0, npix, S);
    if (timing) CK(cudaEventRecord(c->ev[2], st));
    CK(cudaMemsetAsync(a.D, 0, sizeof(unsigned long long) * (size_t)cells, st));
    CK(cudaMemsetAsync(a.Dc, 0, sizeof(int) * (size_t)cells, st));
    const int nrt = hb.rt_base.back();
    for (int s = 0; s < S; ++s)
        k_scatter_window<<<nrt, dim3(32, 8), sizeof(unsigned long long) * hb.win_words, st>>>(
            bt, pix + (int64_t)s * npix, a.sc, a.D, a.Dc, hb.win_words);
    if (timing) CK(cudaEventRecord(c->ev[3], st));
    k_rowscan<<<hb.grow_base.back(), kScanThreads, 0, st>>>(bt, a.D, a.Dc, a.sc);
    launch_st_final(bt, hb.ct_base.back(), hb.rs, pix, S, npix, a.sc, a.D, a.Dc, dh, st);
    CK(cudaGetLastError());
    if (timing) CK(cudaEventRecord(c->ev[4], st));
    if (!device) CK(cudaMemcpyAsync(h_out, c->out_h.p, sizeof(float) * (size_t)cells, cudaMemcpyDeviceToHost, st));
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        CK(cudaMemcpyAsync(c->h_sc, a.sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st));
    }
    if (!device || timing) CK(cudaStreamSynchronize(st));
    c->calls++;
    if (timing) {
        float ms[4];
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&ms[k], c->ev[k], c->ev[k + 1]);
        for (int k = 0; k < 4; ++k) c->acc_ms[k] += ms[k];
        if (stats) {
            stats->ms_bin = ms[0];          // upload + the per-value 2-D batch
            stats->ms_nearest = ms[1];      // lift into slices
            stats->ms_scatter = ms[2];
            stats->ms_finalize = ms[3];
            stats->ms_total = ms[0] + ms[1] + ms[2] + ms[3];
        }
    }
    if (stats) {
        stats->n_points = m;
        stats->n_cells = cells;
        stats->n_pixels = npix * S;
        fold_stats(c->h_sc, 1, stats);
        stats->h2d_bytes = device ? 0 : (int64_t)(16 * n);
        stats->d2h_bytes = device ? 0 : (int64_t)(sizeof(float) * cells);
    }
    return DNNI_OK;
}

extern "C" dnni_status dnni_interpolate_spacetime(dnni_ctx* c, const dnni_workpackage* wp, const dnni_st_options* o,
                                                  const int32_t* xyz, const int32_t* tt, int64_t n, float* h_out,
                                                  dnni_stats* stats) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    if (!wp || !o || !h_out || n < 0 || (n > 0 && (!xyz || !tt)))
        return set_err(c, DNNI_E_INVAL, "NULL argument or negative point count");
    DeviceGuard g(c->device);
    return spacetime_run(c, wp, o, xyz, tt, n, h_out, false, c->stream, stats);
}

extern "C" dnni_status dnni_interpolate_spacetime_device(dnni_ctx* c, const dnni_workpackage* wp,
                                                         const dnni_st_options* o, const int32_t* d_xyz,
                                                         const int32_t* d_t, int64_t n, float* d_h, void* stream,
                                                         dnni_stats* stats) {
    if (!c) return DNNI_E_INVAL;
    c->err.clear();
    if (!wp || !o || !d_h || n < 0 || (n > 0 && (!d_xyz || !d_t)))
        return set_err(c, DNNI_E_INVAL, "NULL argument or negative point count");
    DeviceGuard g(c->device);
    return spacetime_run(c, wp, o, d_xyz, d_t, n, d_h, true, stream ? (cudaStream_t)stream : c->stream, stats);
}
