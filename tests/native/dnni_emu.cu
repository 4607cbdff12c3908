// dnni_emu.cu -- TEST INFRASTRUCTURE: a host build of the engine's per-work-
// package pipeline.  It runs the very same search and packing helpers as the
// device kernels (dnni_kernels.cuh is __host__ __device__ for them), with
// sequential loops in place of the launches and plain adds in place of the
// atomics, so that the CPU-only test suite can check the kernels' algorithm
// bit-exactly against the oracle.  It is not part of the product.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/dnni.h"
#include "../../terranni_b200/csrc/dnni_search.cuh"
#include "../../terranni_b200/csrc/dnni_plan.h"

using namespace dnni;

static float host_height(long long Z, long long C, double zs, double zo, float nodata) {
    if (C <= 0) return nodata;
    volatile double q = (double)Z / (double)C;
    volatile double v = q * zs;
    v = v + zo;
    return (float)v;
}

extern "C" int emu_interpolate(const dnni_workpackage* wp, const int32_t* xyz, const uint32_t* gid, int64_t n,
                               int small_radius, int bin_target, float* h, uint32_t* site, int32_t* r2_out,
                               int64_t* info) {
    TileParams t;
    const char* msg;
    int rs = small_radius ? small_radius : 3;
    dnni_status st = plan_geometry(wp, n, rs, t, &msg);
    if (st) return st;
    int32_t bbox[6] = {INT32_MAX, INT32_MIN, INT32_MAX, INT32_MIN, INT32_MAX, INT32_MIN};
    for (int64_t i = 0; i < n; ++i) {
        const long long x = (long long)xyz[3 * i] - t.ox, y = (long long)xyz[3 * i + 1] - t.oy, z = xyz[3 * i + 2];
        if (x <= -kCoordLimit || x >= kCoordLimit || y <= -kCoordLimit || y >= kCoordLimit || z <= -kCoordLimit ||
            z >= kCoordLimit)
            return DNNI_E_RANGE;
        bbox[0] = std::min<int32_t>(bbox[0], (int32_t)x); bbox[1] = std::max<int32_t>(bbox[1], (int32_t)x);
        bbox[2] = std::min<int32_t>(bbox[2], (int32_t)y); bbox[3] = std::max<int32_t>(bbox[3], (int32_t)y);
        bbox[4] = std::min<int32_t>(bbox[4], (int32_t)z); bbox[5] = std::max<int32_t>(bbox[5], (int32_t)z);
    }
    plan_bins(bbox, n, (double)bin_target, t);
    const BinGrid& g = t.bg;
    std::vector<int> cnt(g.nbins + 1, 0), start(g.nbins + 1, 0);
    std::vector<int4> sorted(n > 0 ? n : 1);
    std::vector<int64_t> pb(n > 0 ? n : 1);
    for (int64_t i = 0; i < n; ++i) {
        pb[i] = point_bin(g, rel_coord(xyz[3 * i], t.ox), rel_coord(xyz[3 * i + 1], t.oy));
        cnt[pb[i]]++;
    }
    int run = 0;
    for (int64_t b = 0; b <= g.nbins; ++b) { start[b] = run; run += cnt[b]; }
    std::vector<int> fill(start.begin(), start.end());
    for (int64_t i = 0; i < n; ++i)
        sorted[fill[pb[i]]++] = make_int4(rel_coord(xyz[3 * i], t.ox), rel_coord(xyz[3 * i + 1], t.oy), xyz[3 * i + 2],
                                          (int)(gid ? gid[i] : (uint32_t)i));
    const int64_t nblk = g.nbins / kBinsPerBlock, nsup = g.nbins / kBinsPerSuper;
    std::vector<uint64_t> bmask(nblk, 0), smask(nsup, 0);
    for (int64_t k = 0; k < nblk; ++k)
        for (int l = 0; l < 64; ++l)
            if (start[k * 64 + l + 1] != start[k * 64 + l]) bmask[k] |= 1ull << l;
    for (int64_t k = 0; k < nsup; ++k)
        for (int m = 0; m < 64; ++m)
            if (bmask[k * 64 + m]) smask[k] |= 1ull << m;
    // nearest non-empty block map (the k_block_rows / k_block_near rule)
    const int n1x = g.nbx >> 3, n1y = g.nby >> 3;
    std::vector<int> rownear((size_t)n1x * n1y, -1);
    std::vector<int64_t> nearmap((size_t)n1x * n1y, -1);
    for (int cy = 0; cy < n1y; ++cy) {
        int last = -1;
        for (int cx = 0; cx < n1x; ++cx) {
            if (bmask[block_index(g, cx, cy)]) last = cx;
            rownear[(size_t)cy * n1x + cx] = last;
        }
        last = -1;
        for (int cx = n1x - 1; cx >= 0; --cx) {
            if (bmask[block_index(g, cx, cy)]) last = cx;
            const int l = rownear[(size_t)cy * n1x + cx];
            if (last >= 0 && (l < 0 || last - cx < cx - l)) rownear[(size_t)cy * n1x + cx] = last;
        }
    }
    for (int cy = 0; cy < n1y; ++cy)
        for (int cx = 0; cx < n1x; ++cx) {
            long long best = LLONG_MAX;
            int bxn = -1, byn = -1;
            for (int d = 0; d < n1y; ++d) {
                if ((long long)d * d > best) break;
                for (int sgn = -1; sgn <= 1; sgn += 2) {
                    if (d == 0 && sgn > 0) continue;
                    const int y = cy + sgn * d;
                    if (y < 0 || y >= n1y) continue;
                    const int x = rownear[(size_t)y * n1x + cx];
                    if (x < 0) continue;
                    const long long v = (long long)(x - cx) * (x - cx) + (long long)d * d;
                    if (v < best) { best = v; bxn = x; byn = y; }
                }
            }
            nearmap[(size_t)cy * n1x + cx] = bxn >= 0 ? block_index(g, bxn, byn) : -1;
        }
    const int64_t npix = (int64_t)t.rw * t.rh, cells = (int64_t)t.ncols * t.nrows;
    std::vector<int2> pix(npix);
    int max_r2 = -1;
    std::vector<int2> farl;   // (pixel, best so far)
    auto settle = [&](int i, int j, const Best& b) {
        const int R2 = r2_of(b.d2, (long long)t.cs * t.cs, t.r2cap);
        pix[(int64_t)j * t.rw + i] = make_int2(b.z, R2);
        if (site) site[(int64_t)j * t.rw + i] = b.gid;
        if (r2_out) r2_out[(int64_t)j * t.rw + i] = R2;
        max_r2 = std::max(max_r2, R2);
    };
    // dense pass: per 32 x 8 tile, staged window (as the device kernel) or the global arrays
    std::vector<int> lstart(kWinMaxBins + 1), gstart(kWinMaxBins);
    std::vector<int4> lpts(kWinMaxPts);
    for (int j0 = 0; j0 < t.rh; j0 += kTileY)
        for (int i0 = 0; i0 < t.rw; i0 += kTileX) {
            bool staged = false;
            int wx0 = 0, wy0 = 0, wnx = 0, wny = 0;
            if (n > 0) {
                tile_window(t, i0, j0, kTileY, wx0, wy0, wnx, wny);
                const int nwb = wnx * wny;
                if (nwb <= kWinMaxBins && wny <= kWinMaxRows) {
                    int run2 = 0;
                    for (int lk = 0; lk < nwb; ++lk) {
                        const int64_t id = bin_id(g, wx0 + lk % wnx, wy0 + lk / wnx);
                        lstart[lk] = run2;
                        gstart[lk] = start[id];
                        run2 += start[id + 1] - start[id];
                    }
                    lstart[nwb] = run2;
                    staged = run2 <= kWinMaxPts;
                    if (staged)
                        for (int lk = 0; lk < nwb; ++lk)
                            for (int q = lstart[lk]; q < lstart[lk + 1]; ++q) lpts[q] = sorted[gstart[lk] + (q - lstart[lk])];
                }
            }
            for (int j = j0; j < std::min(j0 + kTileY, t.rh); ++j)
                for (int i = i0; i < std::min(i0 + kTileX, t.rw); ++i) {
                    if (n == 0) {
                        pix[(int64_t)j * t.rw + i] = make_int2(0, -1);
                        if (site) site[(int64_t)j * t.rw + i] = 0xFFFFFFFFu;
                        if (r2_out) r2_out[(int64_t)j * t.rw + i] = -1;
                        continue;
                    }
                    const int px = (t.rx0 + i) * t.cs, py = (t.ry0 + j) * t.cs;
                    Best b{LLONG_MAX, 0xFFFFFFFFu, INT_MAX, -1};
                    bool done;
                    if (staged) {
                        const BinWindow w{wx0, wy0, wnx, wny, lstart.data(), gstart.data(), lpts.data()};
                        done = window_fits32(g, w) ? search_window_fast32(g, w, px, py, b)
                                                   : search_window_fast(g, w, px, py, b);
                        if (!done) b.idx = window_global_index(w, b.idx);
                    } else {
                        done = search_bins(g, sorted.data(), start.data(), px, py, b);
                    }
                    if (done) settle(i, j, b);
                    else farl.push_back(make_int2(j * t.rw + i, b.idx));
                }
        }
    // far pass
    for (const int2& it : farl) {
        const int i = it.x % t.rw, j = it.x / t.rw;
        const int px = (t.rx0 + i) * t.cs, py = (t.ry0 + j) * t.cs;
        Best b{LLONG_MAX, 0xFFFFFFFFu, INT_MAX, -1};
        if (it.y >= 0) consider(b, sorted[it.y], it.y, px, py);
        finish_search(g, sorted.data(), start.data(), bmask.data(), smask.data(), px, py, b, nearmap.data());
        settle(i, j, b);
    }
    int packed, K;
    long long zbase;
    decide_packing(max_r2, npix, bbox[4], bbox[5], packed, K, zbase);
    std::vector<unsigned long long> D(cells, 0);
    std::vector<int> Dc(cells, 0);
    int64_t spans = 0, bigpix = 0;
    auto emit = [&](int row, int a, int b, unsigned long long v, long long z) {
        if (row < 0 || row >= t.nrows) return;
        a = std::max(a, 0);
        b = std::min(b, t.ncols - 1);
        if (a > b) return;
        const int64_t base = (int64_t)row * t.ncols;
        if (packed) {
            D[base + a] += v;
            if (b + 1 < t.ncols) D[base + b + 1] -= v;
        } else {
            D[base + a] += (unsigned long long)z;
            Dc[base + a] += 1;
            if (b + 1 < t.ncols) { D[base + b + 1] -= (unsigned long long)z; Dc[base + b + 1] -= 1; }
        }
    };
    for (int j = 0; j < t.rh; ++j)
        for (int i = 0; i < t.rw; ++i) {
            const int2 p = pix[(int64_t)j * t.rw + i];
            if (p.y <= rs * rs) continue;
            bigpix++;
            const int r = isqrt_i32(p.y);
            spans += 2 * r + 1;
            const unsigned long long v = span_word(p.x, zbase, K);
            const int px = t.rx0 + i, py = t.ry0 + j;
            int w = r;
            for (int dy = 0; dy <= r; ++dy) {
                const long long t2 = (long long)p.y - (long long)dy * dy;
                while ((long long)w * w > t2) --w;
                emit(py + dy, px - w, px + w, v, p.x);
                if (dy) emit(py - dy, px - w, px + w, v, p.x);
            }
        }
    for (int row = 0; row < t.nrows; ++row) {
        unsigned long long s = 0;
        int sc = 0;
        for (int x = 0; x < t.ncols; ++x) {
            s += D[(int64_t)row * t.ncols + x];
            sc += Dc[(int64_t)row * t.ncols + x];
            D[(int64_t)row * t.ncols + x] = s;
            Dc[(int64_t)row * t.ncols + x] = sc;
        }
    }
    int64_t nodata = 0;
    for (int qy = 0; qy < t.nrows; ++qy)
        for (int qx = 0; qx < t.ncols; ++qx) {
            long long Z = 0, C = 0;
            for (int dy = -rs; dy <= rs; ++dy)
                for (int dx = -rs; dx <= rs; ++dx) {
                    const int d2 = dx * dx + dy * dy;
                    if (d2 > rs * rs) continue;
                    const int ri = qx + dx - t.rx0, rj = qy + dy - t.ry0;
                    if (ri < 0 || rj < 0 || ri >= t.rw || rj >= t.rh) continue;
                    const int2 p = pix[(int64_t)rj * t.rw + ri];
                    if (p.y >= d2 && p.y <= rs * rs) { Z += p.x; C += 1; }
                }
            const int64_t q = (int64_t)qy * t.ncols + qx;
            if (packed) {
                long long zb, cb;
                decode_span_word(D[q], K, zbase, zb, cb);
                Z += zb;
                C += cb;
            } else {
                Z += (long long)D[q];
                C += Dc[q];
            }
            h[q] = host_height(Z, C, t.z_scale, t.z_offset, t.nodata);
            nodata += C <= 0;
        }
    if (info) {
        info[0] = packed; info[1] = K; info[2] = zbase; info[3] = g.bs;
        info[4] = bigpix; info[5] = spans; info[6] = nodata; info[7] = max_r2;
    }
    return 0;
}

// exposes the device helpers r2_of and udiv32 for direct tests
extern "C" int emu_r2_of(long long d2, long long cs2, int cap) { return r2_of(d2, cs2, cap); }

// exposes the block cell-box mask that the far pass's seed uses
extern "C" unsigned long long emu_cell_box_mask8(int a0, int a1, int b0, int b1) {
    return cell_box_mask8(a0, a1, b0, b1);
}

// exposes the planning distance transform used for the segment driver's halos
extern "C" void emu_edt_2d(const unsigned char* occ, int nx, int ny, double* out) {
    const std::vector<double> g = edt_2d(occ, nx, ny);
    for (size_t k = 0; k < g.size(); ++k) out[k] = g[k];
}
