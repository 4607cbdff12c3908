/*
 * nni/nni.h -- drop-in for TerraNNI's `nni::` library interface (nni.h:32-99)
 * on top of the B200 engine's C ABI (dnni.h, libdnni.so).
 *
 * Same namespace, type names, field layouts and function signatures as the
 * reference, so that its caller (binRun, terranni.cpp:394-426) compiles
 * unchanged against this header and links libdnni.so instead of the
 * GL-based nni library:
 *
 *   Point3D / Point4D / OutPoint / WorkPackage / Settings   nni.h:34-81
 *   init, cleanup, setRenderbuffers, printTimes, setupRun,
 *   performNNI, clearRenderbuffers                          nni.h:83-97
 *
 * Semantics follow the engine's canonical mode (dnni.h): raster pixels on the
 * cell lattice, every site's region of influence unbounded, ties to the
 * earliest point in the stream, exact int64 sums.  World coordinates are
 * quantised to int32 LAS units relative to the work-package origin at
 * `xy_scale` (0.01 m unless setCoordinateScale says otherwise); z at
 * `z_scale`.  Cells that no pixel reaches get -9999, as in the reference
 * (cuda_nni.cu:497-498, nni.cpp:842).
 *
 * Errors: the reference's functions return void and exit() on GL failures
 * (nni.cpp:310-316); here every failure throws nni::Error carrying the
 * engine's status and message.
 *
 * setCompatMode(true) switches performNNI to the reference's own default
 * semantics instead (dnni_interpolate_compat): square site and query regions,
 * a pixel lattice Settings::scale times finer than the cells, float32 plane
 * depths with the later-drawn site winning ties, int32 z-codes quantised by
 * Settings::pointMin and Settings::multiplier, truncating divide.  Points are
 * then taken as world doubles, without the LAS quantisation.
 *
 * Space-time (timeRadius > 0, nni.cpp:902-933) runs dnni_interpolate_spacetime
 * on the points the reference's slice loop reads (nni.cpp:722-790, with its
 * renderbuffer reuse across calls in the Delta mode, nni.cpp:325-359, and its
 * stream seeks); the stream must be sorted by time, as the reference's
 * binning leaves it (terranni.cpp:120-126).  timeRadius and curTime must be
 * whole numbers; one time step counts as one world unit of distance, as in
 * drawPlane (nni.cpp:198), unless setTimeScale says otherwise.  Not with
 * setCompatMode.
 */
#ifndef DNNI_NNI_SHIM_H
#define DNNI_NNI_SHIM_H

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include <tpie/stream.h>

#include "../dnni.h"

namespace nni {

struct Point3D {
    double p[3];  // x,y,z
    Point3D(double x, double y, double z, double t = 0) {
        (void)t;
        p[0] = x;
        p[1] = y;
        p[2] = z;
    }
    Point3D() {}
};

struct Point4D : public Point3D {
    int t;
    Point4D(double x, double y, double z, int time = 0) {
        p[0] = x;
        p[1] = y;
        p[2] = z;
        t = time;
    }
    Point4D() {}
};

struct OutPoint {
    int i, j;
    float h;
    OutPoint(int x, int y, float z) {
        i = x;
        j = y;
        h = z;
    }
    OutPoint() {}
};

struct WorkPackage {
    float origin_x, origin_y;            // grid offset
    float grid_origin_x, grid_origin_y;
    int nrows, ncols;
};

struct Settings {
    int scale;
    float cell_size;  // cell dimension
    int nrows, ncols;
    float site_radius;
    double query_radius;
    int algorithm;
    int pointMin;
    int multiplier;
};

class Error : public std::runtime_error {
public:
    Error(dnni_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
    dnni_status status;
};

namespace detail {
struct State {
    dnni_ctx* ctx = nullptr;
    Settings s{};
    double xy_scale = 0.01, z_scale = 0.01;
    int device = 0;
    bool compat = false;
    double time_scale = 1.0;                 // world units per time step
    // space-time: slice times whose sites were read (the reference's rbTimes),
    // the renderbuffer shape they belong to, and every point read for them,
    // by stream position
    std::vector<int> rb_times;
    long long rb_key[3] = {-1, -1, -1};
    std::map<long long, Point4D> st_points;
    double ms_points = 0, ms_engine = 0, ms_write = 0;
    long long calls = 0;
    std::vector<int32_t> xyz;
    std::vector<double> world;
    std::vector<int32_t> times;
    std::vector<uint32_t> gid;
    std::vector<float> h;
};
inline State& state() {
    static State st;
    return st;
}
inline void check(dnni_status rc, const char* what) {
    if (rc != DNNI_OK) {
        const char* m = state().ctx ? dnni_last_error(state().ctx) : "";
        throw Error(rc, std::string(what) + ": " + (m ? m : ""));
    }
}
// pixel_offset as nni::performNNI derives it (nni.cpp:881-883), scaling 1
inline int default_pixel_offset(const Settings& s) {
    const double ps = s.cell_size;
    return (int)std::ceil((s.query_radius - 0.0 * ps) / ps) + 1;
}
inline dnni_workpackage to_dnni(const WorkPackage& wp, int pixel_offset) {
    State& st = state();
    dnni_workpackage d{};
    d.ncols = wp.ncols;
    d.nrows = wp.nrows;
    const double cs = st.s.cell_size / st.xy_scale;
    d.cell_size = (int32_t)std::llround(cs);
    if (d.cell_size <= 0 || std::fabs(cs - d.cell_size) > 1e-6 * cs)
        throw Error(DNNI_E_INVAL, "cell_size is not a whole number of LAS units at the coordinate scale");
    d.origin_x = 0;
    d.origin_y = 0;
    const int po = pixel_offset >= 0 ? pixel_offset : default_pixel_offset(st.s);
    d.raster_x0 = -po;
    d.raster_y0 = -po;
    d.raster_x1 = wp.ncols + po;
    d.raster_y1 = wp.nrows + po;
    d.z_scale = st.z_scale;
    d.z_offset = 0.0;
    d.nodata = -9999.0f;
    return d;
}
}  // namespace detail

/* Coordinate quantisation used to turn world coordinates into int32 LAS
 * units (extension; the reference works on GL floats). */
inline void setCoordinateScale(double xy_scale, double z_scale) {
    detail::state().xy_scale = xy_scale;
    detail::state().z_scale = z_scale;
}

/* Reference-default semantics for the following performNNI calls
 * (extension; the reference's behaviour with its default build options). */
inline void setCompatMode(bool on) { detail::state().compat = on; }

/* World units of distance per time step in space-time interpolation
 * (extension; the reference's planes count one step as one unit). */
inline void setTimeScale(double world_units_per_step) { detail::state().time_scale = world_units_per_step; }

/* Device used by the next init() (extension; the reference uses device 0,
 * cuda_nni.cu:659). */
inline void setDevice(int device) { detail::state().device = device; }

inline void cleanup() {
    detail::State& st = detail::state();
    if (st.ctx) dnni_destroy(st.ctx);
    st.ctx = nullptr;
}

/* nni.cpp:569-598: stores the settings and creates the engine context.
 * Returns the largest supported grid side (the reference returns the GL
 * texture limit). */
inline int init(const Settings& s) {
    detail::State& st = detail::state();
    st.s = s;
    if (!st.ctx) {
        dnni_settings ds{};
        ds.device = st.device;
        dnni_status rc = dnni_init(&ds, &st.ctx);
        if (rc != DNNI_OK) throw Error(rc, "dnni_init failed (no CUDA device?)");
    }
    return 32767;
}

/* nni.cpp:381-462 sized GL renderbuffers; the engine sizes its device
 * scratch on demand, so this only reserves it for a grid of that size. */
inline void setRenderbuffers(int w_width, int w_height, int tC = 1) {
    (void)tC;
    detail::State& st = detail::state();
    if (!st.ctx) throw Error(DNNI_E_STATE, "setRenderbuffers before init");
    dnni_workpackage d{};
    d.ncols = w_width;
    d.nrows = w_height;
    d.cell_size = 1;
    detail::check(dnni_setup_run(st.ctx, &d, 0), "setRenderbuffers");
}

inline void printTimes() {
    const detail::State& st = detail::state();
    std::fprintf(stdout, "Time Results:\n");
    std::fprintf(stdout, "\tRead site points : \t\t%f\n", st.ms_points / 1e3);
    std::fprintf(stdout, "\tInterpolate (GPU): \t\t%f\n", st.ms_engine / 1e3);
    std::fprintf(stdout, "\tWrite query points: \t\t%f\n", st.ms_write / 1e3);
}

/* nni.cpp:601-668: reserves device scratch for this work package. */
inline void setupRun(const WorkPackage& wp, int pixel_offset = -1, int timeCount = 1) {
    (void)timeCount;
    detail::State& st = detail::state();
    if (!st.ctx) throw Error(DNNI_E_STATE, "setupRun before init");
    dnni_workpackage d = detail::to_dnni(wp, pixel_offset);
    detail::check(dnni_setup_run(st.ctx, &d, 0), "setupRun");
}

namespace detail {
inline void emit_outpoints(const WorkPackage& wp, tpie::ami::stream<OutPoint>& out) {
    State& st = state();
    for (int i = 0; i < wp.ncols; i++) {
        for (int j = 0; j < wp.nrows; j++) {
            OutPoint o((int)(i + wp.grid_origin_x), (int)(j + wp.grid_origin_y), st.h[(size_t)j * wp.ncols + i]);
            if (o.i < st.s.ncols && o.j < st.s.nrows) out.write_item(o);
        }
    }
}

// nni.cpp:902-933 for timeRadius > 0: the slice loop's reads and seeks
// (renderInputPoints, nni.cpp:722-790) and, in the Delta mode, the reuse of
// slices already drawn (switchRenderbuffers, nni.cpp:325-359); the points
// read feed dnni_interpolate_spacetime.
inline void performNNISpaceTime(const WorkPackage& wp, tpie::ami::stream<OutPoint>& out,
                                tpie::ami::stream<Point4D>& vec, float timeRadius, float curTime, bool useDelta) {
    State& st = state();
    if (st.compat) throw Error(DNNI_E_INVAL, "space-time interpolation has no reference-compatible mode");
    if (timeRadius < 0 || timeRadius != std::floor(timeRadius) || curTime != std::floor(curTime))
        throw Error(DNNI_E_INVAL, "timeRadius and curTime must be whole, timeRadius >= 0");
    const int rt = (int)timeRadius, cur = (int)curTime;
    const int numRB = useDelta ? 2 * rt + 1 : 1;
    const int po = default_pixel_offset(st.s);
    const long long key[3] = {(long long)wp.ncols + 2 * po, (long long)wp.nrows + 2 * po, numRB};
    if (key[0] != st.rb_key[0] || key[1] != st.rb_key[1] || key[2] != st.rb_key[2]) {
        st.rb_times.assign((size_t)numRB, -1);        // new renderbuffers (nni.cpp:381-410)
        st.st_points.clear();
        for (int k = 0; k < 3; ++k) st.rb_key[k] = key[k];
    }
    TPIE_OS_OFFSET finalSeekTo = vec.tell();
    bool firstSeek = true;
    Point4D* pp;
    for (int j = -rt; j <= rt; j++) {
        const float t = curTime + j;
        bool found = false;
        if (useDelta) {
            for (int v : st.rb_times) found = found || v == (int)t;
            if (!found) {
                size_t mi = 0;
                for (size_t k = 1; k < st.rb_times.size(); ++k)
                    if (st.rb_times[k] < st.rb_times[mi]) mi = k;
                st.rb_times[mi] = (int)t;
            }
        }
        if (useDelta && found) continue;
        TPIE_OS_OFFSET seekto = vec.tell();
        bool foundSeek = false;
        while (vec.read_item(&pp) == tpie::ami::NO_ERROR) {
            const Point4D& p = *pp;
            const TPIE_OS_OFFSET at = vec.tell() - 1;
            if (!foundSeek && p.t >= t + 1 - timeRadius) {
                seekto = at;
                foundSeek = true;
                if (firstSeek) {
                    firstSeek = false;
                    finalSeekTo = at;
                }
            }
            if (std::fabs(t - p.t) <= timeRadius + 0.000001) st.st_points[(long long)at] = p;
            else if (p.t > t + timeRadius) break;
        }
        if (!useDelta && j + 1 > timeRadius) vec.seek(finalSeekTo);
        else vec.seek(seekto);
    }
    st.xyz.clear();
    st.times.clear();
    for (const auto& kv : st.st_points) {
        const Point4D& p = kv.second;
        if (std::abs((long long)p.t - cur) > 2LL * rt) continue;
        const double X = std::llround((p.p[0] - wp.origin_x) / st.xy_scale);
        const double Y = std::llround((p.p[1] - wp.origin_y) / st.xy_scale);
        const double Z = std::llround(p.p[2] / st.z_scale);
        if (std::fabs(X) >= 1073741824.0 || std::fabs(Y) >= 1073741824.0 || std::fabs(Z) >= 1073741824.0)
            throw Error(DNNI_E_RANGE, "point beyond +-2^30 LAS units of the work-package origin");
        st.xyz.push_back((int32_t)X);
        st.xyz.push_back((int32_t)Y);
        st.xyz.push_back((int32_t)Z);
        st.times.push_back(p.t);
    }
    dnni_workpackage d = to_dnni(wp, -1);
    dnni_st_options o{};
    o.cur_time = cur;
    o.time_radius = rt;
    o.time_scale = (int32_t)std::llround(st.time_scale / st.xy_scale);
    st.h.resize((size_t)wp.ncols * wp.nrows);
    dnni_stats stats{};
    const int64_t n = (int64_t)st.times.size();
    check(dnni_interpolate_spacetime(st.ctx, &d, &o, n ? st.xyz.data() : nullptr, n ? st.times.data() : nullptr, n,
                                     st.h.data(), &stats),
          "performNNI");
    st.ms_engine += stats.ms_total;
    st.calls++;
    emit_outpoints(wp, out);
}
}  // namespace detail

/* nni.cpp:870-944.  Reads the points of time slice curTime from `vec` at its
 * current position (2-D: the reference's renderInputPoints loop,
 * nni.cpp:750-788, including where it leaves the stream), interpolates the
 * work package on the GPU and appends one OutPoint per cell of the global
 * grid in the reference's order (nni.cpp:836-858). */
inline void performNNI(const WorkPackage& wp, tpie::ami::stream<OutPoint>& out, tpie::ami::stream<Point4D>& vec,
                       float timeRadius, float curTime, bool useDelta, bool debug = false) {
    (void)debug;
    detail::State& st = detail::state();
    if (!st.ctx) throw Error(DNNI_E_STATE, "performNNI before init");
    if (timeRadius != 0.0f) {
        detail::performNNISpaceTime(wp, out, vec, timeRadius, curTime, useDelta);
        return;
    }
    const float t = curTime;
    TPIE_OS_OFFSET seekto = vec.tell(), finalSeekTo = vec.tell();
    bool foundSeek = false;
    st.xyz.clear();
    st.gid.clear();
    st.world.clear();
    Point4D* pp;
    uint32_t order = 0;
    while (vec.read_item(&pp) == tpie::ami::NO_ERROR) {
        const Point4D& p = *pp;
        if (!foundSeek && p.t >= t + 1 - timeRadius) {
            seekto = vec.tell() - 1;
            finalSeekTo = seekto;
            foundSeek = true;
        }
        if (std::fabs(t - p.t) <= timeRadius + 0.000001 && st.compat) {
            st.world.insert(st.world.end(), p.p, p.p + 3);
        } else if (std::fabs(t - p.t) <= timeRadius + 0.000001) {
            const double X = std::llround((p.p[0] - wp.origin_x) / st.xy_scale);
            const double Y = std::llround((p.p[1] - wp.origin_y) / st.xy_scale);
            const double Z = std::llround(p.p[2] / st.z_scale);
            if (std::fabs(X) >= 1073741824.0 || std::fabs(Y) >= 1073741824.0 || std::fabs(Z) >= 1073741824.0)
                throw Error(DNNI_E_RANGE, "point beyond +-2^30 LAS units of the work-package origin");
            st.xyz.push_back((int32_t)X);
            st.xyz.push_back((int32_t)Y);
            st.xyz.push_back((int32_t)Z);
            st.gid.push_back(order);
        } else if (p.t > t + timeRadius) {
            break;
        }
        ++order;
    }
    if (!useDelta) vec.seek(finalSeekTo);
    else vec.seek(seekto);

    st.h.resize((size_t)wp.ncols * wp.nrows);
    if (st.compat) {
        dnni_compat_settings cs{};
        cs.scale = st.s.scale;
        cs.cell_size = st.s.cell_size;
        cs.site_radius = st.s.site_radius;
        cs.query_radius = st.s.query_radius;
        cs.point_min = st.s.pointMin;
        cs.multiplier = st.s.multiplier;
        cs.total_ncols = st.s.ncols;
        cs.total_nrows = st.s.nrows;
        const dnni_compat_wp cw{wp.origin_x, wp.origin_y, wp.grid_origin_x, wp.grid_origin_y, wp.nrows, wp.ncols};
        const int64_t n = (int64_t)st.world.size() / 3;
        detail::check(dnni_interpolate_compat(st.ctx, &cs, &cw, n ? st.world.data() : nullptr, n, st.h.data(),
                                              nullptr),
                      "performNNI");
    } else {
        dnni_workpackage d = detail::to_dnni(wp, -1);
        dnni_stats stats{};
        const int64_t n = (int64_t)st.gid.size();
        detail::check(dnni_interpolate_segment(st.ctx, &d, n ? st.xyz.data() : nullptr, n ? st.gid.data() : nullptr,
                                               n, st.h.data(), nullptr, &stats),
                      "performNNI");
        st.ms_engine += stats.ms_total;
    }
    st.calls++;
    detail::emit_outpoints(wp, out);
}

/* nni.cpp:362-379 cleared the renderbuffers between work packages.  The
 * engine keeps no per-package device state (each call starts from cleared
 * scratch), so this only forgets the space-time slices read so far; the
 * scratch stays allocated for the next work package and is released by
 * cleanup(). */
inline void clearRenderbuffers() {
    detail::State& st = detail::state();
    std::fill(st.rb_times.begin(), st.rb_times.end(), -1);
    st.st_points.clear();
}

}  // namespace nni

#endif
