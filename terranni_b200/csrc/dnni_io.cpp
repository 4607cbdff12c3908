// dnni_io.cpp -- host-side input and output around the interpolation:
// LAS point files in (the reference's nni_io::las_reader, las_reader.inl:
// 54-70, via libLAS) and grids out (the reference's ESRI ASCII writer
// outputASC, terranni.cpp:428-488, plus a raw binary form).  Plain C++ with
// std::thread; part of libdnni.so.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dnni.h"
#include "../../include/nni_io/las.h"

namespace {

int thread_count(int32_t want) {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    return want > 0 ? std::min<int>(want, 256) : std::min(hw, 64);
}

struct File {
    std::FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

}  // namespace

extern "C" {

dnni_status dnni_las_read_header(const char* path, dnni_las_header* out) {
    if (!path || !out) return DNNI_E_INVAL;
    File fh(path, "rb");
    if (!fh.f) return DNNI_E_IO;
    nni_io::LasHeader h;
    if (!nni_io::las_read_header(fh.f, h, nullptr)) return DNNI_E_IO;
    memset(out, 0, sizeof(*out));
    out->version_major = h.version_major;
    out->version_minor = h.version_minor;
    out->point_format = h.point_format;
    out->record_length = h.record_length;
    out->n_points = h.n_points;
    out->offset_to_points = h.offset_to_points;
    for (int k = 0; k < 3; ++k) {
        out->scale[k] = h.scale[k];
        out->offset[k] = h.offset[k];
        out->min[k] = h.min[k];
        out->max[k] = h.max[k];
    }
    return DNNI_OK;
}

dnni_status dnni_las_read(const char* path, int64_t first, int64_t count, int32_t* xyz, uint16_t* intensity,
                          int32_t nthreads) {
    if (!path || first < 0 || count < 0 || (count > 0 && !xyz)) return DNNI_E_INVAL;
    nni_io::LasHeader h;
    {
        File fh(path, "rb");
        if (!fh.f) return DNNI_E_IO;
        if (!nni_io::las_read_header(fh.f, h, nullptr)) return DNNI_E_IO;
    }
    if ((uint64_t)(first + count) > h.n_points) return DNNI_E_INVAL;
    if (count == 0) return DNNI_OK;
    const int nt = (int)std::min<int64_t>(thread_count(nthreads), std::max<int64_t>(1, count / 65536));
    std::vector<int> status(nt, DNNI_OK);
    auto work = [&](int t) {
        const int64_t a = first + count * t / nt, b = first + count * (t + 1) / nt;
        File fh(path, "rb");
        if (!fh.f) { status[t] = DNNI_E_IO; return; }
        const size_t L = h.record_length;
        const int64_t kBlock = 1 << 16;
        std::vector<unsigned char> buf((size_t)kBlock * L);
        for (int64_t i = a; i < b; i += kBlock) {
            const int64_t m = std::min(kBlock, b - i);
            const long long off = (long long)h.offset_to_points + (long long)i * (long long)L;
            if (fseeko(fh.f, (off_t)off, SEEK_SET) != 0 || std::fread(buf.data(), L, (size_t)m, fh.f) != (size_t)m) {
                status[t] = DNNI_E_IO;
                return;
            }
            for (int64_t k = 0; k < m; ++k) {
                const unsigned char* r = buf.data() + (size_t)k * L;
                int32_t* o = xyz + 3 * (i - first + k);
                std::memcpy(o, r, 12);             // X, Y, Z record integers
                if (intensity) std::memcpy(&intensity[i - first + k], r + 12, 2);
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
    for (int s : status)
        if (s) return (dnni_status)s;
    return DNNI_OK;
}

dnni_status dnni_las_write(const char* path, const int32_t* xyz, const uint16_t* intensity, int64_t n,
                           const double* scale, const double* offset) {
    if (!path || n < 0 || (n > 0 && !xyz) || n > 0xFFFFFFFFll) return DNNI_E_INVAL;
    nni_io::LasHeader h;
    h.n_points = (uint64_t)n;
    int32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        if (scale) h.scale[k] = scale[k];
        if (offset) h.offset[k] = offset[k];
        if (h.scale[k] == 0) return DNNI_E_INVAL;
        if (n > 0) lo[k] = hi[k] = xyz[k];
    }
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], xyz[3 * i + k]);
            hi[k] = std::max(hi[k], xyz[3 * i + k]);
        }
    for (int k = 0; k < 3; ++k) {
        h.min[k] = lo[k] * h.scale[k] + h.offset[k];
        h.max[k] = hi[k] * h.scale[k] + h.offset[k];
    }
    unsigned char hb[227];
    nni_io::las_fill_header_12(hb, h);
    File fh(path, "wb");
    if (!fh.f) return DNNI_E_IO;
    if (std::fwrite(hb, 1, sizeof(hb), fh.f) != sizeof(hb)) return DNNI_E_IO;
    const int64_t kBlock = 1 << 16;
    std::vector<unsigned char> buf((size_t)kBlock * 20);
    for (int64_t i = 0; i < n; i += kBlock) {
        const int64_t m = std::min(kBlock, n - i);
        std::memset(buf.data(), 0, (size_t)m * 20);
        for (int64_t k = 0; k < m; ++k) {
            unsigned char* r = buf.data() + (size_t)k * 20;
            std::memcpy(r, xyz + 3 * (i + k), 12);
            if (intensity) std::memcpy(r + 12, &intensity[i + k], 2);
            r[14] = 0x09;   // return 1 of 1
        }
        if (std::fwrite(buf.data(), 20, (size_t)m, fh.f) != (size_t)m) return DNNI_E_IO;
    }
    return DNNI_OK;
}

dnni_status dnni_write_asc(const char* path, const float* h, int32_t ncols, int32_t nrows, double xll, double yll,
                           double cellsize, float nodata, int32_t nthreads) {
    if (!path || !h || ncols <= 0 || nrows <= 0) return DNNI_E_INVAL;
    File fh(path, "w");
    if (!fh.f) return DNNI_E_IO;
    // header lines and row order as outputASC writes them; values are printed
    // like a C++ stream's default float output (6 significant digits), each
    // followed by a space, one line per grid row from the top (north) row
    std::fprintf(fh.f, "NROWS %d\nNCOLS %d\nXLLCORNER %.10g\nYLLCORNER %.10g\nCELLSIZE %.10g\nNODATA_VALUE %g\n", nrows,
                 ncols, xll, yll, cellsize, (double)nodata);
    const int nt = thread_count(nthreads);
    const int kRows = 64;
    std::vector<std::string> out(nt);
    for (int r0 = 0; r0 < nrows; r0 += kRows * nt) {
        auto work = [&](int t) {
            std::string& s = out[t];
            s.clear();
            char tmp[32];
            const int a = r0 + t * kRows, b = std::min(nrows, a + kRows);
            for (int q = a; q < b; ++q) {
                const float* row = h + (size_t)(nrows - 1 - q) * ncols;
                for (int i = 0; i < ncols; ++i) {
                    const int len = std::snprintf(tmp, sizeof(tmp), "%g ", (double)row[i]);
                    s.append(tmp, (size_t)len);
                }
                s.push_back('\n');
            }
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
        work(0);
        for (auto& x : th) x.join();
        for (int t = 0; t < nt; ++t)
            if (!out[t].empty() && std::fwrite(out[t].data(), 1, out[t].size(), fh.f) != out[t].size()) return DNNI_E_IO;
    }
    return DNNI_OK;
}

dnni_status dnni_write_grid_bin(const char* path, const float* h, int32_t ncols, int32_t nrows, double xll,
                                double yll, double cellsize, float nodata) {
    if (!path || !h || ncols <= 0 || nrows <= 0) return DNNI_E_INVAL;
    File fh(path, "wb");
    if (!fh.f) return DNNI_E_IO;
    unsigned char hd[64];
    std::memset(hd, 0, sizeof(hd));
    std::memcpy(hd, "DNNIGRD1", 8);
    std::memcpy(hd + 8, &ncols, 4);
    std::memcpy(hd + 12, &nrows, 4);
    std::memcpy(hd + 16, &xll, 8);
    std::memcpy(hd + 24, &yll, 8);
    std::memcpy(hd + 32, &cellsize, 8);
    std::memcpy(hd + 40, &nodata, 4);
    if (std::fwrite(hd, 1, sizeof(hd), fh.f) != sizeof(hd)) return DNNI_E_IO;
    const size_t cells = (size_t)ncols * nrows;
    if (std::fwrite(h, sizeof(float), cells, fh.f) != cells) return DNNI_E_IO;
    return DNNI_OK;
}

}  // extern "C"
