/*
 * nni_io/las.h -- the public ASPRS LAS file layout (versions 1.0 to 1.4,
 * point data record formats 0 to 10), header-only.
 *
 * The reference reads LAS through libLAS 1.6 (las_reader.inl:54-70:
 * liblas::Reader, Point::GetX/GetY/GetZ = record integer * scale + offset,
 * GetIntensity), which is not available here; this restates the published
 * format instead.  Only what the interpolation needs is decoded: the header's
 * scale, offset, bounds, point count and record layout, and from each point
 * record the int32 X, Y, Z, the uint16 intensity and the classification.
 * Compressed (LAZ) files are refused.
 */
#ifndef DNNI_NNI_IO_LAS_H
#define DNNI_NNI_IO_LAS_H

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

namespace nni_io {

struct LasHeader {
    uint8_t version_major = 1, version_minor = 2;
    uint8_t point_format = 0;
    uint16_t header_size = 227;
    uint16_t record_length = 20;
    uint32_t offset_to_points = 227;
    uint64_t n_points = 0;
    double scale[3] = {0.01, 0.01, 0.01};
    double offset[3] = {0, 0, 0};
    double min[3] = {0, 0, 0}, max[3] = {0, 0, 0};
};

namespace las_detail {
template <typename T>
inline T get(const unsigned char* p) {
    T v;
    std::memcpy(&v, p, sizeof(T));   // the format is little-endian, as is every host this builds for
    return v;
}
template <typename T>
inline void put(unsigned char* p, T v) {
    std::memcpy(p, &v, sizeof(T));
}
}  // namespace las_detail

// Decodes the public header block; false with *err set when the file is not
// an uncompressed LAS file this reader understands.
inline bool las_parse_header(const unsigned char* b, size_t len, LasHeader& h, std::string* err) {
    using las_detail::get;
    auto fail = [&](const char* m) {
        if (err) *err = m;
        return false;
    };
    if (len < 227 || std::memcmp(b, "LASF", 4) != 0) return fail("not a LAS file (no LASF signature)");
    h.version_major = b[24];
    h.version_minor = b[25];
    if (h.version_major != 1 || h.version_minor > 4) return fail("unsupported LAS version");
    h.header_size = get<uint16_t>(b + 94);
    h.offset_to_points = get<uint32_t>(b + 96);
    const uint8_t fmt = b[104];
    if (fmt & 0xC0) return fail("compressed (LAZ) point data is not supported");
    h.point_format = fmt & 0x3F;
    if (h.point_format > 10) return fail("unsupported point data record format");
    h.record_length = get<uint16_t>(b + 105);
    static const uint16_t kMinLen[11] = {20, 28, 26, 34, 57, 63, 30, 36, 38, 59, 67};
    if (h.record_length < kMinLen[h.point_format]) return fail("point record shorter than its format");
    uint64_t n = get<uint32_t>(b + 107);
    if (h.version_minor >= 4) {
        if (len < 255) return fail("truncated LAS 1.4 header");
        const uint64_t n64 = get<uint64_t>(b + 247);
        if (n == 0 || n64 > n) n = n64;
    }
    h.n_points = n;
    for (int k = 0; k < 3; ++k) {
        h.scale[k] = get<double>(b + 131 + 8 * k);
        h.offset[k] = get<double>(b + 155 + 8 * k);
        h.max[k] = get<double>(b + 179 + 16 * k);
        h.min[k] = get<double>(b + 187 + 16 * k);
    }
    if (h.scale[0] == 0 || h.scale[1] == 0 || h.scale[2] == 0) return fail("zero coordinate scale");
    return true;
}

inline bool las_read_header(std::FILE* f, LasHeader& h, std::string* err) {
    unsigned char b[375];
    std::memset(b, 0, sizeof(b));
    if (std::fseek(f, 0, SEEK_SET) != 0) {
        if (err) *err = "seek failed";
        return false;
    }
    const size_t got = std::fread(b, 1, sizeof(b), f);
    return las_parse_header(b, got, h, err);
}

// Field offsets inside a point record.
inline int las_classification_offset(uint8_t format) { return format >= 6 ? 16 : 15; }

// A LAS 1.2 header for point format 0 (20-byte records) with the given
// transform; bounds from the caller.
inline void las_fill_header_12(unsigned char* b, const LasHeader& h) {
    using las_detail::put;
    std::memset(b, 0, 227);
    std::memcpy(b, "LASF", 4);
    b[24] = 1;
    b[25] = 2;
    std::memcpy(b + 26, "terranni_b200", 13);
    std::memcpy(b + 58, "dnni_las_write", 14);
    put<uint16_t>(b + 94, 227);
    put<uint32_t>(b + 96, 227);
    put<uint32_t>(b + 100, 0);
    b[104] = 0;
    put<uint16_t>(b + 105, 20);
    put<uint32_t>(b + 107, (uint32_t)h.n_points);
    put<uint32_t>(b + 111, (uint32_t)h.n_points);
    for (int k = 0; k < 3; ++k) {
        put<double>(b + 131 + 8 * k, h.scale[k]);
        put<double>(b + 155 + 8 * k, h.offset[k]);
        put<double>(b + 179 + 16 * k, h.max[k]);
        put<double>(b + 187 + 16 * k, h.min[k]);
    }
}

}  // namespace nni_io

#endif
