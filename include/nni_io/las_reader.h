/*
 * nni_io/las_reader.h -- drop-in for TerraNNI's nni_io::las_reader
 * (las_reader.h:34-58, las_reader.inl:25-84) without libLAS: the public LAS
 * layout read directly (nni_io/las.h), buffered.  Each point is handed out
 * as P(x, y, z, intensity) with coordinates = record integer * scale +
 * offset, as liblas::Point::GetX/GetY/GetZ return them, and the intensity as
 * the fourth argument, as las_reader.inl:64 passes it.  No point is skipped
 * (the reference's ignore() never skips either).
 *
 * Difference: get_header() returns nni_io::LasHeader (scale, offset, bounds,
 * count, format) instead of liblas::Header.  Errors on open throw
 * std::runtime_error, as the reference does.
 */
#ifndef DNNI_NNI_IO_LAS_READER_H
#define DNNI_NNI_IO_LAS_READER_H

#include <algorithm>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "las.h"
#include "point_reader.h"

namespace nni_io {

template <typename P, typename Z>
class las_reader : public point_reader<P, Z> {
public:
    virtual ~las_reader() { this->close(); }

    const LasHeader& get_header() const { return head; }

protected:
    virtual void do_open(const std::string& filename) {
        f = std::fopen(filename.c_str(), "rb");
        if (!f) throw std::runtime_error("Could not open file " + filename);
        std::string err;
        if (!las_read_header(f, head, &err)) {
            std::fclose(f);
            f = nullptr;
            throw std::runtime_error("Could not open file " + filename + ": " + err);
        }
        do_reset();
    }
    virtual void do_close() {
        if (f) std::fclose(f);
        f = nullptr;
    }
    virtual void do_reset() {
        next = 0;
        have = used = 0;
        if (f) std::fseek(f, (long)head.offset_to_points, SEEK_SET);
    }
    virtual bool get_next_point(P& point) {
        if (!f || next >= head.n_points) return false;
        if (used == have) {
            const uint64_t want = std::min<uint64_t>(kBlock, head.n_points - next);
            buf.resize((size_t)kBlock * head.record_length);
            have = std::fread(buf.data(), head.record_length, (size_t)want, f);
            used = 0;
            if (have == 0) return false;
        }
        const unsigned char* r = buf.data() + used * head.record_length;
        const int32_t X = las_detail::get<int32_t>(r), Y = las_detail::get<int32_t>(r + 4);
        const int32_t Zr = las_detail::get<int32_t>(r + 8);
        const uint16_t I = las_detail::get<uint16_t>(r + 12);
        point = P(X * head.scale[0] + head.offset[0], Y * head.scale[1] + head.offset[1],
                  Zr * head.scale[2] + head.offset[2], (int)I);
        ++used;
        ++next;
        return true;
    }

private:
    static const size_t kBlock = 1 << 14;
    std::FILE* f = nullptr;
    LasHeader head;
    std::vector<unsigned char> buf;
    size_t have = 0, used = 0;
    uint64_t next = 0;
};

}  // namespace nni_io

#endif
