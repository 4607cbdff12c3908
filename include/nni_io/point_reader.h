/*
 * nni_io/point_reader.h -- TerraNNI's point source interface
 * (point_reader.h:28-45, point_reader.inl): a reader hands out points P one
 * at a time after open(); reset() starts over.  Same template, names and
 * behaviour (next_point returns false when the reader is closed or the
 * points are exhausted).
 */
#ifndef DNNI_NNI_IO_POINT_READER_H
#define DNNI_NNI_IO_POINT_READER_H

#include <string>

namespace nni_io {

template <typename P, typename Z>
class point_reader {
public:
    point_reader() : is_open(false) {}
    virtual ~point_reader() {}
    bool next_point(P& point) {
        if (!is_open) return false;
        return this->get_next_point(point);
    }
    void open(const std::string& filename) {
        this->close();
        this->do_open(filename);
        is_open = true;
    }
    void close() {
        if (is_open) this->do_close();
        is_open = false;
    }
    void reset() {
        if (is_open) this->do_reset();
    }

protected:
    virtual bool get_next_point(P& point) = 0;
    virtual void do_open(const std::string& filename) = 0;
    virtual void do_close() = 0;
    virtual void do_reset() = 0;
    bool is_open;
};

}  // namespace nni_io

#endif
