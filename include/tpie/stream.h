/*
 * tpie/stream.h -- minimal stand-in for TPIE's external-memory stream, for
 * builds of the nni:: boundary without the TPIE library (TerraNNI pulls TPIE
 * as a git submodule, .gitmodules:1-3, which is not present here).
 *
 * Only the subset the NNI hot path and its caller use is provided:
 * read_item / write_item / seek / tell / stream_len (nni.cpp:741-788, 858),
 * truncate / persist and APPEND_STREAM (terranni.cpp:413-417).  Items live in
 * memory; a named stream loads its file (raw item records) on construction
 * and writes it back when destroyed, unless it is a temporary.  With the real
 * TPIE on the include path first, this header is not used.
 */
#ifndef DNNI_TPIE_STREAM_SHIM_H
#define DNNI_TPIE_STREAM_SHIM_H

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

typedef long long TPIE_OS_OFFSET;

namespace tpie {
namespace ami {

enum err { NO_ERROR = 0, IO_ERROR, END_OF_STREAM, READ_ONLY, OS_ERROR };
enum stream_type { READ_STREAM = 1, WRITE_STREAM, APPEND_STREAM, READ_WRITE_STREAM };
enum persistence { PERSIST_DELETE = 0, PERSIST_PERSISTENT };

template <class T>
class stream {
public:
    stream() : pos_(0), persist_(PERSIST_DELETE) {}
    explicit stream(const std::string& path, stream_type t = READ_WRITE_STREAM)
        : path_(path), pos_(0), persist_(PERSIST_PERSISTENT) {
        FILE* f = std::fopen(path.c_str(), "rb");
        if (f) {
            T item;
            while (std::fread(&item, sizeof(T), 1, f) == 1) items_.push_back(item);
            std::fclose(f);
        }
        if (t == APPEND_STREAM) pos_ = (TPIE_OS_OFFSET)items_.size();
    }
    ~stream() {
        if (!path_.empty() && persist_ == PERSIST_PERSISTENT) {
            FILE* f = std::fopen(path_.c_str(), "wb");
            if (f) {
                if (!items_.empty()) std::fwrite(items_.data(), sizeof(T), items_.size(), f);
                std::fclose(f);
            }
        }
    }
    stream(const stream&) = delete;
    stream& operator=(const stream&) = delete;

    err read_item(T** elt) {
        if (pos_ >= (TPIE_OS_OFFSET)items_.size()) return END_OF_STREAM;
        *elt = &items_[(size_t)pos_++];
        return NO_ERROR;
    }
    err write_item(const T& elt) {
        if (pos_ < (TPIE_OS_OFFSET)items_.size()) items_[(size_t)pos_] = elt;
        else items_.push_back(elt);
        ++pos_;
        return NO_ERROR;
    }
    err seek(TPIE_OS_OFFSET off) {
        if (off < 0 || off > (TPIE_OS_OFFSET)items_.size()) return OS_ERROR;
        pos_ = off;
        return NO_ERROR;
    }
    TPIE_OS_OFFSET tell() const { return pos_; }
    TPIE_OS_OFFSET stream_len() const { return (TPIE_OS_OFFSET)items_.size(); }
    err truncate(TPIE_OS_OFFSET off) {
        if (off < 0) return OS_ERROR;
        items_.resize((size_t)off);
        if (pos_ > off) pos_ = off;
        return NO_ERROR;
    }
    void persist(persistence p = PERSIST_PERSISTENT) { persist_ = p; }
    const std::string& name() const { return path_; }

private:
    std::string path_;
    std::vector<T> items_;
    TPIE_OS_OFFSET pos_;
    persistence persist_;
};

}  // namespace ami
}  // namespace tpie

#endif
