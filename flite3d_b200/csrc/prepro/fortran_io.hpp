// Fortran sequential-unformatted record I/O.
//
// Every READ/WRITE statement of the reference on an unformatted unit is one
// record: a 4-byte little-endian length marker, the payload, and the same
// marker again.  Integers are int32 and reals float64 (the reference compiles
// with -r8, SolverSource/makefile:10).  Records larger than 2 GiB (which need
// Fortran sub-records) are rejected: no record of the solver path reaches
// that size for meshes that fit one GPU except the .rst/.res/.unk field
// records above ~53 M nodes, which are written with the sub-record scheme of
// gfortran/ifort (negative continuation markers).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace fio {

struct io_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class Writer {
  public:
    explicit Writer(const char *path) {
        f_ = std::fopen(path, "wb");
        if (!f_) throw io_error(std::string("cannot open for writing: ") + path);
        std::setvbuf(f_, nullptr, _IOFBF, 1 << 22);
    }
    ~Writer() {
        if (f_) std::fclose(f_);
    }
    // a record is assembled in buf_ and flushed by end()
    Writer &i4(int32_t v) { put(&v, 4); return *this; }
    Writer &r8(double v) { put(&v, 8); return *this; }
    Writer &i4s(const int32_t *v, size_t n) { put(v, 4 * n); return *this; }
    Writer &r8s(const double *v, size_t n) { put(v, 8 * n); return *this; }
    void end() {
        const size_t n = buf_.size();
        const size_t kMax = 0x7fffffff - 8;
        if (n <= kMax) {
            int32_t m = (int32_t)n;
            w(&m, 4); w(buf_.data(), n); w(&m, 4);
        } else {
            // sub-record chain: every part but the last carries a negative
            // leading marker; every part but the first a negative trailing one
            size_t off = 0; bool first = true;
            while (off < n) {
                size_t part = std::min(kMax, n - off);
                bool last = off + part == n;
                int32_t lead = last ? (int32_t)part : -(int32_t)part;
                int32_t trail = first ? (int32_t)part : -(int32_t)part;
                w(&lead, 4); w(buf_.data() + off, part); w(&trail, 4);
                off += part; first = false;
            }
        }
        buf_.clear();
    }
    void close() {
        if (f_ && std::fclose(f_) != 0) { f_ = nullptr; throw io_error("close failed"); }
        f_ = nullptr;
    }

  private:
    void put(const void *p, size_t n) {
        const char *c = (const char *)p;
        buf_.insert(buf_.end(), c, c + n);
    }
    void w(const void *p, size_t n) {
        if (std::fwrite(p, 1, n, f_) != n) throw io_error("short write");
    }
    FILE *f_ = nullptr;
    std::vector<char> buf_;
};

class Reader {
  public:
    explicit Reader(const char *path) {
        f_ = std::fopen(path, "rb");
        if (!f_) throw io_error(std::string("cannot open for reading: ") + path);
        std::setvbuf(f_, nullptr, _IOFBF, 1 << 22);
    }
    ~Reader() {
        if (f_) std::fclose(f_);
    }
    // read the next record into the buffer; returns its payload size
    size_t next() {
        rec_.clear(); pos_ = 0;
        bool more = true;
        while (more) {
            int32_t lead = 0, trail = 0;
            if (std::fread(&lead, 4, 1, f_) != 1) throw io_error("unexpected end of file");
            size_t n = (size_t)(lead < 0 ? -(int64_t)lead : lead);
            size_t at = rec_.size();
            rec_.resize(at + n);
            if (n && std::fread(rec_.data() + at, 1, n, f_) != n) throw io_error("truncated record");
            if (std::fread(&trail, 4, 1, f_) != 1) throw io_error("missing trailing record marker");
            if ((trail < 0 ? -(int64_t)trail : trail) != (int64_t)n)
                throw io_error("record markers disagree");
            more = lead < 0;
        }
        return rec_.size();
    }
    int32_t i4() { int32_t v; get(&v, 4); return v; }
    double r8() { double v; get(&v, 8); return v; }
    void i4s(int32_t *v, size_t n) { get(v, 4 * n); }
    void r8s(double *v, size_t n) { get(v, 8 * n); }
    size_t remaining() const { return rec_.size() - pos_; }
    bool at_eof() {
        int c = std::fgetc(f_);
        if (c == EOF) return true;
        std::ungetc(c, f_);
        return false;
    }

  private:
    void get(void *p, size_t n) {
        // a READ may consume a prefix of the record (def_par:843-848 reads
        // only the node number of a (node, normal) record)
        if (pos_ + n > rec_.size()) throw io_error("read past end of record");
        std::memcpy(p, rec_.data() + pos_, n);
        pos_ += n;
    }
    FILE *f_ = nullptr;
    std::vector<char> rec_;
    size_t pos_ = 0;
};

}  // namespace fio
