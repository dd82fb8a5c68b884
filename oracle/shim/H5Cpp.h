/* oracle/shim/H5Cpp.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A project-written stand-in for the subset of the HDF5 C++ API that the
 * reference's src/bubble.cpp uses in OutField (bubble.cpp:919-953), so that
 * the reference compiles unmodified where it lies: libhdf5 is not installed in
 * this image. Nothing is written in HDF5 format. Instead the "file" at `path`
 * becomes a text manifest and each dataset a raw payload next to it:
 *
 *   <path>              lines "dataset <name> <rank> <dim0> [<dim1> [<dim2>]]"
 *                       and   "attr <name> <value printed with %.17g>"
 *   <path>.<name>.f32   the dataset's float32 values, native byte order
 *
 * Chunking, shuffle and deflate settings are accepted and ignored (they do not
 * change the stored values). This is enough to compare snapshot payloads and
 * attributes bit for bit.
 */
#ifndef CB_SHIM_H5CPP_H
#define CB_SHIM_H5CPP_H

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

typedef unsigned long long hsize_t;
#define H5F_ACC_TRUNC 2u
enum { H5S_SCALAR = 0 };

namespace H5 {

class Exception {
  public:
    void printErrorStack() const { std::fprintf(stderr, "H5 shim: write error\n"); }
};

class PredType {
  public:
    explicit PredType(int bytes) : bytes_(bytes) {}
    int bytes() const { return bytes_; }
    static const PredType NATIVE_FLOAT;
    static const PredType NATIVE_DOUBLE;
  private:
    int bytes_;
};
inline const PredType PredType::NATIVE_FLOAT(4);
inline const PredType PredType::NATIVE_DOUBLE(8);

class DataSpace {
  public:
    DataSpace(int rank, const hsize_t *dims) : dims_(dims, dims + rank) {}
    explicit DataSpace(int /*H5S_SCALAR*/) {}
    size_t count() const {
        size_t c = 1;
        for (hsize_t d : dims_) c *= (size_t)d;
        return c;
    }
    const std::vector<hsize_t> &dims() const { return dims_; }
  private:
    std::vector<hsize_t> dims_;
};

class DSetCreatPropList {
  public:
    void setChunk(int, const hsize_t *) {}
    void setShuffle() {}
    void setDeflate(int) {}
};

class DataSet {
  public:
    DataSet(std::string payload, size_t count) : payload_(std::move(payload)), count_(count) {}
    void write(const void *buf, const PredType &type) const {
        FILE *f = std::fopen(payload_.c_str(), "wb");
        if (!f) throw Exception();
        size_t nb = count_ * (size_t)type.bytes();
        if (std::fwrite(buf, 1, nb, f) != nb) { std::fclose(f); throw Exception(); }
        std::fclose(f);
    }
  private:
    std::string payload_;
    size_t count_;
};

class Attribute {
  public:
    Attribute(std::string manifest, std::string name) : manifest_(std::move(manifest)), name_(std::move(name)) {}
    void write(const PredType &type, const void *buf) const {
        FILE *f = std::fopen(manifest_.c_str(), "a");
        if (!f) throw Exception();
        double v = type.bytes() == 8 ? *static_cast<const double *>(buf) : *static_cast<const float *>(buf);
        std::fprintf(f, "attr %s %.17g\n", name_.c_str(), v);
        std::fclose(f);
    }
  private:
    std::string manifest_, name_;
};

class H5File {
  public:
    H5File(const char *path, unsigned /*flags*/) : path_(path) {
        FILE *f = std::fopen(path, "w");
        if (!f) throw Exception();
        std::fclose(f);
    }
    DataSet createDataSet(const std::string &name, const PredType &, const DataSpace &space,
                          const DSetCreatPropList &) const {
        FILE *f = std::fopen(path_.c_str(), "a");
        if (!f) throw Exception();
        std::fprintf(f, "dataset %s %zu", name.c_str(), space.dims().size());
        for (hsize_t d : space.dims()) std::fprintf(f, " %llu", d);
        std::fprintf(f, "\n");
        std::fclose(f);
        return DataSet(path_ + "." + name + ".f32", space.count());
    }
    Attribute createAttribute(const std::string &name, const PredType &, const DataSpace &) const {
        return Attribute(path_, name);
    }
  private:
    std::string path_;
};

}  // namespace H5

#endif
