// Host side of DRAGONHOARD output from device buffers: a writer and a reader
// for the subset of the HDF5 file format that DRAGONHOARD's files use
// (DRAGONHOARD/HDF5Output.cpp:41-97, HDF5Restart.cpp:21-49).
//
// HDF5 itself is not a dependency: the files are laid out from the public
// HDF5 File Format Specification (version 3.0) the way the HDF5 library
// lays them out by default (superblock version 0, version-1 object headers,
// symbol-table groups, chunked datasets indexed by a version-1 B-tree, the
// deflate filter from zlib), so h5py / h5dump / DRAGONGAZE read them.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace hoard {

enum ElemType { kF64 = 0, kF32 = 1, kI32 = 2 };

// One dataset: its absolute path ("/fluid/v/x"), its dimensions slowest
// first (the HDF5 order: {nz, ny, nx}) and its data, row-major.
struct Dataset {
    std::string path;
    int rank = 1;
    uint64_t dims[3] = {0, 0, 0};
    int type = kF64;
    const void* data = nullptr;
};

// A scalar attribute of the root group (HDF5Output.cpp:91-95).
struct Attr {
    std::string name;
    int type = kI32;  // kI32 or kF64
    int32_t i = 0;
    double d = 0.0;
};

// Writes `path`. level > 0: chunked datasets (chunk edge min(dim, 1024) in
// 1D, min(dim, 32) in 2D, min(dim, 16) in 3D, HDF5Output.cpp:50-87) with
// deflate at that level, compressed by `threads` host threads (0: all cores);
// level <= 0: contiguous, uncompressed. Groups are created for every parent
// path of a dataset. Returns 0, or -1 with *err set.
int write_file(const std::string& path, const std::vector<Attr>& attrs, const std::vector<Dataset>& dsets, int level,
               int threads, std::string* err);

// Reader: opens a whole file in memory.
class File {
public:
    // Returns false with *err set when the file is unreadable or outside the
    // supported subset.
    bool open(const std::string& path, std::string* err);
    bool attr(const std::string& name, double* value, std::string* err) const;
    bool has(const std::string& path) const;
    // Dimensions slowest first; rank 0 for a scalar.
    bool shape(const std::string& path, std::vector<uint64_t>* dims, std::string* err) const;
    // Converts the dataset's elements to double, row-major.
    bool read(const std::string& path, std::vector<double>* out, std::string* err) const;

private:
    struct Msg {
        int type;
        size_t body;
        size_t size;
    };
    std::vector<uint8_t> d_;
    uint64_t base_ = 0;
    uint64_t root_ = 0;
    bool header(uint64_t addr, std::vector<Msg>* msgs, std::string* err) const;
    bool lookup(const std::string& path, uint64_t* addr, std::string* err) const;
    bool links(const std::vector<Msg>& msgs, std::vector<std::pair<std::string, uint64_t>>* out,
               std::string* err) const;
    bool group_btree(uint64_t addr, const std::vector<uint8_t>& heap, std::vector<std::pair<std::string, uint64_t>>* out,
                     int depth, std::string* err) const;
    bool heap(uint64_t addr, std::vector<uint8_t>* out, std::string* err) const;
    bool chunk_btree(uint64_t addr, int rank1, const std::vector<uint32_t>& chunk, const std::vector<uint64_t>& dims,
                     int esize, int cls, bool sgn, bool be, const std::vector<std::pair<int, std::vector<uint32_t>>>& filters,
                     std::vector<double>* out, int depth, std::string* err) const;
    bool in_file(uint64_t off, uint64_t n) const { return off <= d_.size() && n <= d_.size() - off; }
};

}  // namespace hoard
