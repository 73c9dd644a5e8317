// datafile.hpp — named-dataset files for the resume data and the capacity-
// matrix cache, in place of the reference's HDF5 files (HighFive): the same
// dataset names ("capacity_matrix", "grid_spacing", "Electron/x",
// "Potential/phi", ...) in one little-endian binary file.
//
// Layout: the 8-byte magic "FOPISDS1"; a uint32 dataset count; per dataset a
// uint16 name length and the name, a uint8 element type (1 float64, 2 int64),
// a uint8 rank, rank uint64 extents, a uint64 payload byte count and the
// payload; finally a uint64 checksum of every byte before it (the bytes as
// zero-padded 8-byte words w_i: sum_i w_i (2i + 1) + byte count, modulo 2^64).
// A file whose checksum, magic or lengths do not match is rejected as corrupt.
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace fopis {
namespace host {

class DataFile {
public:
    enum Type : uint8_t { F64 = 1, I64 = 2 };
    struct Entry {
        Type type = F64;
        std::vector<uint64_t> dims;
        std::vector<uint8_t> bytes;
        uint64_t count() const;
    };

    void put_f64(const std::string& name, const std::vector<uint64_t>& dims, const double* data);
    void put_f64(const std::string& name, double v) { put_f64(name, {}, &v); }
    void put_i64(const std::string& name, const std::vector<uint64_t>& dims, const int64_t* data);
    void put_i64(const std::string& name, int64_t v) { put_i64(name, {}, &v); }

    bool has(const std::string& name) const { return sets_.count(name) != 0; }
    const Entry& get(const std::string& name) const;
    std::vector<double> f64(const std::string& name) const;
    double f64_scalar(const std::string& name) const;
    std::vector<int64_t> i64(const std::string& name) const;
    int64_t i64_scalar(const std::string& name) const;
    std::vector<std::string> names() const;

    // Writes the file (directories must exist); throws std::runtime_error on I/O failure.
    void save(const std::string& path) const;
    // Reads a file; throws std::runtime_error when it is missing or corrupt.
    static DataFile load(const std::string& path);

private:
    void put(const std::string& name, Type t, const std::vector<uint64_t>& dims, const void* data, size_t elem);
    std::map<std::string, Entry> sets_;
};

// Creates a directory and its parents (like mkdir -p); no error if it exists.
void make_dirs(const std::string& path);
bool file_exists(const std::string& path);

}  // namespace host
}  // namespace fopis
