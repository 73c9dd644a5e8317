// datafile.cpp — reader and writer of the named-dataset files (datafile.hpp).
#include "datafile.hpp"

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cstring>
#include <fstream>

namespace fopis {
namespace host {

namespace {

constexpr char kMagic[8] = {'F', 'O', 'P', 'I', 'S', 'D', 'S', '1'};

// File checksum: the bytes, zero-padded to whole 8-byte little-endian words
// w_i, give sum_i w_i (2i + 1) + byte count, modulo 2^64. A flipped bit in
// word i moves the sum by 2^k (2i + 1), never 0 modulo 2^64; a truncation
// changes the count.
uint64_t checksum(const std::vector<uint8_t>& b) {
    uint64_t h = (uint64_t)b.size();
    const size_t nw = (b.size() + 7) / 8;
    for (size_t i = 0; i < nw; ++i) {
        uint64_t w = 0;
        const size_t n = std::min<size_t>(8, b.size() - 8 * i);
        std::memcpy(&w, b.data() + 8 * i, n);
        h += w * (2 * (uint64_t)i + 1);
    }
    return h;
}

template <typename T>
void append(std::vector<uint8_t>& out, T v) {
    uint8_t buf[sizeof(T)];
    std::memcpy(buf, &v, sizeof(T));          // little-endian hosts (x86-64, aarch64)
    out.insert(out.end(), buf, buf + sizeof(T));
}

struct Cursor {
    const std::vector<uint8_t>& b;
    size_t pos;
    size_t end;
    template <typename T>
    T take() {
        if (end - pos < sizeof(T)) throw std::runtime_error("corrupt data file: truncated");
        T v;
        std::memcpy(&v, b.data() + pos, sizeof(T));
        pos += sizeof(T);
        return v;
    }
    void bytes(void* dst, size_t n) {
        if (end - pos < n) throw std::runtime_error("corrupt data file: truncated");
        std::memcpy(dst, b.data() + pos, n);
        pos += n;
    }
};

size_t elem_size(DataFile::Type) { return 8; }

}  // namespace

uint64_t DataFile::Entry::count() const {
    uint64_t n = 1;
    for (uint64_t d : dims) n *= d;
    return n;
}

void DataFile::put(const std::string& name, Type t, const std::vector<uint64_t>& dims, const void* data, size_t elem) {
    if (name.empty() || name.size() > 65535) throw std::invalid_argument("dataset name length");
    Entry e;
    e.type = t;
    e.dims = dims;
    e.bytes.resize((size_t)e.count() * elem);
    if (!e.bytes.empty()) std::memcpy(e.bytes.data(), data, e.bytes.size());
    sets_[name] = std::move(e);
}

void DataFile::put_f64(const std::string& name, const std::vector<uint64_t>& dims, const double* data) {
    put(name, F64, dims, data, sizeof(double));
}
void DataFile::put_i64(const std::string& name, const std::vector<uint64_t>& dims, const int64_t* data) {
    put(name, I64, dims, data, sizeof(int64_t));
}

const DataFile::Entry& DataFile::get(const std::string& name) const {
    auto it = sets_.find(name);
    if (it == sets_.end()) throw std::runtime_error("dataset " + name + " does not exist in the file");
    return it->second;
}

std::vector<double> DataFile::f64(const std::string& name) const {
    const Entry& e = get(name);
    if (e.type != F64) throw std::runtime_error("dataset " + name + " is not float64");
    std::vector<double> v(e.count());
    if (!v.empty()) std::memcpy(v.data(), e.bytes.data(), e.bytes.size());
    return v;
}
double DataFile::f64_scalar(const std::string& name) const {
    const std::vector<double> v = f64(name);
    if (v.size() != 1) throw std::runtime_error("dataset " + name + " is not a scalar");
    return v[0];
}
std::vector<int64_t> DataFile::i64(const std::string& name) const {
    const Entry& e = get(name);
    if (e.type != I64) throw std::runtime_error("dataset " + name + " is not int64");
    std::vector<int64_t> v(e.count());
    if (!v.empty()) std::memcpy(v.data(), e.bytes.data(), e.bytes.size());
    return v;
}
int64_t DataFile::i64_scalar(const std::string& name) const {
    const std::vector<int64_t> v = i64(name);
    if (v.size() != 1) throw std::runtime_error("dataset " + name + " is not a scalar");
    return v[0];
}
std::vector<std::string> DataFile::names() const {
    std::vector<std::string> out;
    for (const auto& kv : sets_) out.push_back(kv.first);
    return out;
}

void DataFile::save(const std::string& path) const {
    std::vector<uint8_t> out(kMagic, kMagic + 8);
    append<uint32_t>(out, (uint32_t)sets_.size());
    for (const auto& kv : sets_) {
        append<uint16_t>(out, (uint16_t)kv.first.size());
        out.insert(out.end(), kv.first.begin(), kv.first.end());
        append<uint8_t>(out, (uint8_t)kv.second.type);
        append<uint8_t>(out, (uint8_t)kv.second.dims.size());
        for (uint64_t d : kv.second.dims) append<uint64_t>(out, d);
        append<uint64_t>(out, (uint64_t)kv.second.bytes.size());
        out.insert(out.end(), kv.second.bytes.begin(), kv.second.bytes.end());
    }
    append<uint64_t>(out, checksum(out));
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    if (!f) throw std::runtime_error("cannot write " + path);
    f.write(reinterpret_cast<const char*>(out.data()), (std::streamsize)out.size());
    if (!f) throw std::runtime_error("cannot write " + path);
}

DataFile DataFile::load(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("file " + path + " does not exist");
    std::vector<uint8_t> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    if (b.size() < 8 + 4 + 8 || std::memcmp(b.data(), kMagic, 8) != 0)
        throw std::runtime_error("corrupt data file " + path + ": bad magic");
    uint64_t stored;
    std::memcpy(&stored, b.data() + b.size() - 8, 8);
    const std::vector<uint8_t> body(b.begin(), b.end() - 8);
    if (checksum(body) != stored) throw std::runtime_error("corrupt data file " + path + ": checksum mismatch");
    Cursor c{b, 8, b.size() - 8};
    DataFile out;
    const uint32_t n = c.take<uint32_t>();
    for (uint32_t i = 0; i < n; ++i) {
        const uint16_t len = c.take<uint16_t>();
        std::string name(len, '\0');
        c.bytes(&name[0], len);
        Entry e;
        const uint8_t t = c.take<uint8_t>();
        if (t != F64 && t != I64) throw std::runtime_error("corrupt data file " + path + ": element type");
        e.type = (Type)t;
        const uint8_t rank = c.take<uint8_t>();
        for (uint8_t r = 0; r < rank; ++r) e.dims.push_back(c.take<uint64_t>());
        const uint64_t nbytes = c.take<uint64_t>();
        if (nbytes > c.end - c.pos || nbytes != e.count() * elem_size(e.type))
            throw std::runtime_error("corrupt data file " + path + ": extents");
        e.bytes.resize((size_t)nbytes);
        c.bytes(e.bytes.data(), (size_t)nbytes);
        out.sets_[name] = std::move(e);
    }
    if (c.pos != c.end) throw std::runtime_error("corrupt data file " + path + ": trailing bytes");
    return out;
}

void make_dirs(const std::string& path) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); ++i) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
                throw std::runtime_error("cannot create directory " + cur);
        }
        if (i < path.size()) cur += path[i];
    }
}

bool file_exists(const std::string& path) {
    struct stat st;
    return stat(path.c_str(), &st) == 0;
}

}  // namespace host
}  // namespace fopis
