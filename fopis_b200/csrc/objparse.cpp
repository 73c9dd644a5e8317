// objparse.cpp — ObjectUtils::getObjectNodesFromObjFile
// (src/Spacecraft/ObjectUtils.cpp:9-333) for the single-rank domain.
//
// A MagicaVoxel .obj lists quads whose four vertices share one coordinate.
// Vertex coordinates are shifted by n/2 per axis (ObjectUtils.cpp:57-59). Every
// grid node on a quad becomes a surface node, numbered in the order quads are
// met and, inside a quad, by the two in-plane axes in increasing order (x quads:
// y then z; y quads: x then z; z quads: x then y) — that numbering is the
// capacity-matrix order. The unit faces of each quad are marked per axis; a cell
// is inside the body when, along each of the three axes, it lies between a pair
// of marked faces found by scanning from the low side (the reference's count of
// 3, ObjectUtils.cpp:178-261). Output indices are glue-layout (+1).
#include <algorithm>
#include <array>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/fopis_gpu.h"

namespace {

struct Dom {
    int n[3];
    size_t at(int i, int j, int k) const { return ((size_t)i * n[1] + j) * n[2] + k; }
    size_t size() const { return (size_t)n[0] * n[1] * n[2]; }
};

bool read_obj(const char* path, int shift[3], std::vector<std::array<int, 3>>& v, std::vector<std::array<int, 4>>& f,
              std::vector<int>* tex = nullptr) {
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) {
        if (line.size() < 2 || line[1] != ' ') continue;
        std::istringstream ss(line.substr(2));
        if (line[0] == 'v') {
            std::array<int, 3> p{};
            for (int a = 0; a < 3; ++a) { ss >> p[a]; p[a] += shift[a]; }
            v.push_back(p);
        } else if (line[0] == 'f') {
            std::array<int, 4> q{};
            int vt = 0;
            for (int t = 0; t < 4; ++t) {
                std::string tok;
                ss >> tok;
                q[t] = std::atoi(tok.c_str());   // stops at the first '/'
                if (t == 0) {
                    const size_t slash = tok.find('/');
                    if (slash != std::string::npos) vt = std::atoi(tok.c_str() + slash + 1);
                }
            }
            f.push_back(q);
            if (tex) tex->push_back(vt);
        }
    }
    return true;
}

}  // namespace

extern "C" int fopis_parse_obj(const char* path, int nx, int ny, int nz, int32_t** cmat_nodes, int* n_cmat,
                               int32_t** cells, int* n_cells) {
    if (!path || !cmat_nodes || !n_cmat || !cells || !n_cells || nx < 2 || ny < 2 || nz < 2) return FOPIS_ERR_ARG;
    Dom d{{nx, ny, nz}};
    int shift[3] = {nx / 2, ny / 2, nz / 2};
    std::vector<std::array<int, 3>> verts;
    std::vector<std::array<int, 4>> faces;
    if (!read_obj(path, shift, verts, faces)) return FOPIS_ERR_ARG;
    std::vector<int32_t> node_id(d.size(), -1);
    std::vector<uint8_t> face[3] = {std::vector<uint8_t>(d.size(), 0), std::vector<uint8_t>(d.size(), 0),
                                    std::vector<uint8_t>(d.size(), 0)};
    std::vector<int32_t> nodes;
    for (const auto& q : faces) {
        std::array<int, 3> p[4];
        for (int t = 0; t < 4; ++t) {
            if (q[t] < 1 || q[t] > (int)verts.size()) return FOPIS_ERR_ARG;
            p[t] = verts[q[t] - 1];
        }
        int normal = -1;
        for (int a = 0; a < 3 && normal < 0; ++a)
            if (p[0][a] == p[1][a] && p[0][a] == p[2][a] && p[0][a] == p[3][a]) normal = a;
        if (normal < 0) return FOPIS_ERR_ARG;   // "Face type cannot be determinted by vertices position."
        const int u = normal == 0 ? 1 : 0, w = normal == 2 ? 1 : 2;
        int lo_u = p[0][u], hi_u = p[0][u], lo_w = p[0][w], hi_w = p[0][w];
        for (int t = 1; t < 4; ++t) {
            lo_u = std::min(lo_u, p[t][u]); hi_u = std::max(hi_u, p[t][u]);
            lo_w = std::min(lo_w, p[t][w]); hi_w = std::max(hi_w, p[t][w]);
        }
        for (int a = lo_u; a <= hi_u; ++a)
            for (int b = lo_w; b <= hi_w; ++b) {
                int c[3];
                c[normal] = p[0][normal]; c[u] = a; c[w] = b;
                if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= nx || c[1] >= ny || c[2] >= nz) return FOPIS_ERR_ARG;
                const size_t id = d.at(c[0], c[1], c[2]);
                if (node_id[id] < 0) {
                    node_id[id] = (int32_t)(nodes.size() / 3);
                    nodes.push_back(c[0] + 1); nodes.push_back(c[1] + 1); nodes.push_back(c[2] + 1);
                }
                if (a < hi_u && b < hi_w) face[normal][id] = 1;
            }
    }
    // per-axis pair scans: cells between a marked face and the next one
    std::vector<uint8_t> hits(d.size(), 0);
    for (int ax = 0; ax < 3; ++ax) {
        const int u = ax == 0 ? 1 : 0, w = ax == 2 ? 1 : 2;
        for (int a = 0; a + 1 < d.n[u]; ++a)
            for (int b = 0; b + 1 < d.n[w]; ++b) {
                int open = -1;
                for (int s = 0; s + 1 < d.n[ax]; ++s) {
                    int c[3];
                    c[ax] = s; c[u] = a; c[w] = b;
                    if (!face[ax][d.at(c[0], c[1], c[2])]) continue;
                    if (open < 0) { open = s; continue; }
                    for (int r = open; r < s; ++r) {
                        int e[3];
                        e[ax] = r; e[u] = a; e[w] = b;
                        hits[d.at(e[0], e[1], e[2])] += 1;
                    }
                    open = -1;
                }
            }
    }
    std::vector<int32_t> inner;
    for (int i = 0; i + 1 < nx; ++i)
        for (int j = 0; j + 1 < ny; ++j)
            for (int k = 0; k + 1 < nz; ++k)
                if (hits[d.at(i, j, k)] == 3) { inner.push_back(i + 1); inner.push_back(j + 1); inner.push_back(k + 1); }
    *n_cmat = (int)(nodes.size() / 3);
    *n_cells = (int)(inner.size() / 3);
    *cmat_nodes = (int32_t*)std::malloc(sizeof(int32_t) * std::max<size_t>(1, nodes.size()));
    *cells = (int32_t*)std::malloc(sizeof(int32_t) * std::max<size_t>(1, inner.size()));
    if (!*cmat_nodes || !*cells) return FOPIS_ERR_NOMEM;
    std::memcpy(*cmat_nodes, nodes.data(), sizeof(int32_t) * nodes.size());
    std::memcpy(*cells, inner.data(), sizeof(int32_t) * inner.size());
    return FOPIS_OK;
}

// Per-node texture lists in the cmat order of fopis_parse_obj: the same quad
// walk, each covered node appending the quad's texture index.
extern "C" int fopis_parse_obj_textures(const char* path, int nx, int ny, int nz, int32_t** start, int32_t** tex,
                                        int* n_cmat) {
    if (!path || !start || !tex || !n_cmat || nx < 2 || ny < 2 || nz < 2) return FOPIS_ERR_ARG;
    Dom d{{nx, ny, nz}};
    int shift[3] = {nx / 2, ny / 2, nz / 2};
    std::vector<std::array<int, 3>> verts;
    std::vector<std::array<int, 4>> faces;
    std::vector<int> ftex;
    if (!read_obj(path, shift, verts, faces, &ftex)) return FOPIS_ERR_ARG;
    std::vector<int32_t> node_id(d.size(), -1);
    std::vector<std::vector<int32_t>> lists;
    for (size_t fi = 0; fi < faces.size(); ++fi) {
        const auto& q = faces[fi];
        std::array<int, 3> p[4];
        for (int t = 0; t < 4; ++t) {
            if (q[t] < 1 || q[t] > (int)verts.size()) return FOPIS_ERR_ARG;
            p[t] = verts[q[t] - 1];
        }
        int normal = -1;
        for (int a = 0; a < 3 && normal < 0; ++a)
            if (p[0][a] == p[1][a] && p[0][a] == p[2][a] && p[0][a] == p[3][a]) normal = a;
        if (normal < 0) return FOPIS_ERR_ARG;
        const int u = normal == 0 ? 1 : 0, w = normal == 2 ? 1 : 2;
        int lo_u = p[0][u], hi_u = p[0][u], lo_w = p[0][w], hi_w = p[0][w];
        for (int t = 1; t < 4; ++t) {
            lo_u = std::min(lo_u, p[t][u]); hi_u = std::max(hi_u, p[t][u]);
            lo_w = std::min(lo_w, p[t][w]); hi_w = std::max(hi_w, p[t][w]);
        }
        for (int a = lo_u; a <= hi_u; ++a)
            for (int b = lo_w; b <= hi_w; ++b) {
                int c[3];
                c[normal] = p[0][normal]; c[u] = a; c[w] = b;
                if (c[0] < 0 || c[1] < 0 || c[2] < 0 || c[0] >= nx || c[1] >= ny || c[2] >= nz) return FOPIS_ERR_ARG;
                const size_t id = d.at(c[0], c[1], c[2]);
                if (node_id[id] < 0) {
                    node_id[id] = (int32_t)lists.size();
                    lists.emplace_back();
                }
                lists[node_id[id]].push_back(ftex[fi]);
            }
    }
    size_t total = 0;
    for (const auto& l : lists) total += l.size();
    *n_cmat = (int)lists.size();
    *start = (int32_t*)std::malloc(sizeof(int32_t) * (lists.size() + 1));
    *tex = (int32_t*)std::malloc(sizeof(int32_t) * std::max<size_t>(1, total));
    if (!*start || !*tex) return FOPIS_ERR_NOMEM;
    size_t at = 0;
    for (size_t m = 0; m < lists.size(); ++m) {
        (*start)[m] = (int32_t)at;
        for (int32_t t : lists[m]) (*tex)[at++] = t;
    }
    (*start)[lists.size()] = (int32_t)at;
    return FOPIS_OK;
}
