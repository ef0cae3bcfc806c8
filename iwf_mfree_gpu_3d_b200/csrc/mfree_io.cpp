// mfree_io.cpp -- tool mesh readers of the reference's scene setup.
//
//   mfree_read_mesh_json    <- json_read_triangles (json_reader.cpp:20-117): MeshLab
//                              JSON; the first numeric lines after "vertices" are
//                              xyz triplets, the first after "connectivity" are
//                              vertex-index triplets; reading stops at ']'.
//   mfree_read_mesh_ldynak  <- ldynak_read_triangles_from_tetmesh
//                              (ldynak_reader.cpp:177-434): LS-DYNA *NODE and
//                              *ELEMENT_SOLID tetrahedra (n4..n8 equal); faces seen
//                              by exactly one tetrahedron form the surface.
//   mfree_read_mesh_ldynak_quad <- ldynak_read_triangles_from_quadmesh
//                              (ldynak_reader.cpp:308-369): *ELEMENT_SOLID
//                              hexahedra (n1..n8); quadrilateral faces seen by
//                              exactly one hexahedron form the surface, each
//                              split into (a, b, c) and (c, d, a).
//
// The LS-DYNA reader returns vertices and faces in the order the reference's
// std::unordered_map iteration produces them (tool_3d_gpu.cu's closest-triangle
// search breaks ties by that order).  To get the same order the same container
// operations are issued in the same sequence: a map from node id to position
// filled in file order and iterated for the linear ids; a map from face to
// count keyed by the sum of the three std::hash<unsigned> values with
// order-independent equality, filled tetrahedron by tetrahedron.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "mfree.h"

namespace {

struct P3 {
    float x, y, z;
};

std::vector<std::string> split_on(const std::string &s, char delim) {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, delim)) out.push_back(item);
    return out;
}
std::vector<std::string> split_ws(const std::string &s) {
    std::istringstream buf(s);
    return std::vector<std::string>(std::istream_iterator<std::string>(buf), std::istream_iterator<std::string>());
}

int emit(const std::vector<P3> &v, const std::vector<int> &t, float **verts, int *nv, int **tris, int *nt) {
    if (v.empty() || t.empty()) return MFREE_ERR_IO;
    *verts = (float *)malloc(sizeof(float) * 3 * v.size());
    *tris = (int *)malloc(sizeof(int) * t.size());
    if (!*verts || !*tris) {
        free(*verts);
        free(*tris);
        return MFREE_ERR_OOM;
    }
    for (size_t i = 0; i < v.size(); i++) {
        (*verts)[3 * i] = v[i].x;
        (*verts)[3 * i + 1] = v[i].y;
        (*verts)[3 * i + 2] = v[i].z;
    }
    std::memcpy(*tris, t.data(), sizeof(int) * t.size());
    *nv = int(v.size());
    *nt = int(t.size() / 3);
    return MFREE_OK;
}

struct Face {
    unsigned i1, i2, i3;
    bool operator==(const Face &o) const {
        std::set<unsigned> a({i1, i2, i3}), b({o.i1, o.i2, o.i3});
        std::set<unsigned> c;
        std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::inserter(c, c.begin()));
        return c.size() == 3;
    }
};
struct FaceHash {
    size_t operator()(const Face &f) const {
        return std::hash<unsigned>()(f.i1) + std::hash<unsigned>()(f.i2) + std::hash<unsigned>()(f.i3);
    }
};
// a hexahedron's face: equal when the two node sets share four members (so a
// face with a repeated node equals no face, itself included, as there)
struct QFace {
    unsigned i1, i2, i3, i4;
    bool operator==(const QFace &o) const {
        std::set<unsigned> a({i1, i2, i3, i4}), b({o.i1, o.i2, o.i3, o.i4});
        std::set<unsigned> c;
        std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::inserter(c, c.begin()));
        return c.size() == 4;
    }
};
struct QFaceHash {
    size_t operator()(const QFace &f) const {
        return std::hash<unsigned>()(f.i1) + std::hash<unsigned>()(f.i2) + std::hash<unsigned>()(f.i3) +
               std::hash<unsigned>()(f.i4);
    }
};

// the node ids of the *ELEMENT section's lines (comment lines skipped): the
// first `count` after the element and part ids; false on a short line
bool read_elements(std::ifstream &in, int count, std::vector<std::vector<unsigned>> &out) {
    std::string line;
    bool sec = false;
    while (std::getline(in, line)) {
        if (line.find('$') != std::string::npos) continue;
        if (line.find("*ELEMENT") != std::string::npos) {
            sec = true;
            continue;
        }
        if (sec && line.find('*') != std::string::npos) break;
        if (!sec) continue;
        auto tok = split_ws(line);
        if (int(tok.size()) < 2 + count) return false;
        std::vector<unsigned> id(count);
        for (int k = 0; k < count; k++) id[k] = unsigned(strtoul(tok[2 + k].c_str(), nullptr, 0));
        out.push_back(id);
    }
    return true;
}

// *NODE section: node id -> position, inserted in file order
bool read_nodes(std::ifstream &in, std::unordered_map<int, P3> &nodes) {
    std::string line;
    bool sec = false;
    while (std::getline(in, line)) {
        if (line.find('$') != std::string::npos) continue;
        if (line.find("*NODE") != std::string::npos) {
            sec = true;
            continue;
        }
        if (sec && line.find('*') != std::string::npos) break;
        if (!sec) continue;
        auto tok = split_ws(line);
        if (tok.size() < 4) return false;
        unsigned nid = unsigned(strtoul(tok[0].c_str(), nullptr, 0));
        double x = std::stod(tok[1]), y = std::stod(tok[2]), z = std::stod(tok[3]);
        nodes.insert({int(nid), P3{float(x), float(y), float(z)}});
    }
    return true;
}

// linear vertex ids in the node map's iteration order
void linear_ids(const std::unordered_map<int, P3> &nodes, std::unordered_map<unsigned, unsigned> &lin,
                std::vector<P3> &v) {
    unsigned it = 0;
    for (auto &kv : nodes) {
        lin.insert({unsigned(kv.first), it});
        v.push_back(kv.second);
        it++;
    }
}

}  // namespace

extern "C" {

int mfree_read_mesh_json(const char *path, float **verts, int *nv, int **tris, int *nt) {
    if (!path || !verts || !nv || !tris || !nt) return MFREE_ERR_ARG;
    std::ifstream in(path);
    if (!in) return MFREE_ERR_IO;
    std::vector<P3> v;
    std::vector<int> t;
    std::string line;
    bool sec = false;
    while (std::getline(in, line)) {
        if (line.find("vertices") != std::string::npos) sec = true;
        if (line.find(']') != std::string::npos) break;
        if (!sec) continue;
        auto tok = split_on(line, ',');
        if (tok.size() >= 3) {
            if (tok.size() % 3) return MFREE_ERR_IO;
            for (size_t i = 0; i < tok.size(); i += 3)
                v.push_back({float(atof(tok[i].c_str())), float(atof(tok[i + 1].c_str())), float(atof(tok[i + 2].c_str()))});
        }
    }
    sec = false;
    while (std::getline(in, line)) {
        if (line.find("connectivity") != std::string::npos) sec = true;
        if (sec && line.find(']') != std::string::npos) break;
        if (!sec) continue;
        auto tok = split_on(line, ',');
        if (tok.size() >= 3) {
            if (tok.size() % 3) return MFREE_ERR_IO;
            for (size_t i = 0; i < tok.size(); i++) t.push_back(atoi(tok[i].c_str()));
        }
    }
    for (int k : t)
        if (k < 0 || k >= int(v.size())) return MFREE_ERR_IO;
    return emit(v, t, verts, nv, tris, nt);
}

int mfree_read_mesh_ldynak(const char *path, float **verts, int *nv, int **tris, int *nt) {
    if (!path || !verts || !nv || !tris || !nt) return MFREE_ERR_ARG;
    std::ifstream in(path);
    if (!in) return MFREE_ERR_IO;
    // tetrahedra: element id, part id, n1..n8 with n4..n8 equal
    std::vector<std::vector<unsigned>> tets;
    if (!read_elements(in, 4, tets) || tets.empty()) return MFREE_ERR_IO;
    std::vector<Face> faces;  // 4 per tetrahedron (ids_to_tet_segment, ldynak_reader.cpp:116-127)
    for (const auto &id : tets) {
        faces.push_back({id[0], id[1], id[3]});
        faces.push_back({id[2], id[1], id[0]});
        faces.push_back({id[1], id[2], id[3]});
        faces.push_back({id[3], id[2], id[0]});
    }
    in.clear();
    in.seekg(0);
    std::unordered_map<int, P3> nodes;
    if (!read_nodes(in, nodes)) return MFREE_ERR_IO;
    std::unordered_map<Face, unsigned, FaceHash> seen;
    for (const Face &f : faces) {
        auto it = seen.find(f);
        if (it != seen.end()) it->second++;
        else seen.insert({f, 1u});
    }
    std::vector<Face> boundary;
    for (auto &kv : seen)
        if (kv.second == 1) boundary.push_back(kv.first);
    std::unordered_map<unsigned, unsigned> lin;
    std::vector<P3> v;
    linear_ids(nodes, lin, v);
    std::vector<int> t;
    for (auto &f : boundary) {
        if (!lin.count(f.i1) || !lin.count(f.i2) || !lin.count(f.i3)) return MFREE_ERR_IO;
        t.push_back(int(lin[f.i1]));
        t.push_back(int(lin[f.i2]));
        t.push_back(int(lin[f.i3]));
    }
    return emit(v, t, verts, nv, tris, nt);
}

int mfree_read_mesh_ldynak_quad(const char *path, float **verts, int *nv, int **tris, int *nt) {
    if (!path || !verts || !nv || !tris || !nt) return MFREE_ERR_ARG;
    std::ifstream in(path);
    if (!in) return MFREE_ERR_IO;
    std::vector<std::vector<unsigned>> hexes;
    if (!read_elements(in, 8, hexes) || hexes.empty()) return MFREE_ERR_IO;
    // the six faces of each hexahedron, in the order and orientation of
    // ids_to_quad_segment (ldynak_reader.cpp:100-114)
    static const int fi[6][4] = {{0, 1, 2, 3}, {7, 6, 5, 4}, {4, 5, 1, 0}, {3, 2, 6, 7}, {0, 3, 7, 4}, {5, 6, 2, 1}};
    in.clear();
    in.seekg(0);
    std::unordered_map<int, P3> nodes;
    if (!read_nodes(in, nodes)) return MFREE_ERR_IO;
    std::unordered_map<QFace, unsigned, QFaceHash> seen;
    for (const auto &h : hexes)
        for (int f = 0; f < 6; f++) {
            const QFace q{h[fi[f][0]], h[fi[f][1]], h[fi[f][2]], h[fi[f][3]]};
            auto it = seen.find(q);
            if (it != seen.end()) it->second++;
            else seen.insert({q, 1u});
        }
    std::vector<QFace> boundary;
    for (auto &kv : seen)
        if (kv.second == 1) boundary.push_back(kv.first);
    std::unordered_map<unsigned, unsigned> lin;
    std::vector<P3> v;
    linear_ids(nodes, lin, v);
    std::vector<int> t;
    for (auto &q : boundary) {
        if (!lin.count(q.i1) || !lin.count(q.i2) || !lin.count(q.i3) || !lin.count(q.i4)) return MFREE_ERR_IO;
        const int a = int(lin[q.i1]), b = int(lin[q.i2]), c = int(lin[q.i3]), d = int(lin[q.i4]);
        t.insert(t.end(), {a, b, c, c, d, a});  // quads_to_tris (ldynak_reader.cpp:264-289)
    }
    return emit(v, t, verts, nv, tris, nt);
}

}  // extern "C"
