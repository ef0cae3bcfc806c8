// mfree_tool.cpp -- host-side setup of a rigid tool (C++).
//
// Reference setup replaced:
//   mesh_compute_vertex_normals   surface_tri_mesh.cpp:410-568  (face normals;
//                                 edge normal = normalised sum of the two faces;
//                                 vertex normal = sum of face normals weighted by
//                                 acos(|cos|) of the corner angle, normalised)
//   mesh_average_edge_length      surface_tri_mesh.cpp:570-584  ((min+max)/2)
//   grid_cpu_tri::update_geometry_mesh / get_cells
//                                 grid_cpu_tri.cpp:48-175        (box of all
//                                 triangles +-1e-4, cells of the average edge
//                                 length, a triangle listed in every cell its
//                                 box overlaps and that it cuts)
//   mesh_triangle::cover_aabb     surface_tri_mesh.cpp:151-278  (Akenine-Moller)
//   tool_3d::tool_3d normal flip  tool_3d.cpp:294-360           (all normals flip
//                                 if a point just outside the grid box tests inside)
// Arithmetic is float, as in the reference's float build (vec3_t = glm::vec3).
#include "mfree_tool.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <unordered_map>

namespace mfree {

namespace {

using V = Vec3f;
inline V add(V a, V b) { return vadd(a, b); }
inline V sub(V a, V b) { return vsub(a, b); }
inline V mul(float s, V a) { return vscale(s, a); }
inline V neg(V a) { return vneg(a); }
inline float dot(V a, V b) { return vdot(a, b); }
inline V cross(V a, V b) { return vcross(a, b); }
inline float length(V a) { return vlength(a); }
inline V normalize(V a) { return mul(1.0f / std::sqrt(dot(a, a)), a); }
inline float comp(V a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }
inline void setc(V &a, int d, float v) { (d == 0 ? a.x : (d == 1 ? a.y : a.z)) = v; }

// closest point on a triangle and the normal of the feature it lies on
// (mesh_triangle::closest_point, surface_tri_mesh.cpp:42-104; the geometry is
// shared with the contact kernel in mfree_geom.h)
void closest_point(const HostTri &T, V qp, V &cp, V &np) {
    switch (closest_on_triangle(T.p1, T.p2, T.p3, qp, cp)) {
        case TF_V1: np = T.np1; break;
        case TF_V2: np = T.np2; break;
        case TF_V3: np = T.np3; break;
        case TF_E12: np = T.ne1; break;
        case TF_E23: np = T.ne2; break;
        case TF_E31: np = T.ne3; break;
        default: np = T.n; break;
    }
}

bool plane_box_overlap(V n, V v, V mb) {
    V vmin, vmax;
    for (int q = 0; q < 3; q++) {
        if (comp(n, q) > 0.f) {
            setc(vmin, q, -comp(mb, q) - comp(v, q));
            setc(vmax, q, comp(mb, q) - comp(v, q));
        } else {
            setc(vmin, q, comp(mb, q) - comp(v, q));
            setc(vmax, q, -comp(mb, q) - comp(v, q));
        }
    }
    if (dot(n, vmin) > 0.f) return false;
    return dot(n, vmax) >= 0.f;
}

// separating-axis triangle/box test: 9 edge x axis tests, 3 box axes, the plane
bool tri_box(const HostTri &T, V bmin, V bmax) {
    V c = mul(0.5f, add(bmin, bmax)), hs = mul(0.5f, sub(bmax, bmin));
    V v0 = sub(T.p1, c), v1 = sub(T.p2, c), v2 = sub(T.p3, c);
    V e[3] = {sub(T.p2, T.p1), sub(T.p3, T.p2), sub(T.p1, T.p3)};
    const V vv[3] = {v0, v1, v2};
    // for edge k the two projections tested are of the vertices not both on the edge
    // (edge 0: v0, v2; edge 1: v0, v1 for y/z; edge 2: v0, v1 / v1, v2) -- as in the
    // published test, which drops the redundant vertex per axis
    auto axis = [&](float pa, float pb, float rad) {
        float lo = std::min(pa, pb), hi = std::max(pa, pb);
        return !(lo > rad || hi < -rad);
    };
    for (int k = 0; k < 3; k++) {
        const V ed = e[k];
        const float fx = std::fabs(ed.x), fy = std::fabs(ed.y), fz = std::fabs(ed.z);
        // vertex pairs per edge and axis: X and Y use (a, b), Z uses (c, d)
        int a, b, cc, d;
        if (k == 0) { a = 0; b = 2; cc = 1; d = 2; }
        else if (k == 1) { a = 0; b = 2; cc = 0; d = 1; }
        else { a = 0; b = 1; cc = 1; d = 2; }
        // X axis: p = ez*v.y - ey*v.z
        float px0 = ed.z * vv[a].y - ed.y * vv[a].z, px1 = ed.z * vv[b].y - ed.y * vv[b].z;
        if (!axis(px0, px1, fz * hs.y + fy * hs.z)) return false;
        // Y axis: p = -ez*v.x + ex*v.z
        float py0 = -ed.z * vv[a].x + ed.x * vv[a].z, py1 = -ed.z * vv[b].x + ed.x * vv[b].z;
        if (!axis(py0, py1, fz * hs.x + fx * hs.z)) return false;
        // Z axis: p = ey*v.x - ex*v.y
        float pz0 = ed.y * vv[cc].x - ed.x * vv[cc].y, pz1 = ed.y * vv[d].x - ed.x * vv[d].y;
        if (!axis(pz0, pz1, fy * hs.x + fx * hs.y)) return false;
    }
    for (int q = 0; q < 3; q++) {
        float lo = std::min(std::min(comp(v0, q), comp(v1, q)), comp(v2, q));
        float hi = std::max(std::max(comp(v0, q), comp(v1, q)), comp(v2, q));
        if (lo > comp(hs, q) || hi < -comp(hs, q)) return false;
    }
    return plane_box_overlap(cross(e[0], e[1]), v0, hs);
}

}  // namespace

bool HostTool::closest_by_shells(Vec3f qp, Vec3f &cp, Vec3f &nrm) const {
    auto cell = [&](float p, int d) {
        long v = long((unsigned)((p - bbmin[d]) / dx));
        long n = d == 0 ? nx : (d == 1 ? ny : nz);
        return std::min(v, n - 1);
    };
    long ix = cell(qp.x, 0), iy = cell(qp.y, 1), iz = cell(qp.z, 2);
    float md = HUGE_VALF;
    V bcp{0, 0, 0}, bn{0, 0, 0};
    long b = ix * ny * nz + iy * nz + iz;
    bool empty = cells[b] == cells[b + 1];
    for (int k = cells[b]; k < cells[b + 1]; k++) {
        V c, n;
        closest_point(boxed[k], qp, c, n);
        float d = dot(sub(c, qp), sub(c, qp));
        if (d < md) { md = d; bcp = c; bn = n; }
    }
    long off = 1, cap = std::max(nx, std::max(ny, nz)) + 2;
    bool done = false;
    while (off <= cap) {
        long li = std::max(ix - off, 0L), lj = std::max(iy - off, 0L), lk = std::max(iz - off, 0L);
        long hi = std::min(ix + off + 1, long(nx)), hj = std::min(iy + off + 1, long(ny)),
             hk = std::min(iz + off + 1, long(nz));
        for (long a = li; a < hi; a++)
            for (long bb = lj; bb < hj; bb++)
                for (long c = lk; c < hk; c++) {
                    if (!(a == li || a == hi - 1 || bb == lj || bb == hj - 1 || c == lk || c == hk - 1)) continue;
                    long box = a * ny * nz + bb * nz + c;
                    for (int k = cells[box]; k < cells[box + 1]; k++) {
                        empty = false;
                        V cc, n;
                        closest_point(boxed[k], qp, cc, n);
                        float d = dot(sub(cc, qp), sub(cc, qp));
                        if (d < md) { md = d; bcp = cc; bn = n; }
                    }
                }
        if (done) break;
        off++;
        if (!empty) done = true;
    }
    cp = bcp;
    nrm = bn;
    return dot(sub(bcp, qp), bn) <= 0.f;
}

bool build_host_tool(HostTool &tool, const float *verts, int nv, const int *tri, int nt, std::string &err) {
    if (nv <= 0 || nt <= 0 || !verts || !tri) {
        err = "empty tool mesh";
        return false;
    }
    std::vector<V> P(nv);
    for (int i = 0; i < nv; i++) P[i] = {verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]};
    std::vector<HostTri> T(nt);
    std::vector<std::vector<int>> vtri(nv);
    struct EK {
        int a, b;
        bool operator==(const EK &o) const { return (a == o.a && b == o.b) || (a == o.b && b == o.a); }
    };
    struct EH {
        size_t operator()(const EK &e) const { return std::hash<unsigned>()(e.a) + std::hash<unsigned>()(e.b); }
    };
    std::unordered_map<EK, std::vector<int>, EH> edges;
    for (int i = 0; i < nt; i++) {
        HostTri &t = T[i];
        t.i1 = tri[3 * i];
        t.i2 = tri[3 * i + 1];
        t.i3 = tri[3 * i + 2];
        if (t.i1 < 0 || t.i1 >= nv || t.i2 < 0 || t.i2 >= nv || t.i3 < 0 || t.i3 >= nv) {
            err = "triangle vertex index out of range";
            return false;
        }
        vtri[t.i1].push_back(i);
        vtri[t.i2].push_back(i);
        vtri[t.i3].push_back(i);
        edges[EK{t.i1, t.i2}].push_back(i);
        edges[EK{t.i2, t.i3}].push_back(i);
        edges[EK{t.i3, t.i1}].push_back(i);
    }
    for (auto &e : edges)
        if (e.second.size() < 2) {
            err = "tool mesh is not closed: an edge belongs to one triangle";
            return false;
        }
    for (auto &t : T) {
        t.p1 = P[t.i1];
        t.p2 = P[t.i2];
        t.p3 = P[t.i3];
        V c = cross(sub(t.p2, t.p1), sub(t.p3, t.p1));
        if (dot(c, c) == 0.f) {
            err = "degenerate tool triangle";
            return false;
        }
        t.n = normalize(c);
    }
    for (auto &t : T) {
        const auto &a = edges[EK{t.i1, t.i2}], &b = edges[EK{t.i2, t.i3}], &c = edges[EK{t.i3, t.i1}];
        t.ne1 = normalize(add(T[a[0]].n, T[a[1]].n));
        t.ne2 = normalize(add(T[b[0]].n, T[b[1]].n));
        t.ne3 = normalize(add(T[c[0]].n, T[c[1]].n));
    }
    auto vnormal = [&](int v) {
        V acc{0, 0, 0};
        for (int ti : vtri[v]) {
            const HostTri &t = T[ti];
            V f1, f2;
            if (t.i1 == v) { f1 = t.p2; f2 = t.p3; }
            if (t.i2 == v) { f1 = t.p1; f2 = t.p3; }
            if (t.i3 == v) { f1 = t.p1; f2 = t.p2; }
            V a = sub(f1, P[v]), b = sub(f2, P[v]);
            float ang = std::acos(std::fabs(dot(a, b) / (length(a) * length(b))));
            acc = add(acc, mul(ang, t.n));
        }
        return normalize(acc);
    };
    for (auto &t : T) {
        t.np1 = vnormal(t.i1);
        t.np2 = vnormal(t.i2);
        t.np3 = vnormal(t.i3);
    }
    float lmin = HUGE_VALF, lmax = 0.f;
    for (auto &t : T) {
        float l1 = length(sub(t.p1, t.p2)), l2 = length(sub(t.p2, t.p3)), l3 = length(sub(t.p3, t.p1));
        lmin = std::min(std::min(std::min(lmin, l1), l2), l3);
        lmax = std::max(std::max(std::max(lmax, l1), l2), l3);
    }
    const float havg = 0.5f * (lmax + lmin);
    float bmin[3] = {HUGE_VALF, HUGE_VALF, HUGE_VALF}, bmax[3] = {-HUGE_VALF, -HUGE_VALF, -HUGE_VALF};
    for (auto &t : T)
        for (int d = 0; d < 3; d++) {
            bmin[d] = std::min(std::min(std::min(comp(t.p1, d), comp(t.p2, d)), comp(t.p3, d)), bmin[d]);
            bmax[d] = std::max(std::max(std::max(comp(t.p1, d), comp(t.p2, d)), comp(t.p3, d)), bmax[d]);
        }
    for (int d = 0; d < 3; d++) {
        bmin[d] = float(double(bmin[d]) - 1e-4);
        bmax[d] = float(double(bmax[d]) + 1e-4);
        tool.bbmin[d] = bmin[d];
        tool.bbmax[d] = bmax[d];
    }
    tool.dx = havg;
    tool.nx = int(std::ceil((bmax[0] - bmin[0]) / havg));
    tool.ny = int(std::ceil((bmax[1] - bmin[1]) / havg));
    tool.nz = int(std::ceil((bmax[2] - bmin[2]) / havg));
    const long ncell = long(tool.nx) * tool.ny * tool.nz;
    if (!(havg > 0.f) || ncell <= 0 || ncell > (1L << 26)) {
        err = "tool grid has an unusable number of cells";
        return false;
    }
    std::vector<std::vector<int>> grid(ncell);
    for (int i = 0; i < nt; i++) {
        const HostTri &t = T[i];
        long il[3], ih[3];
        for (int d = 0; d < 3; d++) {
            float lo = std::min(std::min(comp(t.p1, d), comp(t.p2, d)), comp(t.p3, d));
            float hi = std::max(std::max(comp(t.p1, d), comp(t.p2, d)), comp(t.p3, d));
            il[d] = long((unsigned)((lo - bmin[d]) / havg));
            ih[d] = long((unsigned)((hi - bmin[d]) / havg));
        }
        for (long a = il[0]; a <= ih[0]; a++)
            for (long b = il[1]; b <= ih[1]; b++)
                for (long c = il[2]; c <= ih[2]; c++) {
                    if (a >= tool.nx || b >= tool.ny || c >= tool.nz) continue;
                    V lo{bmin[0] + float(a) * havg, bmin[1] + float(b) * havg, bmin[2] + float(c) * havg};
                    V hi{bmin[0] + float(a + 1) * havg, bmin[1] + float(b + 1) * havg, bmin[2] + float(c + 1) * havg};
                    if (tri_box(t, lo, hi)) grid[a * tool.ny * tool.nz + b * tool.nz + c].push_back(i);
                }
    }
    tool.cells.assign(ncell + 1, 0);
    tool.boxed.clear();
    tool.boxed_src.clear();
    for (long c = 0; c < ncell; c++) {
        tool.cells[c] = int(tool.boxed.size());
        for (int ti : grid[c]) {
            tool.boxed.push_back(T[ti]);
            tool.boxed_src.push_back(ti);
        }
    }
    tool.cells[ncell] = int(tool.boxed.size());
    tool.tris = T;
    V out{float(double(bmax[0]) + 1e-6), float(double(bmax[1]) + 1e-6), float(double(bmax[2]) + 1e-6)};
    V cp, nn;
    if (tool.closest_by_shells(out, cp, nn)) {
        auto flip = [](HostTri &t) {
            t.ne1 = neg(t.ne1); t.ne2 = neg(t.ne2); t.ne3 = neg(t.ne3);
            t.np1 = neg(t.np1); t.np2 = neg(t.np2); t.np3 = neg(t.np3);
            t.n = neg(t.n);
        };
        for (auto &t : tool.tris) flip(t);
        for (auto &t : tool.boxed) flip(t);
    }
    return true;
}

}  // namespace mfree
