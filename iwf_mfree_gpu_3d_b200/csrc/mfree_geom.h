// mfree_geom.h -- float 3-vectors and the closest point on a triangle, shared
// by the host tool setup (mfree_tool.cpp, g++) and the contact kernel
// (mfree_contact.cu, nvcc).  One definition, compiled by both.
//
// The closest point follows the reference's comp_closest_point
// (src/tool_3d_gpu.cu:141-212, host twin mesh_triangle::closest_point,
// src/surface_tri_mesh.cpp:42-104): the barycentric coordinates of the query
// point's projection decide between the face and one of the three edges,
// whose closest point is the clamped projection onto the segment.  Which
// feature the point lies on picks the contact normal (face, edge or vertex
// normal), so the region tests keep the reference's order and comparisons.
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define MFREE_HD __host__ __device__ __forceinline__
#else
#define MFREE_HD inline
#endif

namespace mfree {

struct Vec3f {
    float x, y, z;
};

MFREE_HD Vec3f vadd(Vec3f a, Vec3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
MFREE_HD Vec3f vsub(Vec3f a, Vec3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
MFREE_HD Vec3f vscale(float s, Vec3f a) { return {s * a.x, s * a.y, s * a.z}; }
MFREE_HD Vec3f vneg(Vec3f a) { return {-a.x, -a.y, -a.z}; }
MFREE_HD bool veq(Vec3f a, Vec3f b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
MFREE_HD float vdot(Vec3f a, Vec3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
MFREE_HD Vec3f vcross(Vec3f a, Vec3f b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
MFREE_HD float vlength(Vec3f a) { return sqrtf(vdot(a, a)); }

// closest point to q on the segment from a to b (clamped projection; a
// zero-length segment gives a)
MFREE_HD Vec3f closest_on_segment(Vec3f a, Vec3f b, Vec3f q) {
    const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    const float len2 = dx * dx + dy * dy + dz * dz;
    if (len2 == 0.f) return a;
    const float s = ((b.x - a.x) * (q.x - a.x) + (b.y - a.y) * (q.y - a.y) + (b.z - a.z) * (q.z - a.z)) / len2;
    if (s > 1.f) return b;
    if (s < 0.f) return a;
    return vadd(vscale(1.f - s, a), vscale(s, b));
}

// the triangle feature a closest point lies on
enum TriFeature { TF_FACE = 0, TF_V1, TF_V2, TF_V3, TF_E12, TF_E23, TF_E31 };

// Closest point cp on triangle (v1, v2, v3) to q; returns its feature.  With
// edge vectors ea = v2 - v1, eb = v3 - v1 and w = v1 - q, (sa, sb) solve the
// 2x2 normal equations of the projection cp = v1 + sa ea + sb eb.  A negative
// sa sends the point to edge v1-v3, a negative sb to edge v1-v2, sa + sb > 1
// to edge v2-v3; an edge point equal to one of its end vertices is that vertex.
MFREE_HD int closest_on_triangle(Vec3f v1, Vec3f v2, Vec3f v3, Vec3f q, Vec3f &cp) {
    const Vec3f ea = vsub(v2, v1), eb = vsub(v3, v1), w = vsub(v1, q);
    const float ab = vdot(eb, ea), aa = vdot(ea, ea), bb = vdot(eb, eb);
    const float den = ab * ab - aa * bb;
    const float wb = vdot(eb, w), wa = vdot(ea, w);
    const float sa = (wa * bb - wb * ab) / den, sb = (wb * aa - wa * ab) / den;
    if (sa < 0.f) {
        cp = closest_on_segment(v1, v3, q);
        return veq(cp, v1) ? TF_V1 : (veq(cp, v3) ? TF_V3 : TF_E31);
    }
    if (sb < 0.f) {
        cp = closest_on_segment(v1, v2, q);
        return veq(cp, v1) ? TF_V1 : (veq(cp, v2) ? TF_V2 : TF_E12);
    }
    if (sa + sb > 1.f) {
        cp = closest_on_segment(v2, v3, q);
        return veq(cp, v2) ? TF_V2 : (veq(cp, v3) ? TF_V3 : TF_E23);
    }
    cp = vadd(vadd(v1, vscale(sa, ea)), vscale(sb, eb));
    return TF_FACE;
}

}  // namespace mfree
