// mfree_tool.h -- host-side rigid tool (triangle mesh, normals, triangle grid).
#pragma once

#include <string>
#include <vector>

#include "mfree_geom.h"

namespace mfree {

// mesh_triangle (surface_tri_mesh.h:39-63)
struct HostTri {
    int i1, i2, i3;
    Vec3f p1, p2, p3;
    Vec3f n, np1, np2, np3, ne1, ne2, ne3;
};

// tool_3d + grid_cpu_tri (tool_3d.h:39-78, grid_cpu_tri.h:32-59)
struct HostTool {
    std::vector<HostTri> tris;    // input order
    std::vector<HostTri> boxed;   // triangle-grid order, a triangle once per cell it cuts
    std::vector<int> boxed_src;   // input index of each boxed triangle
    std::vector<int> cells;       // CSR offsets into boxed, num_cell + 1
    int nx = 0, ny = 0, nz = 0;
    float bbmin[3] = {0, 0, 0}, bbmax[3] = {0, 0, 0}, dx = 0.f;
    // closest triangle by expanding shells (tool_3d::contact, tool_3d.cpp:55-161);
    // returns true when the point lies inside
    bool closest_by_shells(Vec3f qp, Vec3f &cp, Vec3f &nrm) const;
};

bool build_host_tool(HostTool &tool, const float *verts, int nv, const int *tris, int nt, std::string &err);

}  // namespace mfree
