// ref_host_shim.cpp -- TEST INFRASTRUCTURE: the reference's (iwf_mfree_gpu_3d)
// host-side scene setup, compiled unchanged from its read-only sources by
// oracle/build_ref.sh into oracle/_ref/libref_host.so, exposed with a C ABI so
// that the new readers and the oracle's tool setup can be checked against it:
//   json_read_triangles                 src/json_reader.cpp:108-117
//   ldynak_read_triangles_from_tetmesh  src/ldynak_reader.cpp:371-434
//   ldynak_read_triangles_from_quadmesh src/ldynak_reader.cpp:308-369
//   mesh_compute_vertex_normals         src/surface_tri_mesh.cpp:410-568
//   mesh_average_edge_length            src/surface_tri_mesh.cpp:570-584
//   tool_3d::tool_3d                    src/tool_3d.cpp:294-360 (normal flip,
//                                       triangle grid src/grid_cpu_tri.cpp:48-175)
// tool_3d keeps its triangle grid private and befriends tool_3d_gpu; the
// GPU-side class is not linked here, so this file defines the one
// tool_3d_gpu constructor it uses to read the grid out (a friend's member).
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "json_reader.h"
#include "ldynak_reader.h"
#include "surface_tri_mesh.h"
#include "tool_3d.h"
#include "tool_3d_gpu.h"

namespace {

struct ToolOut {
    std::vector<float> normals;  // per triangle: n, np1, np2, np3, ne1, ne2, ne3 (21 floats)
    std::vector<int> cells;      // m_num_cells + 1 prefix entries
    std::vector<int> boxed;      // original index of each boxed triangle (idx)
    int n3[3];
    float bbmin[3], bbmax[3], dx;
};
ToolOut g_tool;

int emit(const std::vector<mesh_triangle> &tris, const std::vector<vec3_t> &pos, float **v, int *nv, int **t,
         int *nt) {
    *nv = int(pos.size());
    *nt = int(tris.size());
    *v = (float *)malloc(sizeof(float) * 3 * pos.size() + 4);
    *t = (int *)malloc(sizeof(int) * 3 * tris.size() + 4);
    for (size_t k = 0; k < pos.size(); k++) {
        (*v)[3 * k] = pos[k].x;
        (*v)[3 * k + 1] = pos[k].y;
        (*v)[3 * k + 2] = pos[k].z;
    }
    for (size_t k = 0; k < tris.size(); k++) {
        (*t)[3 * k] = tris[k].i1;
        (*t)[3 * k + 1] = tris[k].i2;
        (*t)[3 * k + 2] = tris[k].i3;
    }
    return 0;
}

void put3(float *o, const vec3_t &a) {
    o[0] = a.x;
    o[1] = a.y;
    o[2] = a.z;
}

}  // namespace

// read-out of the private triangle grid (see the header comment)
tool_3d_gpu::tool_3d_gpu(const tool_3d *tool, float_t) {
    ToolOut &o = g_tool;
    o.cells.assign(tool->m_cells, tool->m_cells + tool->m_num_cells + 1);
    o.boxed.resize(tool->m_num_boxed_tris);
    for (unsigned k = 0; k < tool->m_num_boxed_tris; k++) o.boxed[k] = int(tool->m_boxed_tris[k].idx);
    o.n3[0] = tool->m_grid.nx();
    o.n3[1] = tool->m_grid.ny();
    o.n3[2] = tool->m_grid.nz();
    o.dx = tool->m_grid.dx();
    vec3_t lo, hi;
    tool->get_bbox(lo, hi);
    put3(o.bbmin, lo);
    put3(o.bbmax, hi);
    o.normals.resize(21 * tool->m_triangles.size());
    for (size_t k = 0; k < tool->m_triangles.size(); k++) {
        const mesh_triangle &T = tool->m_triangles[k];
        float *d = &o.normals[21 * k];
        put3(d, T.normal);
        put3(d + 3, T.np1);
        put3(d + 6, T.np2);
        put3(d + 9, T.np3);
        put3(d + 12, T.ne1);
        put3(d + 15, T.ne2);
        put3(d + 18, T.ne3);
    }
}

extern "C" {

int ref_read_json(const char *path, float **v, int *nv, int **t, int *nt) {
    std::vector<mesh_triangle> tris;
    std::vector<vec3_t> pos;
    json_read_triangles(std::string(path), tris, pos);
    return emit(tris, pos, v, nv, t, nt);
}

int ref_read_ldynak_tet(const char *path, float **v, int *nv, int **t, int *nt) {
    std::vector<mesh_triangle> tris;
    std::vector<vec3_t> pos;
    ldynak_read_triangles_from_tetmesh(std::string(path), tris, pos);
    return emit(tris, pos, v, nv, t, nt);
}

int ref_read_ldynak_quad(const char *path, float **v, int *nv, int **t, int *nt) {
    std::vector<mesh_triangle> tris;
    std::vector<vec3_t> pos;
    ldynak_read_triangles_from_quadmesh(std::string(path), tris, pos);
    return emit(tris, pos, v, nv, t, nt);
}

void ref_free(void *p) { free(p); }

// The reference's tool setup (mesh_compute_vertex_normals, mesh_average_edge_length,
// tool_3d) on a mesh in json_read_triangles' form; the results are read with
// ref_tool_*.  Returns the average edge length the tool was built with.
float ref_tool_setup(const float *verts, int nv, const int *tris, int nt) {
    std::vector<vec3_t> pos;
    std::vector<mesh_triangle> T;
    for (int k = 0; k < nv; k++) pos.push_back(vec3_t(verts[3 * k], verts[3 * k + 1], verts[3 * k + 2]));
    for (int k = 0; k < nt; k++) {
        mesh_triangle t;
        t.idx = (unsigned)k;
        t.i1 = tris[3 * k];
        t.i2 = tris[3 * k + 1];
        t.i3 = tris[3 * k + 2];
        T.push_back(t);
    }
    mesh_compute_vertex_normals(T, pos);
    const float_t h = mesh_average_edge_length(T);
    tool_3d tool(T, pos, h);
    tool_3d_gpu readout(&tool, 0.1f);
    (void)readout;
    return h;
}

void ref_tool_info(int *n3, float *bbmin, float *bbmax, float *dx, int *num_cells, int *num_boxed) {
    for (int d = 0; d < 3; d++) {
        n3[d] = g_tool.n3[d];
        bbmin[d] = g_tool.bbmin[d];
        bbmax[d] = g_tool.bbmax[d];
    }
    *dx = g_tool.dx;
    *num_cells = int(g_tool.cells.size()) - 1;
    *num_boxed = int(g_tool.boxed.size());
}

void ref_tool_arrays(float *normals, int *cells, int *boxed) {
    memcpy(normals, g_tool.normals.data(), sizeof(float) * g_tool.normals.size());
    memcpy(cells, g_tool.cells.data(), sizeof(int) * g_tool.cells.size());
    memcpy(boxed, g_tool.boxed.data(), sizeof(int) * g_tool.boxed.size());
}

}  // extern "C"
