// ref_step_main.cu -- scene driver for the comparator build of the reference's
// own GPU step (iwf_mfree_gpu_3d), built by build_ref_gpu.sh.  Not part of the
// library: it links the reference's translation units and calls them the way
// the reference's main() and setup functions do
// (src/mfree_gpu_3d.cpp:75-218, src/Benchmarks/benchmarks_single_grain.cu:674-876),
// on a scene read from a file written by baseline/refgpu.py:
//
//   new particle_gpu(pos, vel, rho, T, h, fixed, tool_p, n)   particle_gpu.cu:114
//   actions_/interactions_setup_* constants                  actions_gpu.cu:659-710, interactions_gpu.cu:561-608
//   mesh_compute_vertex_normals, tool_3d, tool_3d_gpu         surface_tri_mesh.cpp:410, tool_3d.cpp:294, tool_3d_gpu.cu:763
//   new grid_gpu_green(n, bbmin, bbmax, h), new blanking(...)  grid_gpu_green.cu:342, blanking.cpp:29
//   new leap_frog(N_init, num_cell); step(particles, grid, record)   leap_frog.cu:121-206
//
// Usage: ref_step_<variant> scene.bin warmup steps [out.bin]
//   runs `warmup` steps, then times `steps` steps with CUDA events around the
//   loop (the reference's step synchronises the device after its launches),
//   prints one JSON line, and with out.bin writes the particle state after the
//   last step (sorted order, with each particle's creation index, which the
//   driver tags into the unused vel_bc.w) and the tool
//   forces of the last step.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "leap_frog.h"
#include "grid_gpu_green.h"
#include "tool_3d.h"
#include "tool_3d_gpu.h"
#include "blanking.h"
#include "surface_tri_mesh.h"
#include "actions_gpu.h"
#include "interactions_gpu.h"

// the process globals of the reference's main() (src/mfree_gpu_3d.cpp:41-48)
std::vector<tool_3d_gpu *> global_tool;
tool_forces *global_tool_forces = 0;
blanking *global_blanking = 0;
float_t global_time_dt = 0;
float_t global_time_final = 0;
float_t global_time_current = 0;
int global_time_step = 0;

namespace {

struct reader {
    FILE *f;
    template <class T> void get(T *p, size_t n) {
        if (n && fread(p, sizeof(T), n, f) != n) { fprintf(stderr, "scene file truncated\n"); exit(2); }
    }
    int i32() { int v; get(&v, 1); return v; }
    float f32() { float v; get(&v, 1); return v; }
};

struct scene_tool {
    std::vector<float> verts;
    std::vector<int> tris;
    float vel[3], alpha, mu;
    int algorithm;
};

template <class T> void put(FILE *f, const T *p, size_t n) { fwrite(p, sizeof(T), n, f); }

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s scene.bin warmup steps [out.bin]\n", argv[0]);
        return 2;
    }
    FILE *sf = fopen(argv[1], "rb");
    if (!sf) { fprintf(stderr, "cannot open %s\n", argv[1]); return 2; }
    const int warmup = atoi(argv[2]), steps = atoi(argv[3]);
    reader r{sf};
    char magic[8];
    r.get(magic, 8);
    if (memcmp(magic, "MFREESC1", 8) != 0) { fprintf(stderr, "not a scene file\n"); return 2; }
    const int n = r.i32(), ntools = r.i32(), has_joco = r.i32(), cspm = r.i32(), conduction = r.i32();
    float phys_v[6], corr_v[6], joco_v[9], twp_v[6], ttool_v[6], gmin[3], gmax[3], bmin[3], bmax[3];
    r.get(phys_v, 6); r.get(corr_v, 6); r.get(joco_v, 9); r.get(twp_v, 6); r.get(ttool_v, 6);
    r.get(gmin, 3); r.get(gmax, 3);
    const float grid_h = r.f32();
    r.get(bmin, 3); r.get(bmax, 3);
    const float blank_vmax = r.f32(), dt = r.f32();
    std::vector<float4_t> pos(n), vel(n);
    std::vector<float_t> rho(n), T(n), h(n), fixed(n), tool_p(n);
    r.get(&pos[0].x, 4 * (size_t)n); r.get(&vel[0].x, 4 * (size_t)n);
    r.get(rho.data(), n); r.get(T.data(), n); r.get(h.data(), n); r.get(fixed.data(), n); r.get(tool_p.data(), n);
    // optional initial deviatoric stress (mat3x3 per particle, the reference's
    // column-major layout), for checks that start from a loaded state
    const int has_S = r.i32();
    std::vector<mat3x3_t> S0(has_S ? n : 0);
    if (has_S) r.get(&S0[0][0][0], 9 * (size_t)n);
    std::vector<scene_tool> tools(ntools);
    for (auto &t : tools) {
        const int nv = r.i32(), nt = r.i32();
        t.algorithm = r.i32();
        r.get(t.vel, 3);
        t.alpha = r.f32();
        t.mu = r.f32();
        t.verts.resize(3 * (size_t)nv);
        t.tris.resize(3 * (size_t)nt);
        r.get(t.verts.data(), t.verts.size());
        r.get(t.tris.data(), t.tris.size());
    }
    fclose(sf);

#if defined(CSPM)
    const int built_cspm = 1;
#else
    const int built_cspm = 0;
#endif
#if defined(Thermal_Conduction_PSE)
    const int built_conduction = 2;
#else
    const int built_conduction = 1;
#endif
    if (cspm != built_cspm || (conduction != 0 && conduction != built_conduction)) {
        fprintf(stderr, "scene wants cspm=%d conduction=%d, this build has cspm=%d conduction=%d\n", cspm,
                conduction, built_cspm, built_conduction);
        return 3;
    }

    phys_constants phys;
    phys.E = phys_v[0]; phys.nu = phys_v[1]; phys.rho0 = phys_v[2]; phys.K = phys_v[3]; phys.G = phys_v[4];
    phys.mass = phys_v[5];
    corr_constants corr;
    corr.wdeltap = corr_v[0]; corr.stresseps = corr_v[1]; corr.xspheps = corr_v[2];
    corr.alpha = corr_v[3]; corr.beta = corr_v[4]; corr.eta = corr_v[5];
    joco_constants joco;
    joco.A = joco_v[0]; joco.B = joco_v[1]; joco.C = joco_v[2]; joco.n = joco_v[3]; joco.m = joco_v[4];
    joco.Tmelt = joco_v[5]; joco.Tref = joco_v[6]; joco.eps_dot_ref = joco_v[7]; joco.clamp_temp = joco_v[8];
    trml_constants twp, ttool;
    twp.cp = twp_v[0]; twp.tq = twp_v[1]; twp.k = twp_v[2]; twp.alpha = twp_v[3]; twp.T_init = twp_v[4]; twp.eta = twp_v[5];
    ttool.cp = ttool_v[0]; ttool.tq = ttool_v[1]; ttool.k = ttool_v[2]; ttool.alpha = ttool_v[3];
    ttool.T_init = ttool_v[4]; ttool.eta = ttool_v[5];

    particle_gpu *particles = new particle_gpu(pos.data(), vel.data(), rho.data(), T.data(), h.data(), fixed.data(),
                                               tool_p.data(), n);
    check_cuda_error("particles");
    {
        // identity tag: vel_bc.w travels with each particle through the sort
        // (grid_gpu_green.cu:84,105) and the reference's arithmetic never reads
        // it (only vel_bc.xyz, actions_gpu.cu:471-473); xyz stay 0 as the
        // constructor left them
        std::vector<float4_t> tag(n);
        for (int i = 0; i < n; i++) tag[i] = make_float4_t(0.f, 0.f, 0.f, (float_t)i);
        cudaMemcpy(particles->vel_bc, tag.data(), sizeof(float4_t) * n, cudaMemcpyHostToDevice);
    }
    if (has_S) cudaMemcpy(particles->S, S0.data(), sizeof(mat3x3_t) * n, cudaMemcpyHostToDevice);

    for (auto &t : tools) {
        std::vector<vec3_t> positions;
        std::vector<mesh_triangle> triangles;
        for (size_t k = 0; k < t.verts.size() / 3; k++)
            positions.push_back(vec3_t(t.verts[3 * k], t.verts[3 * k + 1], t.verts[3 * k + 2]));
        // what json_read_triangles produces (json_reader.cpp:73-104): index and vertex ids
        for (size_t k = 0; k < t.tris.size() / 3; k++) {
            mesh_triangle tri;
            tri.idx = (unsigned int)k;
            tri.i1 = t.tris[3 * k]; tri.i2 = t.tris[3 * k + 1]; tri.i3 = t.tris[3 * k + 2];
            triangles.push_back(tri);
        }
        mesh_compute_vertex_normals(triangles, positions);
        float_t avg_h = mesh_average_edge_length(triangles);
        tool_3d *cpu_tool = new tool_3d(triangles, positions, avg_h);
        tool_3d_gpu *gt = new tool_3d_gpu(cpu_tool, vec3_t(t.vel[0], t.vel[1], t.vel[2]), phys, t.alpha);
        gt->set_algorithm_type(t.algorithm == 1 ? tool_3d_gpu::contact_algorithm::exhaustive
                                                : tool_3d_gpu::contact_algorithm::spatial_hashing);
        gt->set_mu(t.mu);
        global_tool.push_back(gt);
    }
    global_time_dt = dt;

    grid_base *grid = new grid_gpu_green(n, make_float3_t(gmin[0], gmin[1], gmin[2]),
                                         make_float3_t(gmax[0], gmax[1], gmax[2]), grid_h);
    global_blanking = new blanking(vec3_t(bmin[0], bmin[1], bmin[2]), vec3_t(bmax[0], bmax[1], bmax[2]), blank_vmax);

    actions_setup_corrector_constants(corr);
    actions_setup_physical_constants(phys);
    if (has_joco) actions_setup_johnson_cook_constants(joco);
    actions_setup_thermal_constants_wp(twp);
    interactions_setup_corrector_constants(corr);
    interactions_setup_physical_constants(phys);
    interactions_setup_thermal_constants_workpiece(twp);
    if (ttool.alpha != 0.f && !global_tool.empty()) {
        actions_setup_thermal_constants_tool(ttool);
        interactions_setup_thermal_constants_tool(ttool, global_tool[0]);
    }
    interactions_setup_geometry_constants(grid);
    global_tool_forces = new tool_forces(global_tool.size());

    leap_frog *stepper = new leap_frog(particles->N_init, grid->num_cell());
    check_cuda_error("setup");

    // main(): no step at index 0, then the clock advances once per index
    global_time_step = 1;
    global_time_current = global_time_dt;
    auto advance = [&](bool record) {
        stepper->step(particles, grid, record);
        global_time_step++;
        global_time_current += global_time_dt;
    };
    for (int s = 0; s < warmup; s++) advance(false);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0);
    for (int s = 0; s < steps; s++) advance(argc > 4 && s == steps - 1);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    check_cuda_error("steps");
    printf("{\"n\": %d, \"active\": %u, \"warmup\": %d, \"steps\": %d, \"ms_per_step\": %.6f, \"cspm\": %d, "
           "\"conduction\": %d}\n",
           n, particles->N, warmup, steps, steps ? ms / steps : 0.f, built_cspm, built_conduction);

    if (argc > 4) {
        FILE *of = fopen(argv[4], "wb");
        if (!of) { fprintf(stderr, "cannot write %s\n", argv[4]); return 2; }
        const particle_gpu &p = *particles;
        std::vector<int> idx(n);
        std::vector<float4_t> tag(n);
        std::vector<float4_t> pos_o(n), vel_o(n);
        std::vector<mat3x3_t> S_o(n), St_o(n), R_o(n);
        std::vector<float_t> rho_o(n), T_o(n), eps_o(n), blk_o(n), rhot_o(n), Tt_o(n);
        std::vector<float3_t> fc_o(n), ft_o(n), post_o(n), velt_o(n);
        cudaMemcpy(tag.data(), p.vel_bc, sizeof(float4_t) * n, cudaMemcpyDeviceToHost);
        for (int i = 0; i < n; i++) idx[i] = (int)tag[i].w;
        cudaMemcpy(pos_o.data(), p.pos, sizeof(float4_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(vel_o.data(), p.vel, sizeof(float4_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(S_o.data(), p.S, sizeof(mat3x3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(rho_o.data(), p.rho, sizeof(float_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(T_o.data(), p.T, sizeof(float_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(eps_o.data(), p.eps_pl, sizeof(float_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(blk_o.data(), p.blanked, sizeof(float_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(fc_o.data(), p.fc, sizeof(float3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(ft_o.data(), p.ft, sizeof(float3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(post_o.data(), p.pos_t, sizeof(float3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(velt_o.data(), p.vel_t, sizeof(float3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(St_o.data(), p.S_t, sizeof(mat3x3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(rhot_o.data(), p.rho_t, sizeof(float_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(R_o.data(), p.R, sizeof(mat3x3_t) * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(Tt_o.data(), p.T_t, sizeof(float_t) * n, cudaMemcpyDeviceToHost);
        std::vector<float3> forces = global_tool_forces->get_forces_host();
        check_cuda_error("read-back");
        const int active = (int)p.N, nt = (int)forces.size();
        put(of, "MFREERS1", 8);
        put(of, &n, 1); put(of, &active, 1); put(of, &nt, 1);
        put(of, idx.data(), n);
        put(of, &pos_o[0].x, 4 * (size_t)n); put(of, &vel_o[0].x, 4 * (size_t)n);
        put(of, &S_o[0][0][0], 9 * (size_t)n);
        put(of, rho_o.data(), n); put(of, T_o.data(), n); put(of, eps_o.data(), n); put(of, blk_o.data(), n);
        put(of, &fc_o[0].x, 3 * (size_t)n); put(of, &ft_o[0].x, 3 * (size_t)n);
        put(of, &post_o[0].x, 3 * (size_t)n); put(of, &velt_o[0].x, 3 * (size_t)n);
        put(of, &St_o[0][0][0], 9 * (size_t)n);
        put(of, rhot_o.data(), n); put(of, Tt_o.data(), n);
        put(of, &R_o[0][0][0], 9 * (size_t)n);
        if (nt) put(of, &forces[0].x, 3 * (size_t)nt);
        fclose(of);
    }
    return 0;
}
