// mfree_contact.cu -- end of the step: rigid-tool contact and the work that
// follows it for the particles inside a tool box.
//
// Reference path replaced (src/leap_frog.cu:173-188):
//   tool_3d_gpu::update_tool + do_update_tool   tool_3d_gpu.cu:74-99,907-948 (vertices
//                                               p_init + v t are formed on the fly)
//   do_compute_contact_forces (spatial hashing, safe) tool_3d_gpu.cu:585-681
//       establish_contact_by_ray / _by_normal, comp_closest_point,
//       triangle_ray_intersect                  tool_3d_gpu.cu:101-444
//   do_compute_contact_forces_n2 (exhaustive)   tool_3d_gpu.cu:455-583
//   tool_forces (atomicAdd)                     tool_3d_gpu.cu:30-69 -- here a
//                                               fixed-order block reduction
//   do_material_fric_heat_gen                   actions_gpu.cu:192-220
//   do_boundary_conditions(_thermal)            actions_gpu.cu:451-487
//   do_move_tool_particles (blanked tail)       actions_gpu.cu:55-68
//
// One thread per particle; only particles inside a tool box do contact work
// (the pair kernel's epilogue has already finished every other particle).
#include "mfree_geom.h"
#include "mfree_kernels.cuh"

namespace mfree {

namespace {

// vector algebra of the contact code on the shared float 3-vector
using V3 = Vec3f;
__device__ __forceinline__ V3 v3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return vadd(a, b); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return vsub(a, b); }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return vscale(s, a); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return vdot(a, b); }
__device__ __forceinline__ V3 cross(V3 a, V3 b) { return vcross(a, b); }
__device__ __forceinline__ float len(V3 a) { return vlength(a); }
__device__ __forceinline__ V3 ld(const float4 *p, int i) {
    float4 v = p[i];
    return {v.x, v.y, v.z};
}

// current vertex p_init + v t (do_update_tool)
__device__ __forceinline__ V3 vert(const ToolDev &T, const float4 *p, int i, float t) {
    float4 v = p[i];
    return {v.x + T.vel[0] * t, v.y + T.vel[1] * t, v.z + T.vel[2] * t};
}

// closest point on triangle k and the normal of the feature it lies on
// (comp_closest_point, tool_3d_gpu.cu:141-212; the geometry is shared with the
// host setup in mfree_geom.h)
__device__ void closest_point(const ToolDev &T, int k, float t, V3 qp, V3 &cp, V3 &np) {
    switch (closest_on_triangle(vert(T, T.p1, k, t), vert(T, T.p2, k, t), vert(T, T.p3, k, t), qp, cp)) {
        case TF_V1: np = ld(T.np1, k); break;
        case TF_V2: np = ld(T.np2, k); break;
        case TF_V3: np = ld(T.np3, k); break;
        case TF_E12: np = ld(T.ne1, k); break;
        case TF_E23: np = ld(T.ne2, k); break;
        case TF_E31: np = ld(T.ne3, k); break;
        default: np = ld(T.n, k); break;
    }
}

// Moller-Trumbore along +z (triangle_ray_intersect, tool_3d_gpu.cu:248-280)
__device__ bool ray_z(const ToolDev &T, int k, float t, V3 o, float &tt) {
    const float EPS = 0.0000001f;
    V3 v0 = vert(T, T.p1, k, t), v1 = vert(T, T.p2, k, t), v2 = vert(T, T.p3, k, t);
    V3 e1 = v1 - v0, e2 = v2 - v0;
    V3 dir = v3(0.f, 0.f, 1.f);
    V3 h = cross(dir, e2);
    float a = dot(e1, h);
    if (a > -EPS && a < EPS) return false;
    float f = 1.f / a;
    V3 s = o - v0;
    float u = f * dot(s, h);
    if (u < 0.f || u > 1.f) return false;
    V3 q = cross(s, e1);
    float v = f * dot(dir, q);
    if (v < 0.f || u + v > 1.f) return false;
    tt = f * dot(e2, q);
    return tt > EPS;
}

__device__ __forceinline__ void unhash(const ToolDev &T, const ToolClock &B, V3 p, int &ix, int &iy, int &iz) {
    // (unsigned int) cast of unhash_pos (tool_3d_gpu.cu:101-107), kept inside the grid
    ix = int(min((unsigned)((p.x - B.bbmin[0]) / T.dx), unsigned(T.nx - 1)));
    iy = int(min((unsigned)((p.y - B.bbmin[1]) / T.dx), unsigned(T.ny - 1)));
    iz = int(min((unsigned)((p.z - B.bbmin[2]) / T.dx), unsigned(T.nz - 1)));
}

// +z ray parity over the tri-grid column (establish_contact_by_ray, :382-444)
__device__ bool inside_by_ray(const ToolDev &T, const ToolClock &B, float t, V3 qp) {
    int ix, iy, iz;
    unhash(T, B, qp, ix, iy, iz);
    unsigned ni = 0;
    for (; iz < T.nz; ++iz) {
        const int box = (ix * T.ny + iy) * T.nz + iz;
        for (int k = T.cells[box]; k < T.cells[box + 1]; k++) {
            float tt;
            if (ray_z(T, k, t, qp, tt)) {
                V3 ip = qp + tt * v3(0.f, 0.f, 1.f);
                float lox = B.bbmin[0] + ix * T.dx, loy = B.bbmin[1] + iy * T.dx, loz = B.bbmin[2] + iz * T.dx;
                float hix = B.bbmin[0] + (ix + 1) * T.dx, hiy = B.bbmin[1] + (iy + 1) * T.dx,
                      hiz = B.bbmin[2] + (iz + 1) * T.dx;
                if (lox <= ip.x && ip.x < hix && loy <= ip.y && ip.y < hiy && loz <= ip.z && ip.z < hiz) ni++;
            }
        }
    }
    return (ni % 2) != 0;
}

// closest triangle by expanding shells until one is non-empty, plus one more
// shell (establish_contact_by_normal, :282-380); bounded by the grid size
__device__ void closest_by_shells(const ToolDev &T, const ToolClock &B, float t, V3 qp, V3 &cp, V3 &nrm,
                                  DevClock *clk) {
    int ix, iy, iz;
    unhash(T, B, qp, ix, iy, iz);
    float md = __int_as_float(0x7f800000);  // DBL_MAX stored in a float
    cp = qp;
    nrm = v3(0.f, 0.f, 0.f);
    int box = (ix * T.ny + iy) * T.nz + iz;
    if (T.cells[box + 1] > T.cells[box] && !bounds_ok(clk, T.cells[box + 1] - 1, T.num_tris)) return;
    bool empty_so_far = T.cells[box] == T.cells[box + 1];
    for (int k = T.cells[box]; k < T.cells[box + 1]; k++) {
        V3 c, n;
        closest_point(T, k, t, qp, c, n);
        V3 d = c - qp;
        float dd = dot(d, d);
        if (dd < md) { md = dd; cp = c; nrm = n; }
    }
    const int cap = max(T.nx, max(T.ny, T.nz)) + 2;
    bool all_done = false;
    int off = 1;
    for (; off <= cap; ) {
        const int li = max(ix - off, 0), lj = max(iy - off, 0), lk = max(iz - off, 0);
        const int hi = min(ix + off + 1, T.nx), hj = min(iy + off + 1, T.ny), hk = min(iz + off + 1, T.nz);
        for (int a = li; a < hi; a++)
            for (int b = lj; b < hj; b++)
                for (int c = lk; c < hk; c++) {
                    bool on = a == li || a == hi - 1 || b == lj || b == hj - 1 || c == lk || c == hk - 1;
                    if (!on) continue;
                    const int bx = (a * T.ny + b) * T.nz + c;
                    if (T.cells[bx + 1] > T.cells[bx] && !bounds_ok(clk, T.cells[bx + 1] - 1, T.num_tris)) continue;
                    for (int k = T.cells[bx]; k < T.cells[bx + 1]; k++) {
                        empty_so_far = false;
                        V3 cc, n;
                        closest_point(T, k, t, qp, cc, n);
                        V3 d = cc - qp;
                        float dd = dot(d, d);
                        if (dd < md) { md = dd; cp = cc; nrm = n; }
                    }
                }
        if (all_done) break;
        off++;
        if (!empty_so_far) all_done = true;
    }
    if (off > cap) atomicAdd(&clk->contact_cap, 1ull);
}

}  // namespace

// one thread per particle; particles of the blanked tail only translate if
// they are tool particles
__device__ __forceinline__ void finalize_body(const StepArgs &a, int bid) {
    const Params &P = a.p;
    const int i = bid * 256 + threadIdx.x;
    const int N = a.clk->n_active;
    const bool rec = a.clk->record != 0;
    const State &S = a.b;
    float fsum[MAX_TOOLS][3];
    if (rec)
        for (int k = 0; k < P.num_tools; k++) fsum[k][0] = fsum[k][1] = fsum[k][2] = 0.f;
    do {
        if (i >= P.n_init) break;
        if (i >= N) {
            const float4 fc = S.fc4[i];
            if (fc.w == 1.f) {
                float4 pos = S.pos4[i];
                if (P.precision) {
                    float4 lo = S.lo4[i];
                    acc_comp(pos.x, lo.x, P.dt, P.tool0_vel[0]);
                    acc_comp(pos.y, lo.y, P.dt, P.tool0_vel[1]);
                    acc_comp(pos.z, lo.z, P.dt, P.tool0_vel[2]);
                    S.lo4[i] = lo;
                } else {
                    pos.x = fmaf(P.tool0_vel[0], P.dt, pos.x);
                    pos.y = fmaf(P.tool0_vel[1], P.dt, pos.y);
                    pos.z = fmaf(P.tool0_vel[2], P.dt, pos.z);
                }
                S.pos4[i] = pos;
            }
            break;
        }
        float4 pos = S.pos4[i];
        float4 fc = S.fc4[i];
        if (fc.w == 1.f) break;  // tool particle
        if (!contact_candidate(a, pos.x, pos.y, pos.z)) break;
        const float t = a.clk->t;
        const float dt = P.dt;
        float4 vel = S.vel4[i], ft = S.ft4[i];
        V3 qp = v3(pos.x, pos.y, pos.z);
        V3 n_last = v3(0.f, 0.f, 0.f);
        for (int k = 0; k < P.num_tools; k++) {
            if (!in_tool_box(a, k, pos.x, pos.y, pos.z)) continue;
            const ToolDev &T = a.tools[k];
            const ToolClock &B = a.clk->tool[k];
            V3 cp, n;
            if (T.hashed) {
                if (!inside_by_ray(T, B, t, qp)) continue;
                closest_by_shells(T, B, t, qp, cp, n, a.clk);
            } else {
                float md = 3.402823466e+38f;  // FLT_MAX
                cp = qp;
                n = v3(0.f, 0.f, 0.f);
                for (int kk = 0; kk < T.num_tris; kk++) {
                    V3 c, nn;
                    closest_point(T, kk, t, qp, c, nn);
                    V3 d = c - qp;
                    float dd = dot(d, d);
                    if (dd < md) { md = dd; cp = c; n = nn; }
                }
                if (dot(cp - qp, n) > 0.f) continue;
            }
            // the reference's operation order, divisions included
            // (tool_3d_gpu.cu:630-661): fN = ((-m gN) n) / dt^2 * alpha,
            // kdeltae = ((alpha m) vr) / dt, fT = (fy fstar) / |fstar|
            const float gN = dot(qp - cp, n);
            const float dt2 = dt * dt;
            const V3 mgn = (-P.mass * gN) * n;
            V3 fN = v3(mgn.x / dt2 * T.alpha, mgn.y / dt2 * T.alpha, mgn.z / dt2 * T.alpha);
            V3 fT = v3(0.f, 0.f, 0.f);
            if (T.mu != 0.f) {
                V3 vm = P.friction_tool_vel ? v3(T.vel[0], T.vel[1], T.vel[2]) : v3(0.f, 0.f, 0.f);
                V3 v = v3(vel.x, vel.y, vel.z) - vm;
                V3 vr = v3(v.x - v.x * n.x, v.y - v.y * n.y, v.z - v.z * n.z);
                const V3 amv = (T.alpha * P.mass) * vr;
                V3 kde = v3(amv.x / dt, amv.y / dt, amv.z / dt);
                float fy = T.mu * len(fN);
                V3 fs = v3(ft.x, ft.y, ft.z) - kde;
                float lfs = len(fs);
                if (lfs > fy) {
                    const V3 ffs = fy * fs;
                    fT = v3(ffs.x / lfs, ffs.y / lfs, ffs.z / lfs);
                } else {
                    fT = fs;
                }
            }
            fc.x = fN.x; fc.y = fN.y; fc.z = fN.z;
            ft.x = fT.x; ft.y = fT.y; ft.z = fT.z;
            n_last = n;
            if (rec) {
                fsum[k][0] += fN.x + fT.x;
                fsum[k][1] += fN.y + fT.y;
                fsum[k][2] += fN.z + fT.z;
            }
        }
        // friction heat (do_material_fric_heat_gen) with the first tool's velocity
        float4 sb = S.sb4[i];
        float T = sb.z;
        if (P.fric_heat) {
            const float fm = sqrtf(ft.x * ft.x + ft.y * ft.y + ft.z * ft.z);
            if (fm != 0.f) {
                const float dx = vel.x - P.tool0_vel[0], dy = vel.y - P.tool0_vel[1], dz = vel.z - P.tool0_vel[2];
                const float dn = dx * n_last.x + dy * n_last.y + dz * n_last.z;
                const float rx = dx - dn, ry = dy - dn, rz = dz - dn;
                const float vm = sqrtf(rx * rx + ry * ry + rz * rz);
                T += P.wp_eta * dt * fm * vm / (P.wp_cp * P.mass);
            }
        }
        // boundary conditions
        const float fixed = S.dsb4[i].w;
        if (fixed != 0.f) {
            const float4 bc = S.bc4[i];
            vel.x = bc.x; vel.y = bc.y; vel.z = bc.z;
            fc.x = fc.y = fc.z = 0.f;
            float4 da = S.da4[i], dv = S.dv4[i];
            da.x = da.y = da.z = 0.f;
            dv.x = dv.y = dv.z = 0.f;
            S.da4[i] = da;
            S.dv4[i] = dv;
            if (P.precision) {
                float4 lo = S.lo4[i], lob = S.lo4b[i];
                lo.w = 0.f; lob.x = lob.y = 0.f;
                S.lo4[i] = lo;
                S.lo4b[i] = lob;
            }
        }
        if (P.thermal && fixed == 1.f) T = P.wp_Tinit;
        sb.z = T;
        S.sb4[i] = sb;
        S.vel4[i] = vel;
        S.fc4[i] = fc;
        S.ft4[i] = ft;
        if (P.diagnostics) a.s.nrm[i] = make_float4(n_last.x, n_last.y, n_last.z, 0.f);
    } while (false);
    if (!rec) return;
    // fixed-order block reduction of the tool forces
    __shared__ float red[8][3 * MAX_TOOLS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < P.num_tools; k++)
        for (int d = 0; d < 3; d++) {
            float v = (i < P.n_init && i < N) ? fsum[k][d] : 0.f;
            for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[warp][3 * k + d] = v;
        }
    __syncthreads();
    if (threadIdx.x < 3 * P.num_tools) {
        float s = 0.f;
        for (int w = 0; w < 8; w++) s += red[w][threadIdx.x];
        a.s.force_part[size_t(bid) * (3 * MAX_TOOLS) + threadIdx.x] = s;
    }
}

// sum of the per-block partials: thread t adds blocks t, t+256, ... in order,
// then a fixed tree over the 256 threads (deterministic for a given grid)
__device__ __forceinline__ void force_final_body(const StepArgs &a, int num_blocks, float *out) {
    if (!a.clk->record) return;
    __shared__ float red[256];
    for (int c = 0; c < 3 * a.p.num_tools; c++) {
        float s = 0.f;
        for (int b = threadIdx.x; b < num_blocks; b += 256) s += a.s.force_part[size_t(b) * (3 * MAX_TOOLS) + c];
        red[threadIdx.x] = s;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[c] = red[0];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) kb_finalize(BatchTable T) {
    const int s = find_scene(T.pblk, T.nscenes, blockIdx.x);
    finalize_body(scene_args(T, s), int(blockIdx.x) - T.pblk[s]);
}
// one block per scene
__global__ void __launch_bounds__(256) kb_force_final(BatchTable T) {
    __shared__ StepArgs sa;
    load_scene_args(sa, T, blockIdx.x);
    __syncthreads();
    if (sa.p.num_tools > 0) force_final_body(sa, (sa.p.n_init + 255) / 256, sa.s.forces);
}

}  // namespace mfree
