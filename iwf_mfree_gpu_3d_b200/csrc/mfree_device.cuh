// mfree_device.cuh -- device-side layout and per-particle physics of the
// B200 SPH cutting step.
//
// HBM layout (all structure-of-arrays, 16-byte float4 records):
//   persistent particle state, two copies (the stable sort gathers copy A
//   into copy B every step, as grid_gpu_green's reorder_data does,
//   grid_gpu_green.cu:72-125):
//     pos4 = (x, y, z, h)          vel4 = (vx, vy, vz, rho)
//     sa4  = (Sxx, Syy, Szz, Sxy)  sb4  = (Sxz, Syz, T, eps_pl)
//     da4  = (xdot, ydot, zdot, rho_t)     dv4 = (vx_t, vy_t, vz_t, T_t)
//     dsa4 = (Sxx_t, Syy_t, Szz_t, Sxy_t)  dsb4 = (Sxz_t, Syz_t, eps_pl_dot, fixed)
//     fc4  = (fc.x, fc.y, fc.z, tool_p)    ft4 = (ft.x, ft.y, ft.z, blanked)
//     bc4  = (vbc.x, vbc.y, vbc.z, id bits)
//     lo4  = (x_lo, y_lo, z_lo, vx_lo), lo4b = (vy_lo, vz_lo, -, -)  [precision form]
//   The deviatoric stress is symmetric in the reference (every writer keeps
//   S[c][r] == S[r][c]: predict/correct element-wise, Jaumann
//   omega*S + S*omega^T, radial return), so 6 components are stored.
//   half-step neighbour records, six float4 (96 bytes) per particle in sorted
//   order, written by the predictor and read by the pair loop: P alone, then
//   V, A, B, R, C interleaved per particle (80 bytes); a halo column is one
//   contiguous range of each of the two, staged into shared memory by two bulk
//   copies:
//     P = (x, y, z, tool_flag)      V = (vx, vy, vz, rho)
//     A = sigma(xx, yy, zz, xy)     B = (sigma_xz, sigma_yz, c = sqrt(K/rho), h)
//     R = R(xx, yy, zz, xy)         C = (R_xz, R_yz, T, m/rho)
//   with sigma = (S - p I)/rho^2 (the per-particle factor of the stress
//   divergence, interactions_gpu.cu:389-399) and R the artificial stress.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "mfree.h"

namespace mfree {

constexpr int MAX_TOOLS = 8;
constexpr int TILE_Z_MAX = 8;  // largest pair-kernel tile depth (cells along z)

// time-varying scalars kept on the device so a step can be replayed from a
// CUDA graph: the clock kernel advances them at the start of every step
struct ToolClock {
    float bbmin[3], bbmax[3];  // tri-grid box, advanced by v*dt per step (tool_3d_gpu.cu:926-932)
};
struct DevClock {
    float t;          // global_time_current used by this step
    int pending;      // 1 once a step has run: the next clock tick adds dt first
    int n_active;     // N (particles not blanked), written by the scan
    int record;       // record tool forces this step
    int staging_timeouts;  // pair-kernel staging waits that ran out (that block left its tiles undone)
    int parity;       // which of the two state copies holds this step's input (flips every step)
    unsigned max_disp;  // float bits: the largest move of a particle in this step's predictor, in cells
                        // (the pair kernel's stencil-pruning margin; reset by the clock kernel every step)
    long long step_index;
    float blank_min[3], blank_max[3];
    float grid_min[3];
    ToolClock tool[MAX_TOOLS];
    // device-detected conditions (mfree_counters)
    unsigned long long secant_failures, out_of_grid, contact_cap, nan_blanked, full_stencil_steps;
    unsigned long long bounds_errors;  // bounds-checked builds: indices from data that fell outside their array
    unsigned long long pse_zero_targets;  // PSE variants: targets of tiles whose PSE sum is exactly zero (all
                                          // staged temperatures equal), run without the PSE terms
};

// Bounds-checked build (-DMFREE_BOUNDS_CHECK, libmfree_checked.so): every
// index computed from data at the places below is tested against its array;
// one outside is counted in the scene's clock and the access is skipped or
// redirected to element 0, so a wrong index shows as a count, not a fault.
// In the normal build the test is constant true and compiles away.
#ifdef MFREE_BOUNDS_CHECK
__device__ __forceinline__ bool bounds_ok(DevClock *clk, long long idx, long long lim) {
    if (idx >= 0 && idx < lim) return true;
    if (clk) atomicAdd(&clk->bounds_errors, 1ull);
    return false;
}
// a range [start, start + len) of an array of lim elements; len 0 is always
// fine
__device__ __forceinline__ bool range_ok(DevClock *clk, long long start, long long len, long long lim) {
    if (len == 0 || (len > 0 && start >= 0 && start + len <= lim)) return true;
    if (clk) atomicAdd(&clk->bounds_errors, 1ull);
    return false;
}
#else
__device__ __forceinline__ constexpr bool bounds_ok(DevClock *, long long, long long) { return true; }
__device__ __forceinline__ constexpr bool range_ok(DevClock *, long long, long long, long long) { return true; }
#endif

struct ToolDev {
    // boxed (hashed) or all (exhaustive) triangles, SoA of float4 (x, y, z, -)
    const float4 *p1, *p2, *p3;           // initial vertices (p_init)
    const float4 *n, *np1, *np2, *np3, *ne1, *ne2, *ne3;
    const int *cells;                     // CSR offsets (hashed), num_cell + 1
    int num_tris;                         // triangles in p1.. (boxed count or total)
    int nx, ny, nz;
    float dx;
    float vel[3];
    float alpha, mu;
    int hashed;                           // 1: spatial hashing with ray parity (safe), 0: exhaustive
    float birth, death;
};

struct Params {
    // physics (phys_constants)
    float mass, K, G, rho0, c0sq;  // c0sq = sqrtf(K/rho0)^2 as do_material_eos computes it
    // correctors (corr_constants)
    float wdeltap, stresseps, xspheps, av_alpha, av_beta, av_eta;
    float inv_wdeltap;  // 1 / wdeltap (0 when artificial stress is off)
    // thermal
    float wp_alpha, wp_cp, wp_tq, wp_Tinit, wp_eta, tool_alpha;
    int thermal;       // m_thermal of actions_gpu.cu: workpiece or tool diffusivity != 0
    int fric_heat;     // workpiece eta != 0
    // Johnson-Cook (joco_constants)
    float jc_A, jc_B, jc_C, jc_n, jc_m, jc_Tmelt, jc_Tref, jc_epsdot_ref, jc_clamp;
    int plastic, max_secant_iter;
    // options
    int cspm, conduction, precision, diagnostics, friction_tool_vel;
    // grid (geom_constants)
    int gnx, gny, gnz, num_cell;
    float gdx;
    float grid_vel[3], grid_min0[3];
    int grid_moving;
    // blanking
    int blank_on;
    float blank_min0[3], blank_max0[3], blank_vel[3], vmax2;
    // time
    float dt;
    int n_init;
    int num_tools;
    float tool0_vel[3];  // global_tool[0]->get_vel(): friction heat and tool particles
    int record_every;
    int tile_z;  // cells per pair-kernel tile along z (1..TILE_Z_MAX)
    int stage_extra;  // bytes added to the staging byte count: nonzero only to make the waits run out (tests)
    int full_stencil;  // 1: the pair kernel visits every stencil candidate (no geometric pruning)
};

// Geometric pruning of the pair kernel's stencil (variants without PSE): a
// candidate lies in the cell its position at the hash gave it, moved by the
// predictor.  The predictor records the step's largest move per axis (in
// cells); the pair kernel widens every cell by that plus PRUNE_SLACK, which
// covers the rounding of the hash and of the distance arithmetic (~1e-7
// relative, against ~4e-3 cells).  A move beyond PRUNE_DISP_MAX cells (or a
// NaN) switches the step to the full stencil.
constexpr float PRUNE_DISP_MAX = 0.25f;
constexpr float PRUNE_SLACK = 1.0f / 256.0f;

struct State {
    float4 *pos4, *vel4, *sa4, *sb4, *da4, *dv4, *dsa4, *dsb4, *fc4, *ft4, *bc4, *lo4, *lo4b;
};

struct Rec {
    float4 P, V, A, B, R, C;
};
enum { REC_P = 0, REC_V, REC_A, REC_B, REC_R, REC_C, REC_N };

// One allocation of REC_N * n_init float4: the P records at f[REC_P] = base
// (stride 1), then the other five interleaved per particle, f[k] = base +
// n_init + (k - 1) with stride REC_X; particle i's record k is
// f[k][i * rec_stride(k)].
constexpr int REC_X = REC_N - 1;
__host__ __device__ constexpr int rec_stride(int k) { return k == REC_P ? 1 : REC_X; }
struct Records {
    float4 *f[REC_N];
};

struct Scratch {
    unsigned *key;         // cell id per particle (num_cell = blanked), current order
    unsigned *key_sorted;  // cell id in sorted order
    int *perm;             // sorted position -> previous position
    int *count;            // num_cell + 1 counters
    int *first;            // exclusive scan of count: num_cell + 2 entries
    int *tile_sum;         // per-tile sums of the scan
    int *blank_block;      // blanked particles per hash block, scanned in place
    int *nnb;              // neighbour counts (diagnostics)
    float4 *pos_half;      // half-step positions (diagnostics)
    float4 *nrm;           // contact normal (diagnostics)
    float *force_part;     // per-block partial tool forces (3 per tool per block)
    float *forces;         // per-tool force of the last recorded step (3 per tool)
};

struct alignas(16) StepArgs {
    Params p;
    State a, b;   // a = state before the sort, b = sorted state
    Records r;
    Scratch s;
    DevClock *clk;
    ToolDev tools[MAX_TOOLS];
};

// ------------------------------------------------------------- helpers ----

__device__ __forceinline__ bool nan_or_inf(float v) { return isnan(v) || isinf(v); }

// r^2 in the unfused order ((dx*dx + dy*dy) + dz*dz): the neighbour-count
// definition shared with the oracle
__device__ __forceinline__ float dist2_rn(float dx, float dy, float dz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}
// 1e-8 <= r^2 < 4 h^2 (kernels.cuh:41); the reference compares the float r^2
// with the double literal 1e-8, i.e. r^2 > 9.99999994e-9f (largest float below 1e-8)
__device__ __forceinline__ bool in_support(float r2, float h) {
    float four_h2 = __fmul_rn(__fmul_rn(4.0f, h), h);
    return !(r2 >= four_h2) && (r2 > 9.99999994e-9f);
}

// ------------------------------------------------------ eigen solver ----
// Eberly's robust symmetric 3x3 eigensolver with the branch choices of
// src/eigen_solver.cu:19-302 (eigenvalues ascending, right-handed vectors).
struct Eig3 {
    float l0, l1, l2;
    float3 e1, e2, e3;
};

__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 scale3(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }

__device__ inline float3 eig_vec0(float a00, float a01, float a02, float a11, float a12, float a22, float ev) {
    float3 r0 = make_float3(a00 - ev, a01, a02), r1 = make_float3(a01, a11 - ev, a12),
           r2 = make_float3(a02, a12, a22 - ev);
    float3 c01 = cross3(r0, r1), c02 = cross3(r0, r2), c12 = cross3(r1, r2);
    float d0 = dot3(c01, c01), d1 = dot3(c02, c02), d2 = dot3(c12, c12);
    float dmax = d0;
    int imax = 0;
    if (d1 > dmax) { dmax = d1; imax = 1; }
    if (d2 > dmax) imax = 2;
    float3 c = imax == 0 ? c01 : (imax == 1 ? c02 : c12);
    float d = imax == 0 ? d0 : (imax == 1 ? d1 : d2);
    return scale3(1.0f / sqrtf(d), c);
}
__device__ inline float3 eig_vec1(float a00, float a01, float a02, float a11, float a12, float a22, float3 w,
                                  float ev) {
    float3 U;
    if (fabsf(w.x) > fabsf(w.y)) {
        float il = 1.0f / sqrtf(w.x * w.x + w.z * w.z);
        U = make_float3(-w.z * il, 0.f, w.x * il);
    } else {
        float il = 1.0f / sqrtf(w.y * w.y + w.z * w.z);
        U = make_float3(0.f, w.z * il, -w.y * il);
    }
    float3 V = cross3(w, U);
    float3 AU = make_float3(a00 * U.x + a01 * U.y + a02 * U.z, a01 * U.x + a11 * U.y + a12 * U.z,
                            a02 * U.x + a12 * U.y + a22 * U.z);
    float3 AV = make_float3(a00 * V.x + a01 * V.y + a02 * V.z, a01 * V.x + a11 * V.y + a12 * V.z,
                            a02 * V.x + a12 * V.y + a22 * V.z);
    float m00 = dot3(U, AU) - ev, m01 = dot3(U, AV), m11 = dot3(V, AV) - ev;
    float am00 = fabsf(m00), am01 = fabsf(m01), am11 = fabsf(m11);
    if (am00 >= am11) {
        if (fmaxf(am00, am01) > 0.f) {
            if (am00 >= am01) {
                m01 /= m00;
                m00 = 1.0f / sqrtf(1.0f + m01 * m01);
                m01 *= m00;
            } else {
                m00 /= m01;
                m01 = 1.0f / sqrtf(1.0f + m00 * m00);
                m00 *= m01;
            }
            return make_float3(m01 * U.x - m00 * V.x, m01 * U.y - m00 * V.y, m01 * U.z - m00 * V.z);
        }
        return U;
    }
    if (fmaxf(am11, am01) > 0.f) {
        if (am11 >= am01) {
            m01 /= m11;
            m11 = 1.0f / sqrtf(1.0f + m01 * m01);
            m01 *= m11;
        } else {
            m11 /= m01;
            m01 = 1.0f / sqrtf(1.0f + m11 * m11);
            m11 *= m01;
        }
        return make_float3(m11 * U.x - m01 * V.x, m11 * U.y - m01 * V.y, m11 * U.z - m01 * V.z);
    }
    return U;
}
__device__ inline Eig3 solve_eigen3(float a00, float a01, float a02, float a11, float a12, float a22) {
    Eig3 o;
    float mx = fmaxf(fmaxf(fmaxf(fabsf(a00), fabsf(a01)), fmaxf(fabsf(a02), fabsf(a11))),
                     fmaxf(fabsf(a12), fabsf(a22)));
    o.e1 = make_float3(1.f, 0.f, 0.f);
    o.e2 = make_float3(0.f, 1.f, 0.f);
    o.e3 = make_float3(0.f, 0.f, 1.f);
    if (mx < 9.99999994e-9f || !(mx == mx)) {  // maxAbsElement < 1e-8
        o.l0 = o.l1 = o.l2 = 0.f;
        if (!(mx == mx)) o.l0 = o.l1 = o.l2 = mx;
        return o;
    }
    float inv = 1.0f / mx;
    a00 *= inv; a01 *= inv; a02 *= inv; a11 *= inv; a12 *= inv; a22 *= inv;
    float off = a01 * a01 + a02 * a02 + a12 * a12;
    if (off > 0.f) {
        float q = (a00 + a11 + a22) / 3.0f;
        float b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
        float p = sqrtf((b00 * b00 + b11 * b11 + b22 * b22 + off * 2.0f) / 6.0f);
        float c00 = b11 * b22 - a12 * a12;
        float c01 = a01 * b22 - a12 * a02;
        float c02 = a01 * a12 - b11 * a02;
        float det = (b00 * c00 - a01 * c01 + a02 * c02) / (p * p * p);
        float half = fminf(fmaxf(det * 0.5f, -1.0f), 1.0f);
        float ang = acosf(half) / 3.0f;
        float beta2 = cosf(ang) * 2.0f;
        float beta0 = cosf(ang + 2.09439510239319549f) * 2.0f;
        float beta1 = -(beta0 + beta2);
        o.l0 = q + p * beta0;
        o.l1 = q + p * beta1;
        o.l2 = q + p * beta2;
        if (half >= 0.f) {
            o.e3 = eig_vec0(a00, a01, a02, a11, a12, a22, o.l2);
            o.e2 = eig_vec1(a00, a01, a02, a11, a12, a22, o.e3, o.l1);
            o.e1 = cross3(o.e2, o.e3);
        } else {
            o.e1 = eig_vec0(a00, a01, a02, a11, a12, a22, o.l0);
            o.e2 = eig_vec1(a00, a01, a02, a11, a12, a22, o.e1, o.l1);
            o.e3 = cross3(o.e1, o.e2);
        }
    } else {
        o.l0 = a00;
        o.l1 = a11;
        o.l2 = a22;
    }
    o.l0 *= mx;
    o.l1 *= mx;
    o.l2 *= mx;
    return o;
}

// artificial stress of do_corrector_artificial_stress (actions_gpu.cu:70-132):
// Rot has the eigenvectors as rows, so R = Rot diag(lambda') Rot^T, i.e.
// R(r,c) = sum_k e_r[k] lambda'_k e_c[k] with lambda' = -eps*max(lambda,0)/rho^2.
// Output order (xx, yy, zz, xy, xz, yz).
__device__ inline void artificial_stress(float sxx, float syy, float szz, float sxy, float sxz, float syz, float p,
                                         float rho, float eps, float out[6]) {
    Eig3 e = solve_eigen3(sxx - p, sxy, sxz, syy - p, syz, szz - p);
    float rhoi21 = 1.0f / (rho * rho);
    float l[3] = {e.l0, e.l1, e.l2};
#pragma unroll
    for (int k = 0; k < 3; k++) l[k] = l[k] > 0.f ? -eps * l[k] * rhoi21 : 0.f;
    const float3 E[3] = {e.e1, e.e2, e.e3};
    auto comp = [&](int a, int k) { return k == 0 ? E[a].x : (k == 1 ? E[a].y : E[a].z); };
    auto Rrc = [&](int r, int c) {
        return comp(r, 0) * l[0] * comp(c, 0) + comp(r, 1) * l[1] * comp(c, 1) + comp(r, 2) * l[2] * comp(c, 2);
    };
    out[0] = Rrc(0, 0);
    out[1] = Rrc(1, 1);
    out[2] = Rrc(2, 2);
    out[3] = Rrc(0, 1);
    out[4] = Rrc(0, 2);
    out[5] = Rrc(1, 2);
}

// ------------------------------------------------------- Johnson-Cook ----
// sigma_yield / opt_fun / solve_secant (plasticity.cuh:28-93), evaluated the
// way the reference's FP32 build evaluates them: in FP64, from FP32 inputs,
// with the strain-rate logarithm taken as logf and multiplied by C in float
// (log_t = logf in types.h).  The secant stops on an absolute change of the
// plastic multiplier below 1e-6; in FP32 its finite-difference slope at the
// starting multiplier of 1e-8 is below the resolution of g and the iterates part
// from the FP64 ones (the plastic strain of a loaded state differed by 2-3 %
// after one step), so the root is solved in FP64.  Only yielding particles
// reach it.
__device__ __forceinline__ double jc_sigma_yield(const Params &P, double eps_pl, double eps_pl_dot, double T) {
    const double theta = (T - (double)P.jc_Tref) / (double)(P.jc_Tmelt - P.jc_Tref);
    const double a = (double)P.jc_A + (double)P.jc_B * pow(eps_pl, (double)P.jc_n);
    const double ed = eps_pl_dot / (double)P.jc_epsdot_ref;
    const double b = ed > 1.0 ? 1.0 + (double)(P.jc_C * logf((float)ed)) : pow(1.0 + ed, (double)P.jc_C);
    const double c = 1.0 - pow(theta, (double)P.jc_m);
    return a * b * c;
}
__device__ __forceinline__ double jc_opt(const Params &P, double dl, double normS, double eps0, double T, double dt) {
    const double s23 = 0.81649658092772603;  // sqrt(2/3) in double
    const double dlp = fmax(dl, 0.0);
    return normS - 2.0 * (double)P.G * dl - s23 * jc_sigma_yield(P, eps0 + s23 * dlp, s23 * dlp / dt, T);
}
// out of line: its FP64 registers stay out of the calling kernel's allocation
static __device__ __noinline__ double jc_secant(const Params &P, double init, double normS, double eps0, double T,
                                         double dt, int *failed) {
    double dl = init;
    for (int iter = 0;; iter++) {
        const double g = jc_opt(P, dl, normS, eps0, T, dt);
        const double dl1 = dl * 1.01;
        const double g1 = jc_opt(P, dl1, normS, eps0, T, dt);
        const double slope = (g - g1) / (dl - dl1);
        const double old = dl;
        dl = dl - g / slope;
        if (dl < 0.0) dl = -0.1 * dl;
        if (fabs(dl - old) < 1e-6) return dl;
        if (iter > P.max_secant_iter) {
            *failed = 1;
            return dl;
        }
    }
}
static __device__ __noinline__ float jc_yield_stress(const Params &P, float eps_pl, float eps_pl_dot, float T) {
    return (float)jc_sigma_yield(P, eps_pl, eps_pl_dot, T);
}
// the same yield stress in FP32, only to screen out the clearly elastic
// particles before the FP64 evaluation: its relative error is below 1e-4 even
// next to the melting temperature (1 - theta^m ~ 7e-4 at the clamp), so a von
// Mises stress under 0.99 of it is under the FP64 value as well
__device__ __forceinline__ float jc_yield_stress_screen(const Params &P, float eps_pl, float eps_pl_dot, float T) {
    const float theta = (T - P.jc_Tref) / (P.jc_Tmelt - P.jc_Tref);
    const float a = P.jc_A + P.jc_B * powf(eps_pl, P.jc_n);
    const float ed = eps_pl_dot / P.jc_epsdot_ref;
    const float b = ed > 1.0f ? 1.0f + P.jc_C * logf(ed) : powf(1.0f + ed, P.jc_C);
    const float c = 1.0f - powf(theta, P.jc_m);
    return a * b * c;
}

// A first screen without powf or logf, for the particles far below yield
// (most of a cutting scene): with A > 0, B, C >= 0, eps_pl, eps_pl_dot >= 0
// and 0 <= theta < 1 the yield stress is at least A (1 - theta^m) (the strain
// and rate factors are at least 1), and theta^m is bounded from above by the
// approximate exp2/log2 pair inflated by 1e-3.  A von Mises stress under 0.98
// of that bound is under 0.99 of jc_yield_stress_screen as well (its FP32
// rounding and the bound's error stay far inside the 1 % between 0.98 and
// 0.99 while 1 - theta^m >= 1e-3), so the particle is elastic by the same
// test as before and its results are the same bits.
__device__ __forceinline__ bool jc_clearly_elastic(const Params &P, float svm, float eps_pl, float eps_pl_dot, float T) {
    const float theta = (T - P.jc_Tref) / (P.jc_Tmelt - P.jc_Tref);
    if (!(P.jc_A > 0.f && P.jc_B >= 0.f && P.jc_C >= 0.f && P.jc_m > 0.f && P.jc_epsdot_ref > 0.f && eps_pl >= 0.f &&
          eps_pl_dot >= 0.f && theta >= 0.f && theta < 1.f))
        return false;
    float l2, p;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"(theta));  // theta = 0: -inf, and p = 0
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(p) : "f"(P.jc_m * l2));
    const float c = 1.0f - 1.001f * p;
    return c >= 1e-3f && svm < 0.98f * P.jc_A * c;
}

// Jaumann stress rate (actions_gpu.cu:134-190): S_t = 2G(epsdot - tr/3 I) + W S + S W^T,
// L[a][b] = d v_a / d x_b, W(r,c) = (L_rc - L_cr)/2.  In/out order (xx, yy, zz, xy, xz, yz).
__device__ __forceinline__ void jaumann(const float L[9], const float S[6], float G, float out[6]) {
    float e00 = L[0], e11 = L[4], e22 = L[8];
    float e01 = 0.5f * (L[1] + L[3]), e02 = 0.5f * (L[2] + L[6]), e12 = 0.5f * (L[5] + L[7]);
    float w01 = 0.5f * (L[1] - L[3]), w02 = 0.5f * (L[2] - L[6]), w12 = 0.5f * (L[5] - L[7]);
    // W = [[0, w01, w02], [-w01, 0, w12], [-w02, -w12, 0]]
    float s00 = S[0], s11 = S[1], s22 = S[2], s01 = S[3], s02 = S[4], s12 = S[5];
    // A = W S
    float A00 = w01 * s01 + w02 * s02;
    float A01 = w01 * s11 + w02 * s12;
    float A02 = w01 * s12 + w02 * s22;
    float A10 = -w01 * s00 + w12 * s02;
    float A11 = -w01 * s01 + w12 * s12;
    float A12 = -w01 * s02 + w12 * s22;
    float A20 = -w02 * s00 - w12 * s01;
    float A21 = -w02 * s01 - w12 * s11;
    float A22 = -w02 * s02 - w12 * s12;
    float tr3 = (e00 + e11 + e22) * (1.0f / 3.0f);
    float g2 = 2.0f * G;
    out[0] = g2 * (e00 - tr3) + 2.f * A00;
    out[1] = g2 * (e11 - tr3) + 2.f * A11;
    out[2] = g2 * (e22 - tr3) + 2.f * A22;
    out[3] = g2 * e01 + (A01 + A10);
    out[4] = g2 * e02 + (A02 + A20);
    out[5] = g2 * e12 + (A12 + A21);
}

// compensated (hi, lo) += d, d = dt * rate with its product error
__device__ __forceinline__ void acc_comp(float &hi, float &lo, float dt, float rate) {
    float d = dt * rate;
    float de = fmaf(dt, rate, -d);
    float s = hi + d;
    float bb = s - hi;
    float err = (hi - (s - bb)) + (d - bb);
    float l = lo + (de + err);
    float h2 = s + l;
    lo = l - (h2 - s);
    hi = h2;
}

}  // namespace mfree
