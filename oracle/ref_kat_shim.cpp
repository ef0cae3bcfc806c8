// ref_kat_shim.cpp -- TEST INFRASTRUCTURE: exposes functions of the reference
// (iwf_mfree_gpu_3d) compiled unchanged, for the host, from its read-only
// sources, so that the oracle's restatements can be checked against them:
//   cubic_spline, lapl_pse            src/kernels.cuh:26-92
//   solve_eigen                       src/eigen_solver.cu:212-302
//   sigma_yield, solve_secant         src/plasticity.cuh:28-93
// These are __device__ / __host__ __device__ functions without texture or GLM
// use; oracle/build_ref.sh defines __device__ and __host__ empty so that g++
// compiles them as host code (the reference's FP32 build, float_t = float).
#include <cmath>
#include <cfloat>
#include "constants_structs.h"
#include "kernels.cuh"
#include "eigen_solver.cu"
#include "plasticity.cuh"

extern "C" {
void ref_cubic_spline(const float *pi, const float *pj, float h, float *w4) {
    float4 a = make_float4(pi[0], pi[1], pi[2], 0.f), b = make_float4(pj[0], pj[1], pj[2], 0.f);
    float4 w = cubic_spline(a, b, h);
    w4[0] = w.x; w4[1] = w.y; w4[2] = w.z; w4[3] = w.w;
}
float ref_lapl_pse(const float *pi, const float *pj, float h) {
    float4 a = make_float4(pi[0], pi[1], pi[2], 0.f), b = make_float4(pj[0], pj[1], pj[2], 0.f);
    return lapl_pse(a, b, h);
}
// a = a00 a01 a02 a11 a12 a22; out = eval, e1, e2, e3
void ref_solve_eigen(const float *a, float *out) {
    float3 ev, e1, e2, e3;
    solve_eigen(a[0], a[1], a[2], a[3], a[4], a[5], ev, e1, e2, e3);
    float3 v[4] = {ev, e1, e2, e3};
    for (int k = 0; k < 4; k++) { out[3 * k] = v[k].x; out[3 * k + 1] = v[k].y; out[3 * k + 2] = v[k].z; }
}
static joco_constants mk(const float *j) {
    joco_constants c;
    c.A = j[0]; c.B = j[1]; c.C = j[2]; c.n = j[3]; c.m = j[4]; c.Tmelt = j[5]; c.Tref = j[6];
    c.eps_dot_ref = j[7]; c.clamp_temp = j[8];
    return c;
}
double ref_sigma_yield(const float *jc, double eps, double epsd, double t) { return sigma_yield(mk(jc), eps, epsd, t); }
double ref_solve_secant(const float *jc, double init, double tol, double normS, double eps0, double t, double dt,
                        double mu, int *failed) {
    bool f = false;
    double r = solve_secant(mk(jc), init, tol, normS, eps0, t, dt, mu, f);
    *failed = f;
    return r;
}
}
