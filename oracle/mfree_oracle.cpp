// mfree_oracle.cpp -- CPU oracle for the SPH cutting step.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU, the algorithm of
// leap_frog::step of iwf_mfree_gpu_3d (src/leap_frog.cu:121-195) and of every
// kernel it launches, quirks included, so that the CUDA path can be checked
// against it.  Only the tests, the smoke check and the CPU-baseline leg of the
// benchmark load it; the product never does.
//
// Two instantiations:
//   double : the FP64 restatement ("USE_DOUBLE" semantics, src/types.h:32-62)
//            used for the per-field relative-L2 parity checks;
//   float  : the reference's FP32 build semantics (including the places where
//            the reference computes in double inside a float build), used for
//            tight one-step checks.
// The integer pipeline (cell hash, stable sort, cell ranges, neighbour counts)
// is also exported in FP32 for the bit-exact checks (hash_fp32, sort_cells,
// neighbour_counts_fp32).
//
// Pinning: the kernel function, the eigen solver and the Johnson-Cook secant
// are compared against the reference's own functions compiled on the host from
// the read-only sources (oracle/build_ref.sh -> oracle/_ref/libref_kat.so).
// The GLM-dependent parts (artificial-stress rotation, Jaumann rate, CSPM
// inverse, contact vector algebra) are restated from GLM's documented
// column-major semantics and are not pinned by a reference run: GLM is not
// installed and the reference GPU code does not compile with CUDA 12.
//
// The third-party algorithm used by the reference's eigen solver is David
// Eberly's published "robust eigensolver for 3x3 symmetric matrices"
// (Geometric Tools 3.0.2, the version the reference cites in
// src/eigen_solver.cu); the triangle/box overlap test is Akenine-Moller's
// published separating-axis test (cited in src/surface_tri_mesh.cpp:151-152);
// the ray test is Moller-Trumbore.  All three are restated here from their
// published descriptions with the reference's choices of branches.

#include "mfree.h"

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------- math ----
template <class R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    R &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class R> V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> V3<R> operator*(V3<R> a, R s) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> V3<R> operator/(V3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> V3<R> cmul(V3<R> a, V3<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> bool operator==(V3<R> a, V3<R> b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
template <class R> R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class R> R length(V3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> V3<R> normalize(V3<R> a) { return a * (R(1) / std::sqrt(dot(a, a))); }

// 3x3 matrix stored as GLM does: m[col][row].
template <class R> struct M3 {
    R m[3][3];
    M3() { std::memset(m, 0, sizeof(m)); }
    explicit M3(R d) { std::memset(m, 0, sizeof(m)); m[0][0] = m[1][1] = m[2][2] = d; }
    R *operator[](int c) { return m[c]; }
    const R *operator[](int c) const { return m[c]; }
};
// element (row r, col c) = m[c][r]; product in the usual mathematical sense
template <class R> M3<R> mul(const M3<R> &a, const M3<R> &b) {
    M3<R> o;
    for (int c = 0; c < 3; c++)
        for (int r = 0; r < 3; r++) o.m[c][r] = a.m[0][r] * b.m[c][0] + a.m[1][r] * b.m[c][1] + a.m[2][r] * b.m[c][2];
    return o;
}
template <class R> M3<R> transpose(const M3<R> &a) {
    M3<R> o;
    for (int c = 0; c < 3; c++)
        for (int r = 0; r < 3; r++) o.m[c][r] = a.m[r][c];
    return o;
}
// determinant / inverse: cofactor expansion over the first column of the
// mathematical matrix A(r,c) = m[c][r]
template <class R> R determinant(const M3<R> &a) {
    auto A = [&](int r, int c) { return a.m[c][r]; };
    return A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) - A(1, 0) * (A(0, 1) * A(2, 2) - A(0, 2) * A(2, 1)) +
           A(2, 0) * (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1));
}
template <class R> M3<R> inverse(const M3<R> &a) {
    auto A = [&](int r, int c) { return a.m[c][r]; };
    R inv_det = R(1) / determinant(a);
    M3<R> o;  // o(r,c) = cofactor(c,r)/det
    auto cof = [&](int r, int c) {
        int r0 = (r + 1) % 3, r1 = (r + 2) % 3, c0 = (c + 1) % 3, c1 = (c + 2) % 3;
        return A(r0, c0) * A(r1, c1) - A(r0, c1) * A(r1, c0);
    };
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) o.m[c][r] = cof(c, r) * inv_det;
    return o;
}

// ------------------------------------------------------- kernel function ----
// cubic_spline (src/kernels.cuh:26-69): value and gradient of the 3-D cubic
// B-spline with support 2h; zero if r^2 >= 4h^2 or r^2 < 1e-8.
template <class R> struct W4 { R w, wx, wy, wz; };
template <class R> inline bool in_support(R rr2, R h) {
    return !(rr2 >= 4 * h * h || double(rr2) < 1e-8);
}
template <class R> W4<R> cubic_spline(R xi, R yi, R zi, R xj, R yj, R zj, R hi) {
    W4<R> o{0, 0, 0, 0};
    R xij = xi - xj, yij = yi - yj, zij = zi - zj;
    R rr2 = xij * xij + yij * yij + zij * zij;
    R h1 = 1 / hi;
    R fourh2 = 4 * hi * hi;
    if (rr2 >= fourh2 || double(rr2) < 1e-8) return o;
    R rad = std::sqrt(rr2);
    R q = rad * h1;
    // the literals are double: the reference's float build evaluates these
    // sub-expressions in double and rounds on assignment
    using D = double;
    R fac = R(M_1_PI * D(h1) * D(h1) * D(h1));
    R val, der;
    if (q > 1) {
        R t = 2 - q, t2 = t * t;
        val = R(0.25 * D(t2) * D(t));
        der = R(-0.75 * D(t2) * D(h1) / D(rad));
    } else {
        val = R(1 - 1.5 * D(q) * D(q) * (1 - 0.5 * D(q)));
        der = R(-3.0 * D(q) * (1 - 0.75 * D(q)) * D(h1) / D(rad));
    }
    o.w = val * fac;
    o.wx = der * xij * fac;
    o.wy = der * yij * fac;
    o.wz = der * zij * fac;
    return o;
}
// lapl_pse (src/kernels.cuh:71-92): Gaussian PSE weight 4/(h^5 pi^1.5) exp(-r^2/h^2)
template <class R> R lapl_pse(R xi, R yi, R zi, R xj, R yj, R zj, R hi) {
    R xij = xi - xj, yij = yi - yj, zij = zi - zj;
    R xx = std::sqrt(xij * xij + yij * yij + zij * zij);
    R h2 = hi * hi, h4 = h2 * h2, h5 = hi * h4;
    return R(4. / (double(h5) * M_PI * std::sqrt(M_PI)) * std::exp(double(-xx * xx / h2)));
}
// PSE in the FP32 build evaluates 4./(h5*M_PI*sqrt(M_PI))*exp(...) in double
// (the literals are double); the FP64 instantiation is all double anyway.

// ---------------------------------------------------------- eigen solver ----
// Eberly's robust eigensolver for symmetric 3x3 (as used by
// do_corrector_artificial_stress, src/eigen_solver.cu:212-302): eigenvalues in
// ascending order, right-handed orthonormal eigenvectors, same branch choices.
template <class R> struct Eig { V3<R> eval, e1, e2, e3; };

template <class R> static void orth_complement(V3<R> W, V3<R> &U, V3<R> &V) {
    if (std::fabs(W.x) > std::fabs(W.y)) {
        R il = R(1) / std::sqrt(W.x * W.x + W.z * W.z);
        U = V3<R>(-W.z * il, R(0), W.x * il);
    } else {
        R il = R(1) / std::sqrt(W.y * W.y + W.z * W.z);
        U = V3<R>(R(0), W.z * il, -W.y * il);
    }
    V = cross(W, U);
}
template <class R> static V3<R> eigvec0(R a00, R a01, R a02, R a11, R a12, R a22, R ev) {
    V3<R> r0(a00 - ev, a01, a02), r1(a01, a11 - ev, a12), r2(a02, a12, a22 - ev);
    V3<R> c01 = cross(r0, r1), c02 = cross(r0, r2), c12 = cross(r1, r2);
    R d0 = dot(c01, c01), d1 = dot(c02, c02), d2 = dot(c12, c12);
    R dmax = d0;
    int imax = 0;
    if (d1 > dmax) { dmax = d1; imax = 1; }
    if (d2 > dmax) imax = 2;
    V3<R> c = imax == 0 ? c01 : (imax == 1 ? c02 : c12);
    R d = imax == 0 ? d0 : (imax == 1 ? d1 : d2);
    R inv = R(1) / std::sqrt(d);
    return c * inv;
}
template <class R> static V3<R> eigvec1(R a00, R a01, R a02, R a11, R a12, R a22, V3<R> e0, R ev) {
    V3<R> U, V;
    orth_complement(e0, U, V);
    V3<R> AU(a00 * U.x + a01 * U.y + a02 * U.z, a01 * U.x + a11 * U.y + a12 * U.z, a02 * U.x + a12 * U.y + a22 * U.z);
    V3<R> AV(a00 * V.x + a01 * V.y + a02 * V.z, a01 * V.x + a11 * V.y + a12 * V.z, a02 * V.x + a12 * V.y + a22 * V.z);
    R m00 = U.x * AU.x + U.y * AU.y + U.z * AU.z - ev;
    R m01 = U.x * AV.x + U.y * AV.y + U.z * AV.z;
    R m11 = V.x * AV.x + V.y * AV.y + V.z * AV.z - ev;
    R am00 = std::fabs(m00), am01 = std::fabs(m01), am11 = std::fabs(m11);
    if (am00 >= am11) {
        R mx = std::max(am00, am01);
        if (mx > R(0)) {
            if (am00 >= am01) {
                m01 /= m00;
                m00 = R(1) / std::sqrt(R(1) + m01 * m01);
                m01 *= m00;
            } else {
                m00 /= m01;
                m01 = R(1) / std::sqrt(R(1) + m00 * m00);
                m00 *= m01;
            }
            return m01 * U - m00 * V;
        }
        return U;
    }
    R mx = std::max(am11, am01);
    if (mx > R(0)) {
        if (am11 >= am01) {
            m01 /= m11;
            m11 = R(1) / std::sqrt(R(1) + m01 * m01);
            m01 *= m11;
        } else {
            m11 /= m01;
            m01 = R(1) / std::sqrt(R(1) + m11 * m11);
            m11 *= m01;
        }
        return m11 * U - m01 * V;
    }
    return U;
}
template <class R> Eig<R> solve_eigen(R a00, R a01, R a02, R a11, R a12, R a22) {
    Eig<R> o;
    R mx = std::max(std::max(std::max(std::fabs(a00), std::fabs(a01)), std::max(std::fabs(a02), std::fabs(a11))),
                    std::max(std::fabs(a12), std::fabs(a22)));
    if (double(mx) < 1e-8) {
        o.eval = V3<R>(0, 0, 0);
        o.e1 = V3<R>(1, 0, 0); o.e2 = V3<R>(0, 1, 0); o.e3 = V3<R>(0, 0, 1);
        return o;
    }
    R inv = R(1) / mx;
    a00 *= inv; a01 *= inv; a02 *= inv; a11 *= inv; a12 *= inv; a22 *= inv;
    R off = a01 * a01 + a02 * a02 + a12 * a12;
    if (off > R(0)) {
        R q = (a00 + a11 + a22) / R(3);
        R b00 = a00 - q, b11 = a11 - q, b22 = a22 - q;
        R p = std::sqrt((b00 * b00 + b11 * b11 + b22 * b22 + off * R(2)) / R(6));
        R c00 = b11 * b22 - a12 * a12;
        R c01 = a01 * b22 - a12 * a02;
        R c02 = a01 * a12 - b11 * a02;
        R det = (b00 * c00 - a01 * c01 + a02 * c02) / (p * p * p);
        R half = det * R(0.5);
        half = std::min(std::max(half, R(-1)), R(1));
        R ang = std::acos(half) / R(3);
        const R two_thirds_pi = R(2.09439510239319549);
        R beta2 = std::cos(ang) * R(2);
        R beta0 = std::cos(ang + two_thirds_pi) * R(2);
        R beta1 = -(beta0 + beta2);
        o.eval = V3<R>(q + p * beta0, q + p * beta1, q + p * beta2);
        if (half >= R(0)) {
            o.e3 = eigvec0(a00, a01, a02, a11, a12, a22, o.eval.z);
            o.e2 = eigvec1(a00, a01, a02, a11, a12, a22, o.e3, o.eval.y);
            o.e1 = cross(o.e2, o.e3);
        } else {
            o.e1 = eigvec0(a00, a01, a02, a11, a12, a22, o.eval.x);
            o.e2 = eigvec1(a00, a01, a02, a11, a12, a22, o.e1, o.eval.y);
            o.e3 = cross(o.e1, o.e2);
        }
    } else {
        o.eval = V3<R>(a00, a11, a22);
        o.e1 = V3<R>(1, 0, 0); o.e2 = V3<R>(0, 1, 0); o.e3 = V3<R>(0, 0, 1);
    }
    o.eval = o.eval * mx;
    return o;
}

// ---------------------------------------------------------- Johnson-Cook ----
// sigma_yield / opt_fun / solve_secant (src/plasticity.cuh:28-93).  The
// reference evaluates these in double even in its float build; the rate term
// uses log_t, which is logf in the float build.
struct JC { double A, B, C, n, m, Tmelt, Tref, eps_dot_ref, clamp_temp; };

inline double sigma_yield(const JC &jc, double eps_pl, double eps_pl_dot, double t, bool float_log) {
    double theta = (t - jc.Tref) / (jc.Tmelt - jc.Tref);
    double a = jc.A + jc.B * std::pow(eps_pl, jc.n);
    double b;
    double ed = eps_pl_dot / jc.eps_dot_ref;
    if (ed > 1.0)
        // float build: log_t is logf and jc.C is a float, so the product is a float product
        b = float_log ? 1.0 + double(float(jc.C) * std::log(float(ed))) : 1.0 + jc.C * std::log(ed);
    else
        b = std::pow(1.0 + ed, jc.C);
    double c = 1.0 - std::pow(theta, jc.m);
    return a * b * c;
}
inline double opt_fun(const JC &jc, double dl, double normS, double eps0, double t, double dt, double mu, bool fl) {
    double e = eps0 + std::sqrt(2.0 / 3.0) * std::fmax(dl, 0.);
    double ed = std::sqrt(2.0 / 3.0) * std::fmax(dl, 0.) / dt;
    return normS - 2 * mu * dl - std::sqrt(2.0 / 3.0) * sigma_yield(jc, e, ed, t, fl);
}
inline double solve_secant(const JC &jc, double init, double tol, double normS, double eps0, double t, double dt,
                           double mu, int max_iter, bool fl, bool &failed) {
    double dl = init, dl_old;
    int iter = 0;
    for (;;) {
        double g = opt_fun(jc, dl, normS, eps0, t, dt, mu, fl);
        double dl1 = dl * 1.01;
        double g1 = opt_fun(jc, dl1, normS, eps0, t, dt, mu, fl);
        double slope = (g - g1) / (dl - dl1);
        dl_old = dl;
        dl = dl - g / slope;
        if (dl < 0.) dl = -0.1 * dl;
        if (std::fabs(dl - dl_old) < tol) return dl;
        if (iter > max_iter) { failed = true; return dl; }
        iter++;
    }
}

// ------------------------------------------------------------- the tool ----
template <class R> struct Tri {
    int i1, i2, i3;
    V3<R> p1, p2, p3, p1i, p2i, p3i;
    V3<R> n, np1, np2, np3, ne1, ne2, ne3;
};

// closest point on a triangle with the normal of the feature hit
// (surface_tri_mesh.cpp:42-128, tool_3d_gpu.cu:109-212)
template <class R> V3<R> closest_on_segment(V3<R> p1, V3<R> p2, V3<R> p) {
    R dx = p1.x - p2.x, dy = p1.y - p2.y, dz = p1.z - p2.z;
    R ns2 = dx * dx + dy * dy + dz * dz;
    if (ns2 == 0) return p1;
    R t = ((p2.x - p1.x) * (p.x - p1.x) + (p2.y - p1.y) * (p.y - p1.y) + (p2.z - p1.z) * (p.z - p1.z)) / ns2;
    if (t > 1) return p2;
    if (t < 0) return p1;
    return (1 - t) * p1 + t * p2;
}
template <class R> void closest_point(const Tri<R> &T, V3<R> qp, V3<R> &cp, V3<R> &np) {
    V3<R> p1p2 = T.p2 - T.p1, p1p3 = T.p3 - T.p1, pp1 = T.p1 - qp;
    R B = dot(p1p3, p1p2), E = dot(p1p2, p1p2), C = dot(p1p3, p1p3);
    R det = B * B - E * C;
    R A = dot(p1p3, pp1), D = dot(p1p2, pp1);
    R t1 = (D * C - A * B) / det, t2 = (A * E - D * B) / det;
    if (t1 < 0) {
        cp = closest_on_segment(T.p1, T.p3, qp);
        np = cp == T.p1 ? T.np1 : (cp == T.p3 ? T.np3 : T.ne3);
    } else if (t2 < 0) {
        cp = closest_on_segment(T.p1, T.p2, qp);
        np = cp == T.p1 ? T.np1 : (cp == T.p2 ? T.np2 : T.ne1);
    } else if (t1 + t2 > 1) {
        cp = closest_on_segment(T.p2, T.p3, qp);
        np = cp == T.p2 ? T.np2 : (cp == T.p3 ? T.np3 : T.ne2);
    } else {
        cp = T.p1 + t1 * p1p2 + t2 * p1p3;
        np = T.n;
    }
}
// Moller-Trumbore (surface_tri_mesh.cpp:315-348, tool_3d_gpu.cu:248-280)
template <class R> bool ray_intersect(const Tri<R> &T, V3<R> o, V3<R> dir, R &t) {
    const R EPS = R(0.0000001);
    V3<R> e1 = T.p2 - T.p1, e2 = T.p3 - T.p1;
    V3<R> h = cross(dir, e2);
    R a = dot(e1, h);
    if (a > -EPS && a < EPS) return false;
    R f = R(1) / a;
    V3<R> s = o - T.p1;
    R u = f * dot(s, h);
    if (u < 0.0 || u > 1.0) return false;
    V3<R> q = cross(s, e1);
    R v = f * dot(dir, q);
    if (v < 0.0 || u + v > 1.0) return false;
    t = f * dot(e2, q);
    return t > EPS;
}
// triangle / axis-aligned box overlap (surface_tri_mesh.cpp:151-278)
template <class R> bool plane_box_overlap(V3<R> n, V3<R> v, V3<R> mb) {
    V3<R> vmin, vmax;
    for (int q = 0; q < 3; q++) {
        if (n[q] > 0) { vmin[q] = -mb[q] - v[q]; vmax[q] = mb[q] - v[q]; }
        else { vmin[q] = mb[q] - v[q]; vmax[q] = -mb[q] - v[q]; }
    }
    if (dot(n, vmin) > 0) return false;
    return dot(n, vmax) >= 0;
}
template <class R> bool cover_aabb(const Tri<R> &T, V3<R> bmin, V3<R> bmax) {
    V3<R> c = R(0.5) * (bmin + bmax), hs = R(0.5) * (bmax - bmin);
    V3<R> v0 = T.p1 - c, v1 = T.p2 - c, v2 = T.p3 - c;
    V3<R> e0 = T.p2 - T.p1, e1 = T.p3 - T.p2, e2 = T.p1 - T.p3;
    auto mm = [](R a, R b, R &lo, R &hi) { if (a < b) { lo = a; hi = b; } else { lo = b; hi = a; } };
    R lo, hi, p0, p1, p2, rad;
    // edge e0: axes x, y, z crossed with e0
    R fx = std::fabs(e0.x), fy = std::fabs(e0.y), fz = std::fabs(e0.z);
    p0 = e0.z * v0.y - e0.y * v0.z; p2 = e0.z * v2.y - e0.y * v2.z; mm(p0, p2, lo, hi);
    rad = fz * hs.y + fy * hs.z; if (lo > rad || hi < -rad) return false;
    p0 = -e0.z * v0.x + e0.x * v0.z; p2 = -e0.z * v2.x + e0.x * v2.z; mm(p0, p2, lo, hi);
    rad = fz * hs.x + fx * hs.z; if (lo > rad || hi < -rad) return false;
    p1 = e0.y * v1.x - e0.x * v1.y; p2 = e0.y * v2.x - e0.x * v2.y;
    if (p2 < p1) { lo = p2; hi = p1; } else { lo = p1; hi = p2; }
    rad = fy * hs.x + fx * hs.y; if (lo > rad || hi < -rad) return false;
    // edge e1
    fx = std::fabs(e1.x); fy = std::fabs(e1.y); fz = std::fabs(e1.z);
    p0 = e1.z * v0.y - e1.y * v0.z; p2 = e1.z * v2.y - e1.y * v2.z; mm(p0, p2, lo, hi);
    rad = fz * hs.y + fy * hs.z; if (lo > rad || hi < -rad) return false;
    p0 = -e1.z * v0.x + e1.x * v0.z; p2 = -e1.z * v2.x + e1.x * v2.z; mm(p0, p2, lo, hi);
    rad = fz * hs.x + fx * hs.z; if (lo > rad || hi < -rad) return false;
    p0 = e1.y * v0.x - e1.x * v0.y; p1 = e1.y * v1.x - e1.x * v1.y; mm(p0, p1, lo, hi);
    rad = fy * hs.x + fx * hs.y; if (lo > rad || hi < -rad) return false;
    // edge e2
    fx = std::fabs(e2.x); fy = std::fabs(e2.y); fz = std::fabs(e2.z);
    p0 = e2.z * v0.y - e2.y * v0.z; p1 = e2.z * v1.y - e2.y * v1.z; mm(p0, p1, lo, hi);
    rad = fz * hs.y + fy * hs.z; if (lo > rad || hi < -rad) return false;
    p0 = -e2.z * v0.x + e2.x * v0.z; p1 = -e2.z * v1.x + e2.x * v1.z; mm(p0, p1, lo, hi);
    rad = fz * hs.x + fx * hs.z; if (lo > rad || hi < -rad) return false;
    p1 = e2.y * v1.x - e2.x * v1.y; p2 = e2.y * v2.x - e2.x * v2.y;
    if (p2 < p1) { lo = p2; hi = p1; } else { lo = p1; hi = p2; }
    rad = fy * hs.x + fx * hs.y; if (lo > rad || hi < -rad) return false;
    // box axes
    auto mm3 = [](R a, R b, R c, R &l, R &h) { l = h = a; if (b < l) l = b; if (b > h) h = b; if (c < l) l = c; if (c > h) h = c; };
    mm3(v0.x, v1.x, v2.x, lo, hi); if (lo > hs.x || hi < -hs.x) return false;
    mm3(v0.y, v1.y, v2.y, lo, hi); if (lo > hs.y || hi < -hs.y) return false;
    mm3(v0.z, v1.z, v2.z, lo, hi); if (lo > hs.z || hi < -hs.z) return false;
    return plane_box_overlap(cross(e0, e1), v0, hs);
}

template <class R> struct Tool {
    std::vector<Tri<R>> tris;    // input order
    std::vector<Tri<R>> boxed;   // tri-grid order (duplicated per cell)
    std::vector<unsigned> cells; // CSR offsets, num_cell + 1
    long nx = 0, ny = 0, nz = 0;
    R bbmin[3], bbmax[3], dx;    // tri grid (moves with the tool)
    V3<R> vel;
    R alpha = R(0.1), mu = 0;
    int algo = MFREE_CONTACT_HASHED;
    R birth = -R(FLT_MAX), death = R(FLT_MAX);
    float force[3] = {0, 0, 0};
    double force_acc[3] = {0, 0, 0};

    unsigned unhash(V3<R> p, long &ix, long &iy, long &iz) const {
        ix = long((unsigned)((p.x - bbmin[0]) / dx));
        iy = long((unsigned)((p.y - bbmin[1]) / dx));
        iz = long((unsigned)((p.z - bbmin[2]) / dx));
        ix = std::min(ix, nx - 1); iy = std::min(iy, ny - 1); iz = std::min(iz, nz - 1);
        return unsigned(ix * ny * nz + iy * nz + iz);
    }
    // closest triangle by expanding shells (tool_3d.cpp:55-161, tool_3d_gpu.cu:282-380)
    bool by_normal(V3<R> qp, V3<R> &cp, V3<R> &nrm) const {
        long ix, iy, iz;
        unsigned b = unhash(qp, ix, iy, iz);
        R md = R(DBL_MAX > double(FLT_MAX) && sizeof(R) == 4 ? HUGE_VALF : DBL_MAX);
        V3<R> bcp, bn;
        bool first_empty = cells[b] == cells[b + 1];
        for (unsigned k = cells[b]; k < cells[b + 1]; k++) {
            V3<R> c, n;
            closest_point(boxed[k], qp, c, n);
            R d = dot(c - qp, c - qp);
            if (d < md) { md = d; bcp = c; bn = n; }
        }
        long off = 1;
        bool all_done = false, empty_so_far = first_empty;
        long cap = std::max(nx, std::max(ny, nz)) + 2;
        while (off <= cap) {
            long li = std::max(ix - off, 0L), lj = std::max(iy - off, 0L), lk = std::max(iz - off, 0L);
            long hi = std::min(ix + off + 1, nx), hj = std::min(iy + off + 1, ny), hk = std::min(iz + off + 1, nz);
            for (long a = li; a < hi; a++)
                for (long bb = lj; bb < hj; bb++)
                    for (long c = lk; c < hk; c++) {
                        bool on = a == li || a == hi - 1 || bb == lj || bb == hj - 1 || c == lk || c == hk - 1;
                        if (!on) continue;
                        long box = a * ny * nz + bb * nz + c;
                        for (unsigned k = cells[box]; k < cells[box + 1]; k++) {
                            empty_so_far = false;
                            V3<R> cc, n;
                            closest_point(boxed[k], qp, cc, n);
                            R d = dot(cc - qp, cc - qp);
                            if (d < md) { md = d; bcp = cc; bn = n; }
                        }
                    }
            if (all_done) break;
            if (!empty_so_far) { off++; all_done = true; continue; }
            off++;
        }
        cp = bcp;
        nrm = bn;
        return dot(bcp - qp, bn) <= 0;  // sign < 0 (tool_3d_gpu.cu:373-379)
    }
    // +z ray parity over the tri-grid column (tool_3d_gpu.cu:382-444)
    bool by_ray(V3<R> qp) const {
        long ix, iy, iz;
        unhash(qp, ix, iy, iz);
        V3<R> dir(0, 0, 1);
        unsigned ni = 0;
        for (; iz < nz; ++iz) {
            long box = ix * ny * nz + iy * nz + iz;
            for (unsigned k = cells[box]; k < cells[box + 1]; k++) {
                R t;
                if (ray_intersect(boxed[k], qp, dir, t)) {
                    V3<R> ip = qp + t * dir;
                    R lox = bbmin[0] + R(ix) * dx, loy = bbmin[1] + R(iy) * dx, loz = bbmin[2] + R(iz) * dx;
                    R hix = bbmin[0] + R(ix + 1) * dx, hiy = bbmin[1] + R(iy + 1) * dx, hiz = bbmin[2] + R(iz + 1) * dx;
                    if (lox <= ip.x && ip.x < hix && loy <= ip.y && ip.y < hiy && loz <= ip.z && ip.z < hiz) ni++;
                }
            }
        }
        return (ni % 2) != 0;
    }
};

// mesh_compute_vertex_normals + mesh_average_edge_length + tool_3d ctor
// (surface_tri_mesh.cpp:410-584, grid_cpu_tri.cpp:48-175, tool_3d.cpp:294-360)
template <class R>
bool build_tool(Tool<R> &tool, const float *verts, int nv, const int *tri, int nt, std::string &err) {
    std::vector<V3<R>> P(nv);
    for (int i = 0; i < nv; i++) P[i] = V3<R>(R(verts[3 * i]), R(verts[3 * i + 1]), R(verts[3 * i + 2]));
    std::vector<Tri<R>> T(nt);
    std::vector<std::vector<int>> vtri(nv);
    struct EK { int a, b; bool operator==(const EK &o) const { return (a == o.a && b == o.b) || (a == o.b && b == o.a); } };
    struct EH { size_t operator()(const EK &e) const { return std::hash<unsigned>()(e.a) + std::hash<unsigned>()(e.b); } };
    std::unordered_map<EK, std::vector<int>, EH> edges;
    for (int i = 0; i < nt; i++) {
        T[i].i1 = tri[3 * i]; T[i].i2 = tri[3 * i + 1]; T[i].i3 = tri[3 * i + 2];
        if (T[i].i1 < 0 || T[i].i1 >= nv || T[i].i2 < 0 || T[i].i2 >= nv || T[i].i3 < 0 || T[i].i3 >= nv) {
            err = "triangle vertex index out of range";
            return false;
        }
        vtri[T[i].i1].push_back(i); vtri[T[i].i2].push_back(i); vtri[T[i].i3].push_back(i);
        edges[EK{T[i].i1, T[i].i2}].push_back(i);
        edges[EK{T[i].i2, T[i].i3}].push_back(i);
        edges[EK{T[i].i3, T[i].i1}].push_back(i);
    }
    for (auto &e : edges)
        if (e.second.size() < 2) { err = "tool mesh is not closed (an edge has one triangle)"; return false; }
    for (auto &t : T) {
        t.p1 = t.p1i = P[t.i1]; t.p2 = t.p2i = P[t.i2]; t.p3 = t.p3i = P[t.i3];
        t.n = normalize(cross(t.p2 - t.p1, t.p3 - t.p1));
    }
    for (auto &t : T) {
        auto &a = edges[EK{t.i1, t.i2}], &b = edges[EK{t.i2, t.i3}], &c = edges[EK{t.i3, t.i1}];
        t.ne1 = normalize(T[a[0]].n + T[a[1]].n);
        t.ne2 = normalize(T[b[0]].n + T[b[1]].n);
        t.ne3 = normalize(T[c[0]].n + T[c[1]].n);
    }
    auto vnormal = [&](int v) {
        V3<R> acc(0, 0, 0);
        for (int ti : vtri[v]) {
            const Tri<R> &t = T[ti];
            V3<R> f1, f2;
            if (t.i1 == v) { f1 = t.p2; f2 = t.p3; }
            if (t.i2 == v) { f1 = t.p1; f2 = t.p3; }
            if (t.i3 == v) { f1 = t.p1; f2 = t.p2; }
            V3<R> a = f1 - P[v], b = f2 - P[v];
            R ang = std::acos(std::fabs(dot(a, b) / (length(a) * length(b))));
            acc = acc + ang * t.n;
        }
        return normalize(acc);
    };
    for (auto &t : T) { t.np1 = vnormal(t.i1); t.np2 = vnormal(t.i2); t.np3 = vnormal(t.i3); }
    // average edge length = (min + max)/2
    R lmin = R(sizeof(R) == 4 ? HUGE_VALF : DBL_MAX), lmax = 0;
    for (auto &t : T) {
        R l1 = length(t.p1 - t.p2), l2 = length(t.p2 - t.p3), l3 = length(t.p3 - t.p1);
        lmin = std::min(std::min(std::min(lmin, l1), l2), l3);
        lmax = std::max(std::max(std::max(lmax, l1), l2), l3);
    }
    R havg = R(0.5) * (lmax + lmin);
    // triangle grid
    R inf = R(sizeof(R) == 4 ? HUGE_VALF : DBL_MAX);
    R bmin[3] = {inf, inf, inf}, bmax[3] = {-inf, -inf, -inf};
    for (auto &t : T)
        for (int d = 0; d < 3; d++) {
            bmin[d] = std::min(std::min(std::min(t.p1[d], t.p2[d]), t.p3[d]), bmin[d]);
            bmax[d] = std::max(std::max(std::max(t.p1[d], t.p2[d]), t.p3[d]), bmax[d]);
        }
    for (int d = 0; d < 3; d++) { bmin[d] = R(bmin[d] - 1e-4); bmax[d] = R(bmax[d] + 1e-4); }
    tool.dx = havg;
    long n3[3];
    for (int d = 0; d < 3; d++) {
        tool.bbmin[d] = bmin[d];
        tool.bbmax[d] = bmax[d];
        R l = bmax[d] - bmin[d];
        n3[d] = long(std::ceil(l / havg));
    }
    tool.nx = n3[0]; tool.ny = n3[1]; tool.nz = n3[2];
    long ncell = tool.nx * tool.ny * tool.nz;
    if (ncell <= 0 || ncell > (1L << 26)) { err = "tool grid has an unusable number of cells"; return false; }
    std::vector<std::vector<int>> grid(ncell);
    for (int i = 0; i < nt; i++) {
        const Tri<R> &t = T[i];
        V3<R> lo, hi;
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(std::min(t.p1[d], t.p2[d]), t.p3[d]);
            hi[d] = std::max(std::max(t.p1[d], t.p2[d]), t.p3[d]);
        }
        long il[3], ih[3];
        for (int d = 0; d < 3; d++) {
            il[d] = long((unsigned)((lo[d] - bmin[d]) / havg));
            ih[d] = long((unsigned)((hi[d] - bmin[d]) / havg));
        }
        for (long a = il[0]; a <= ih[0]; a++)
            for (long b = il[1]; b <= ih[1]; b++)
                for (long c = il[2]; c <= ih[2]; c++) {
                    if (a >= tool.nx || b >= tool.ny || c >= tool.nz) continue;
                    long lin = a * tool.ny * tool.nz + b * tool.nz + c;
                    V3<R> clo(bmin[0] + R(a) * havg, bmin[1] + R(b) * havg, bmin[2] + R(c) * havg);
                    V3<R> chi(bmin[0] + R(a + 1) * havg, bmin[1] + R(b + 1) * havg, bmin[2] + R(c + 1) * havg);
                    if (cover_aabb(t, clo, chi)) grid[lin].push_back(i);
                }
    }
    tool.cells.assign(ncell + 1, 0);
    tool.boxed.clear();
    for (long c = 0; c < ncell; c++) {
        tool.cells[c] = unsigned(tool.boxed.size());
        for (int ti : grid[c]) tool.boxed.push_back(T[ti]);
    }
    tool.cells[ncell] = unsigned(tool.boxed.size());
    tool.tris = T;
    // inside/outside convention: flip every normal if a point just outside the
    // grid box tests inside
    V3<R> out(R(bmax[0] + 1e-6), R(bmax[1] + 1e-6), R(bmax[2] + 1e-6));
    V3<R> cp, nn;
    if (tool.by_normal(out, cp, nn)) {
        auto flip = [](Tri<R> &t) {
            t.ne1 = -t.ne1; t.ne2 = -t.ne2; t.ne3 = -t.ne3;
            t.np1 = -t.np1; t.np2 = -t.np2; t.np3 = -t.np3; t.n = -t.n;
        };
        for (auto &t : tool.tris) flip(t);
        for (auto &t : tool.boxed) flip(t);
    }
    return true;
}

// ------------------------------------------------------------ the step ----
template <class R> struct Sim {
    int N = 0, Ninit = 0;
    // particle_gpu fields (particle_gpu.h:36-99) + particle id
    std::vector<V3<R>> pos, vel, vel_bc, fc, ft, nrm, pos_t, vel_t, pos_half;
    std::vector<R> h, rho, p, fixed, blanked, tool_p, eps, epsd, T, rho_t, T_t;
    std::vector<M3<R>> S, Rs, S_t, S_der, v_der;
    std::vector<int> idx, hash, id, nnb;
    // snapshot of the predictor (leap_frog.cu:21-40)
    std::vector<V3<R>> pos0, vel0;
    std::vector<M3<R>> S0;
    std::vector<R> rho0, T0;
    // grid (grid_gpu_base.h:52-115)
    bool grid_set = false;
    R g_bbmin[3], g_bbmax[3], g_bbmin0[3], g_bbmax0[3], g_dx;
    long g_nx, g_ny, g_nz, g_ncell;
    V3<R> g_vel;
    bool g_adaptive = false;  // unlocked grid (grid_gpu_green(max_cell, N))
    long g_max_cell = 0;
    std::vector<int> cell_start, cell_end;
    // blanking (blanking.cpp)
    bool blank_set = false;
    V3<R> b_min, b_max, b_min0, b_max0, b_vel;
    R b_vmax2 = 0;
    // constants
    mfree_phys phys{};
    mfree_corr corr{};
    mfree_trml twp{}, ttool{};
    JC jc{};
    bool plastic = false;
    mfree_options opt{};
    std::vector<Tool<R>> tools;
    R dt = 0, t = 0;
    bool float_semantics = sizeof(R) == 4;
    int64_t secant_fail = 0;

    bool thermal() const { return twp.alpha != 0 || ttool.alpha != 0; }

    void init(int n, const float *p4, const float *v4, const float *rh, const float *Ti, const float *hh,
              const float *fx, const float *tp) {
        N = Ninit = n;
        pos.assign(n, {}); vel.assign(n, {}); vel_bc.assign(n, {}); fc.assign(n, {}); ft.assign(n, {});
        nrm.assign(n, {}); pos_t.assign(n, {}); vel_t.assign(n, {}); pos_half.assign(n, {});
        h.assign(n, 0); rho.assign(n, 0); p.assign(n, 0); fixed.assign(n, 0); blanked.assign(n, 0);
        tool_p.assign(n, 0); eps.assign(n, 0); epsd.assign(n, 0); T.assign(n, 0); rho_t.assign(n, 0); T_t.assign(n, 0);
        S.assign(n, M3<R>()); Rs.assign(n, M3<R>()); S_t.assign(n, M3<R>()); S_der.assign(n, M3<R>()); v_der.assign(n, M3<R>());
        idx.assign(n, 0); hash.assign(n, 0); id.assign(n, 0); nnb.assign(n, 0);
        pos0.assign(n, {}); vel0.assign(n, {}); S0.assign(n, M3<R>()); rho0.assign(n, 0); T0.assign(n, 0);
        for (int i = 0; i < n; i++) {
            pos[i] = V3<R>(p4[4 * i], p4[4 * i + 1], p4[4 * i + 2]);
            vel[i] = V3<R>(v4[4 * i], v4[4 * i + 1], v4[4 * i + 2]);
            rho[i] = rh[i];
            h[i] = hh[i];
            T[i] = Ti ? Ti[i] : 0;
            fixed[i] = fx ? fx[i] : 0;
            tool_p[i] = tp ? tp[i] : 0;
            idx[i] = i;
            id[i] = i;
        }
    }

    // grid_base::set_geometry (grid_gpu_base.cu:237-273), float rounding of the
    // FP32 build reproduced when R = float
    void set_grid(const float *bmin, const float *bmax, float hh) {
        for (int d = 0; d < 3; d++) {
            g_bbmin[d] = g_bbmin0[d] = R(double(bmin[d]) - 1e-6);
            g_bbmax[d] = g_bbmax0[d] = R(double(bmax[d]) + 1e-6);
        }
        g_dx = R(double(R(hh) * R(2.0)) / 2.);
        R l[3];
        for (int d = 0; d < 3; d++) l[d] = g_bbmax[d] - g_bbmin[d];
        g_nx = long(std::ceil(l[0] / g_dx));
        g_ny = long(std::ceil(l[1] / g_dx));
        g_nz = long(std::ceil(l[2] / g_dx));
        g_ncell = g_nx * g_ny * g_nz;
        g_vel = V3<R>(0, 0, 0);
        grid_set = true;
        g_adaptive = false;
        cell_start.assign(g_ncell, -1);
        cell_end.assign(g_ncell, -1);
    }
    void set_grid_adaptive(long max_cell) {
        g_adaptive = true;
        g_max_cell = max_cell;
        g_nx = g_ny = g_nz = g_ncell = 1;
        g_dx = 0;
        for (int d = 0; d < 3; d++) g_bbmin[d] = g_bbmin0[d] = g_bbmax[d] = g_bbmax0[d] = 0;
        g_vel = V3<R>(0, 0, 0);
        grid_set = true;
        cell_start.assign(1, -1);
        cell_end.assign(1, -1);
    }

    // ---- do_blanking (actions_gpu.cu:489-531) ----
    static bool bad(R v) { return std::isnan(v) || std::isinf(v); }
    void blanking() {
        // blanking::update (blanking.cpp:43-51)
        b_min = b_min0 + t * b_vel;
        b_max = b_max0 + t * b_vel;
        for (int i = 0; i < Ninit; i++) {
            V3<R> q = pos[i], v = vel[i];
            bool fast = v.x * v.x + v.y * v.y + v.z * v.z >= b_vmax2;
            bool in = q.x >= b_min.x && q.x <= b_max.x && q.y >= b_min.y && q.y <= b_max.y && q.z >= b_min.z &&
                      q.z <= b_max.z;
            if (fast || !in) {
                blanked[i] = 1;
            } else {
                bool inv = bad(pos_t[i].x) || bad(pos_t[i].y) || bad(pos_t[i].z) || bad(vel_t[i].x) ||
                           bad(vel_t[i].y) || bad(vel_t[i].z) || bad(S_t[i][0][0]) || bad(S_t[i][1][1]) ||
                           bad(S_t[i][2][2]) || bad(S_t[i][0][1]) || bad(S_t[i][1][2]) || bad(S_t[i][2][0]) ||
                           bad(rho_t[i]) || bad(T_t[i]);
                if (!inv) blanked[i] = 0;
            }
        }
    }

    // ---- compute_hashes + adapt_particle_number + do_sort ----
    int cell_of(V3<R> q) const {
        int ix = int((q.x - g_bbmin[0]) / g_dx);
        int iy = int((q.y - g_bbmin[1]) / g_dx);
        int iz = int((q.z - g_bbmin[2]) / g_dx);
        return int(long(ix) * g_ny * g_nz + long(iy) * g_nz + long(iz));
    }
    // update_geometry, unlocked branch (grid_gpu_base.cu:185-233): the box of
    // the first N particles of the current order (+-1e-6) and their largest h
    // as the cell edge, in the arithmetic of the build (R); NaN coordinates are
    // left out
    int adapt_grid() {
        R mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0}, mh = 0;
        bool seen[3] = {false, false, false}, seen_h = false;
        for (int i = 0; i < N; i++) {
            const R v[3] = {pos[i].x, pos[i].y, pos[i].z};
            for (int d = 0; d < 3; d++) {
                if (std::isnan(v[d])) continue;
                if (!seen[d] || v[d] < mn[d]) mn[d] = v[d];
                if (!seen[d] || v[d] > mx[d]) mx[d] = v[d];
                seen[d] = true;
            }
            if (!std::isnan(h[i]) && (!seen_h || h[i] > mh)) {
                mh = h[i];
                seen_h = true;
            }
        }
        if (!seen[0] || !seen[1] || !seen[2] || !seen_h) return MFREE_ERR_EMPTY;
        for (int d = 0; d < 3; d++) {
            g_bbmin[d] = R(double(mn[d]) - 1e-6);
            g_bbmax[d] = R(double(mx[d]) + 1e-6);
        }
        const R kernel_width = 2;
        g_dx = mh * kernel_width / 2;
        long n3[3];
        for (int d = 0; d < 3; d++) {
            const R l = g_bbmax[d] - g_bbmin[d];
            n3[d] = long(std::ceil(l / g_dx));
        }
        g_nx = n3[0]; g_ny = n3[1]; g_nz = n3[2];
        g_ncell = g_nx * g_ny * g_nz;
        if (g_ncell >= g_max_cell || g_ncell <= 0) return MFREE_ERR_ARG;  // the reference asserts
        cell_start.assign(g_ncell, -1);
        cell_end.assign(g_ncell, -1);
        return MFREE_OK;
    }

    int sort_and_cells() {
        if (g_adaptive) {
            int st = adapt_grid();
            if (st) return st;
        }
        // update_geometry, locked branch (grid_gpu_base.cu:166-183)
        if (!g_adaptive && (g_vel.x != 0 || g_vel.y != 0 || g_vel.z != 0))
            for (int d = 0; d < 3; d++) {
                g_bbmin[d] = g_bbmin0[d] + t * g_vel[d];
                g_bbmax[d] = g_bbmax0[d] + t * g_vel[d];
            }
        for (int i = 0; i < Ninit; i++) hash[i] = blanked[i] == 1 ? INT_MAX : cell_of(pos[i]);
        if (blank_set) {
            int nout = 0;
            for (int i = 0; i < Ninit; i++) nout += hash[i] == INT_MAX;
            N = Ninit - nout;
            if (N == 0) return MFREE_ERR_EMPTY;
        }
        for (int i = 0; i < Ninit; i++) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return hash[a] < hash[b]; });
        std::vector<int> h2(Ninit);
        for (int i = 0; i < Ninit; i++) h2[i] = hash[idx[i]];
        hash.swap(h2);
        auto perm = [&](auto &v) {
            auto o = v;
            for (int i = 0; i < Ninit; i++) o[i] = v[idx[i]];
            v.swap(o);
        };
        perm(pos); perm(vel); perm(vel_bc); perm(fc); perm(ft); perm(h); perm(rho); perm(S); perm(eps); perm(epsd);
        perm(T); perm(fixed); perm(blanked); perm(tool_p); perm(pos_t); perm(vel_t); perm(rho_t); perm(S_t); perm(T_t);
        perm(id);
        std::fill(cell_start.begin(), cell_start.end(), -1);
        std::fill(cell_end.begin(), cell_end.end(), -1);
        for (int i = 0; i < N; i++) {
            int hsh = hash[i];
            if (hsh < 0 || hsh >= g_ncell) continue;  // reference writes out of bounds here
            if (i == 0 || hsh != hash[i - 1]) {
                cell_start[hsh] = i;
                if (i > 0 && hash[i - 1] >= 0 && hash[i - 1] < g_ncell) cell_end[hash[i - 1]] = i;
            }
            if (i == N - 1) cell_end[hsh] = i + 1;
        }
        return MFREE_OK;
    }

    // ---- init + predict (leap_frog.cu:30-70) ----
    void predict() {
        for (int i = 0; i < Ninit; i++) {
            if (blanked[i] == 1) continue;
            pos0[i] = pos[i]; vel0[i] = vel[i]; S0[i] = S[i]; rho0[i] = rho[i]; T0[i] = T[i];
        }
        for (int i = 0; i < Ninit; i++) {
            if (blanked[i] == 1) continue;
            // the literal 0.5 makes the reference evaluate this in double
            auto pr = [&](R x0, R d) { return R(double(x0) + 0.5 * double(dt) * double(d)); };
            pos[i] = V3<R>(pr(pos0[i].x, pos_t[i].x), pr(pos0[i].y, pos_t[i].y), pr(pos0[i].z, pos_t[i].z));
            vel[i] = V3<R>(pr(vel0[i].x, vel_t[i].x), pr(vel0[i].y, vel_t[i].y), pr(vel0[i].z, vel_t[i].z));
            for (int c = 0; c < 3; c++)
                for (int r = 0; r < 3; r++) S[i][c][r] = pr(S0[i][c][r], S_t[i][c][r]);
            rho[i] = pr(rho0[i], rho_t[i]);
            T[i] = pr(T0[i], T_t[i]);
            pos_half[i] = pos[i];
        }
    }

    // ---- do_material_eos + do_corrector_artificial_stress (actions_gpu.cu:40-132) ----
    void eos_artstress() {
        R c0 = std::sqrt(R(phys.K) / R(phys.rho0));
        for (int i = 0; i < N; i++) {
            if (blanked[i] == 1 || tool_p[i] == 1) continue;
            p[i] = c0 * c0 * (rho[i] - R(phys.rho0));
        }
        R eps_as = corr.stresseps;
        if (eps_as == 0) return;
        for (int i = 0; i < N; i++) {
            if (blanked[i] == 1 || tool_p[i] == 1) continue;
            double rhoi21 = 1. / double(rho[i] * rho[i]);
            const M3<R> &Si = S[i];
            R sxx = Si[0][0] - p[i], syy = Si[1][1] - p[i], szz = Si[2][2] - p[i];
            Eig<R> e = solve_eigen<R>(sxx, Si[0][1], Si[0][2], syy, Si[1][2], szz);
            R lam[3] = {e.eval.x, e.eval.y, e.eval.z};
            for (int k = 0; k < 3; k++) lam[k] = lam[k] > 0 ? R(-double(eps_as) * double(lam[k]) * rhoi21) : R(0);
            // Rot has the eigenvectors as rows (GLM fills columns): R = Rot diag Rot^T
            V3<R> ev[3] = {e.e1, e.e2, e.e3};
            M3<R> Rot, D;
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) Rot[c][r] = ev[r][c];
            for (int k = 0; k < 3; k++) D[k][k] = lam[k];
            Rs[i] = mul(mul(Rot, D), transpose(Rot));
        }
    }

    // ---- do_interactions_monaghan (interactions_gpu.cu:152-471) ----
    void interactions() {
        const R mass = phys.mass, K = phys.K;
        const R wdeltap = corr.wdeltap, alpha = corr.alpha, beta = corr.beta, eta = corr.eta, eps = corr.xspheps;
        const bool brook = opt.conduction == MFREE_COND_BROOKSHAW;
        const long nx = g_nx, ny = g_ny, nz = g_nz;
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < N; i++) {
            if (blanked[i] == 1) continue;
            R tool_i = tool_p[i];
            R th_alpha = tool_i == 0 ? R(twp.alpha) : R(ttool.alpha);
            V3<R> pi = pos[i], vi = vel[i];
            const M3<R> &Si = S[i], &Ri = Rs[i];
            R hi = h[i], rhoi = rho[i], prsi = p[i];
            R Ti = 0;
            if (brook && th_alpha != 0) Ti = T[i];
            R rhoi21 = R(1. / double(rhoi * rhoi));
            int hs = hash[i];
            long gi = hs / (nz * ny), gj = (hs - gi * ny * nz) / nz, gk = hs % nz;
            long li = std::max(gi - 2, 0L), lj = std::max(gj - 2, 0L), lk = std::max(gk - 2, 0L);
            long hi_ = std::min(gi + 3, nx), hj = std::min(gj + 3, ny), hk = std::min(gk + 3, nz);
            M3<R> vder, sder;
            V3<R> vt, xt;
            R Tl = 0;
            int count = 0;
            M3<R> invB(1);
            if (opt.cspm) {
                M3<R> B;
                if (tool_i != 1) {
                    for (long a = li; a < hi_; a++)
                        for (long b = lj; b < hj; b++)
                            for (long c = lk; c < hk; c++) {
                                long cell = a * ny * nz + b * nz + c;
                                int cs = cell_start[cell], ce = cell_end[cell];
                                if (cs == -1) continue;
                                for (int j = cs; j < ce; j++) {
                                    if (blanked[j] == 1 || tool_p[j] == 1) continue;
                                    V3<R> pj = pos[j];
                                    R volj = mass / rho[j];
                                    W4<R> w = cubic_spline(pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, hi);
                                    R d[3] = {pi.x - pj.x, pi.y - pj.y, pi.z - pj.z};
                                    R g[3] = {w.wx, w.wy, w.wz};
                                    for (int r = 0; r < 3; r++)
                                        for (int cc = 0; cc < 3; cc++) B[cc][r] -= volj * d[r] * g[cc];
                                }
                            }
                }
                R det = determinant(B);
                if (double(det) > 1e-8) invB = inverse(B);
            }
            for (long a = li; a < hi_; a++)
                for (long b = lj; b < hj; b++)
                    for (long c = lk; c < hk; c++) {
                        long cell = a * ny * nz + b * nz + c;
                        int cs = cell_start[cell], ce = cell_end[cell];
                        if (cs == -1) continue;
                        for (int j = cs; j < ce; j++) {
                            if (blanked[j] == 1) continue;
                            V3<R> pj = pos[j], vj = vel[j];
                            const M3<R> &Sj = S[j], &Rj = Rs[j];
                            R hj_ = h[j], rhoj = rho[j], prsj = p[j];
                            R Tj = 0;
                            if (brook && th_alpha != 0) Tj = T[j];
                            R tool_j = tool_p[j];
                            R volj = mass / rhoj;
                            R rhoj21 = R(1. / double(rhoj * rhoj));
                            W4<R> ww = cubic_spline(pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, hi);
                            {
                                R dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
                                if (in_support(dx * dx + dy * dy + dz * dz, hi)) count++;
                            }
                            R w = ww.w, wx, wy, wz;
                            if (!opt.cspm) {
                                wx = ww.wx; wy = ww.wy; wz = ww.wz;
                            } else {
                                wx = ww.wx * invB[0][0] + ww.wy * invB[1][0] + ww.wz * invB[2][0];
                                wy = ww.wx * invB[0][1] + ww.wy * invB[1][1] + ww.wz * invB[2][1];
                                wz = ww.wx * invB[0][2] + ww.wy * invB[1][2] + ww.wz * invB[2][2];
                            }
                            if (!(tool_i == 1) && !(tool_j == 1)) {
                                R g[3] = {wx, wy, wz};
                                R dv[3] = {vj.x - vi.x, vj.y - vi.y, vj.z - vi.z};
                                for (int r = 0; r < 3; r++)
                                    for (int cc = 0; cc < 3; cc++) vder[r][cc] += dv[r] * g[cc] * volj;
                                R Rxx = 0, Ryy = 0, Rzz = 0, Rxy = 0, Rxz = 0, Ryz = 0;
                                if (wdeltap > 0) {
                                    R fab = w / wdeltap;
                                    fab *= fab;
                                    fab *= fab;
                                    Rxx = fab * (Ri[0][0] + Rj[0][0]);
                                    Rxy = fab * (Ri[0][1] + Rj[0][1]);
                                    Ryy = fab * (Ri[1][1] + Rj[1][1]);
                                    Rxz = fab * (Ri[0][2] + Rj[0][2]);
                                    Ryz = fab * (Ri[1][2] + Rj[1][2]);
                                    Rzz = fab * (Ri[2][2] + Rj[2][2]);
                                }
                                sder[0][0] += mass * ((Si[0][0] - prsi) * rhoi21 + (Sj[0][0] - prsj) * rhoj21 + Rxx) * wx;
                                sder[0][1] += mass * (Si[0][1] * rhoi21 + Sj[0][1] * rhoj21 + Rxy) * wy;
                                sder[0][2] += mass * (Si[0][2] * rhoi21 + Sj[0][2] * rhoj21 + Rxz) * wz;
                                sder[1][0] += mass * (Si[1][0] * rhoi21 + Sj[1][0] * rhoj21 + Rxy) * wx;
                                sder[1][1] += mass * ((Si[1][1] - prsi) * rhoi21 + (Sj[1][1] - prsj) * rhoj21 + Ryy) * wy;
                                sder[1][2] += mass * (Si[1][2] * rhoi21 + Sj[1][2] * rhoj21 + Ryz) * wz;
                                sder[2][0] += mass * (Si[2][0] * rhoi21 + Sj[2][0] * rhoj21 + Rxz) * wx;
                                sder[2][1] += mass * (Si[2][1] * rhoi21 + Sj[2][1] * rhoj21 + Ryz) * wy;
                                sder[2][2] += mass * ((Si[2][2] - prsi) * rhoi21 + (Sj[2][2] - prsj) * rhoj21 + Rzz) * wz;
                                R xij = pi.x - pj.x, yij = pi.y - pj.y, zij = pi.z - pj.z;
                                R vx = vi.x - vj.x, vy = vi.y - vj.y, vz = vi.z - vj.z;
                                R vr = vx * xij + vy * yij + vz * zij;
                                R rhoij = R(0.5) * (rhoi + rhoj);
                                if (vr < 0) {
                                    R ci = std::sqrt(K / rhoi), cj = std::sqrt(K / rhoj);
                                    R cij = R(0.5) * (ci + cj), hij = R(0.5) * (hi + hj_);
                                    R r2 = xij * xij + yij * yij + zij * zij;
                                    R muij = (hij * vr) / (r2 + eta * eta * hij * hij);
                                    R piij = (-alpha * cij * muij + beta * muij * muij) / rhoij;
                                    vt.x += -mass * piij * wx;
                                    vt.y += -mass * piij * wy;
                                    vt.z += -mass * piij * wz;
                                }
                                xt.x += -eps * w * mass / rhoij * vx;
                                xt.y += -eps * w * mass / rhoij * vy;
                                xt.z += -eps * w * mass / rhoij * vz;
                            }
                            if (brook && th_alpha != 0) {
                                R xij = pi.x - pj.x, yij = pi.y - pj.y, zij = pi.z - pj.z;
                                R rij = std::sqrt(xij * xij + yij * yij + zij * zij);
                                if (double(rij) > 1e-8) {
                                    R ex = xij / rij, ey = yij / rij, ez = zij / rij;
                                    R r1 = R(1. / double(rij));
                                    Tl += R(2.0) * (mass / rhoj) * (Ti - Tj) * r1 * (ex * wx + ey * wy + ez * wz);
                                }
                            }
                        }
                    }
            S_der[i] = sder;
            v_der[i] = vder;
            pos_t[i] = xt;
            vel_t[i] = vt;
            nnb[i] = count;
            if (brook && th_alpha != 0) T_t[i] = th_alpha * Tl;
        }
    }

    // ---- do_interactions_heat (interactions_gpu.cu:89-150) ----
    void heat_pse() {
        if (twp.alpha == 0) return;
        const R mass = phys.mass;
        const long nx = g_nx, ny = g_ny, nz = g_nz;
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < N; i++) {
            V3<R> pi = pos[i];
            R hi = h[i], Ti = T[i];
            R al = tool_p[i] == 1 ? R(ttool.alpha) : R(twp.alpha);
            int hs = hash[i];
            long gi = hs / (nz * ny), gj = (hs - gi * ny * nz) / nz, gk = hs % nz;
            long li = std::max(gi - 2, 0L), lj = std::max(gj - 2, 0L), lk = std::max(gk - 2, 0L);
            long hi_ = std::min(gi + 3, nx), hj = std::min(gj + 3, ny), hk = std::min(gk + 3, nz);
            R acc = 0;
            for (long a = li; a < hi_; a++)
                for (long b = lj; b < hj; b++)
                    for (long c = lk; c < hk; c++) {
                        long cell = a * ny * nz + b * nz + c;
                        int cs = cell_start[cell], ce = cell_end[cell];
                        if (cs == -1) continue;
                        for (int j = cs; j < ce; j++) {
                            V3<R> pj = pos[j];
                            R w2 = lapl_pse(pi.x, pi.y, pi.z, pj.x, pj.y, pj.z, hi);
                            acc += (T[j] - Ti) * w2 * mass / rho[j];
                        }
                    }
            T_t[i] = al * acc;
        }
    }

    // ---- Jaumann, continuity, momentum, advection (actions_gpu.cu:134-300) ----
    void rates() {
        const R G = phys.G, mass = phys.mass;
        for (int i = 0; i < N; i++) {
            if (blanked[i] == 1 || tool_p[i] == 1) continue;
            const M3<R> &L = v_der[i];  // L[a][b] = d v_a / d x_b
            const M3<R> &Si = S[i];
            M3<R> ed, om, Sm, I(1);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    // epsdot(r=a,c=b) = 1/2(L_ab + L_ba); omega(r,c) = 1/2(L_rc - L_cr)
                    ed[b][a] = a == b ? L[a][a] : R(0.5) * (L[a][b] + L[b][a]);
                    om[b][a] = a == b ? R(0) : R(0.5) * (L[a][b] - L[b][a]);
                }
            Sm[0][0] = Si[0][0]; Sm[1][1] = Si[1][1]; Sm[2][2] = Si[2][2];
            Sm[0][1] = Sm[1][0] = Si[0][1];
            Sm[0][2] = Sm[2][0] = Si[0][2];
            Sm[1][2] = Sm[2][1] = Si[1][2];
            R tr = ed[0][0] + ed[1][1] + ed[2][2];
            M3<R> a = mul(om, Sm), b = mul(Sm, transpose(om));
            M3<R> o;
            for (int c = 0; c < 3; c++)
                for (int r = 0; r < 3; r++)
                    o[c][r] = R(2.) * G * (ed[c][r] - R(1. / 3.) * tr * I[c][r]) + a[c][r] + b[c][r];
            S_t[i] = o;
            rho_t[i] = R(-double(rho[i]) * double(L[0][0] + L[1][1] + L[2][2]));
            const M3<R> &D = S_der[i];
            vel_t[i].x += D[0][0] + D[0][1] + D[0][2] + fc[i].x / mass + ft[i].x / mass;
            vel_t[i].y += D[1][0] + D[1][1] + D[1][2] + fc[i].y / mass + ft[i].y / mass;
            vel_t[i].z += D[2][0] + D[2][1] + D[2][2] + fc[i].z / mass + ft[i].z / mass;
            pos_t[i] = pos_t[i] + vel[i];
        }
    }

    // ---- correct (leap_frog.cu:72-100) ----
    void correct() {
        for (int i = 0; i < Ninit; i++) {
            if (blanked[i] == 1) continue;
            pos[i] = pos0[i] + dt * pos_t[i];
            vel[i] = vel0[i] + dt * vel_t[i];
            for (int c = 0; c < 3; c++)
                for (int r = 0; r < 3; r++) S[i][c][r] = S0[i][c][r] + dt * S_t[i][c][r];
            rho[i] = rho0[i] + dt * rho_t[i];
            T[i] = T0[i] + dt * T_t[i];
        }
    }

    // ---- do_plasticity_johnson_cook (actions_gpu.cu:371-449) ----
    void plasticity() {
        if (!plastic) return;
        const double mu = phys.G;
        const bool fl = float_semantics;
        int64_t fails = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : fails)
        for (int i = 0; i < N; i++) {
            if (blanked[i] == 1 || tool_p[i] == 1) continue;
            M3<R> Sx = S[i];
            R sxx = Sx[0][0], syy = Sx[1][1], szz = Sx[2][2], sxy = Sx[0][1], syz = Sx[1][2], szx = Sx[2][0];
            R nS = std::sqrt(sxx * sxx + syy * syy + szz * szz + 2 * (sxy * sxy + syz * syz + szx * szx));
            R e0 = eps[i], ed0 = epsd[i], Tc = T[i];
            if (jc.clamp_temp != 0) Tc = (Tc > R(jc.Tmelt)) ? R(jc.Tmelt - 1) : Tc;
            R svm = std::sqrt(R(3.0 / 2.0)) * nS;
            R sY = R(sigma_yield(jc, e0, ed0, Tc, fl));
            if (svm < sY) { epsd[i] = 0; continue; }
            bool failed = false;
            double init = std::fmax(double(ed0) * double(dt) * std::sqrt(2. / 3.), 1e-8);
            R dl = R(solve_secant(jc, init, 1e-6, nS, e0, Tc, dt, mu, opt.max_secant_iter, fl, failed));
            if (failed) fails++;
            R e1 = e0 + std::sqrt(R(2.0 / 3.0)) * std::max(dl, R(0));
            R ed1 = std::sqrt(R(2.0 / 3.0)) * std::max(dl, R(0)) / dt;
            eps[i] = e1;
            epsd[i] = ed1;
            auto f = [&](R s) { return R(double(s) - double(s) / double(nS) * double(dl) * 2. * mu); };
            M3<R> Sn;
            Sn[0][0] = f(sxx); Sn[1][1] = f(syy); Sn[2][2] = f(szz);
            Sn[0][1] = Sn[1][0] = f(sxy);
            Sn[1][2] = Sn[2][1] = f(syz);
            Sn[2][0] = Sn[0][2] = f(szx);
            S[i] = Sn;
            if (twp.tq != 0) {
                R de = e1 - e0;
                R sY2 = R(sigma_yield(jc, e1, ed1, Tc, fl));
                T[i] += R(twp.tq) / (R(twp.cp) * rho[i]) * de * sY2;
            }
        }
        secant_fail += fails;
    }

    // ---- contact (tool_3d_gpu.cu:455-681, 873-948) ----
    void contact(bool record) {
        for (int i = 0; i < N; i++) { fc[i] = V3<R>(); ft[i] = V3<R>(); nrm[i] = V3<R>(); }
        for (auto &tool : tools) {
            for (int d = 0; d < 3; d++) tool.force_acc[d] = 0;
            if (tool.boxed.empty()) continue;
            // update_tool: vertices at p_init + v t, bbox advanced by v dt
            auto upd = [&](Tri<R> &tr) {
                tr.p1 = tr.p1i + tool.vel * t;
                tr.p2 = tr.p2i + tool.vel * t;
                tr.p3 = tr.p3i + tool.vel * t;
            };
            if (tool.algo == MFREE_CONTACT_HASHED) for (auto &tr : tool.boxed) upd(tr);
            else for (auto &tr : tool.tris) upd(tr);
            for (int d = 0; d < 3; d++) {
                tool.bbmin[d] += dt * tool.vel[d];
                tool.bbmax[d] += dt * tool.vel[d];
            }
            if (t < tool.birth || t > tool.death) continue;
            const R mass = phys.mass;
            const R dt2 = dt * dt;
            V3<R> vm(0, 0, 0);
            if (opt.friction_tool_vel) vm = tool.vel;
            std::vector<V3<R>> fsum(Ninit);
#pragma omp parallel for schedule(dynamic, 256)
            for (int i = 0; i < N; i++) {
                if (blanked[i] == 1 || tool_p[i] == 1) continue;
                V3<R> qp = pos[i];
                bool in = qp.x > tool.bbmin[0] && qp.x < tool.bbmax[0] && qp.y > tool.bbmin[1] && qp.y < tool.bbmax[1] &&
                          qp.z > tool.bbmin[2] && qp.z < tool.bbmax[2];
                if (!in) continue;
                V3<R> cp, n;
                if (tool.algo == MFREE_CONTACT_HASHED) {
                    if (!tool.by_ray(qp)) continue;
                    tool.by_normal(qp, cp, n);
                } else {
                    R md = R(FLT_MAX);
                    for (auto &tr : tool.tris) {
                        V3<R> c, nn;
                        closest_point(tr, qp, c, nn);
                        R d = dot(c - qp, c - qp);
                        if (d < md) { md = d; cp = c; n = nn; }
                    }
                    if (dot(cp - qp, n) > 0) continue;
                }
                R gN = dot(qp - cp, n);
                V3<R> fN = (-mass * gN * n) / dt2 * tool.alpha;
                V3<R> fT(0, 0, 0);
                if (tool.mu != 0) {
                    V3<R> v = vel[i] - vm;
                    V3<R> vr = v - cmul(v, n);
                    V3<R> kde = (tool.alpha * mass * vr) / dt;
                    R fy = tool.mu * length(fN);
                    V3<R> fs = ft[i] - kde;
                    if (length(fs) > fy) fT = (fy * fs) / length(fs);
                    else fT = fs;
                }
                fc[i] = fN;
                ft[i] = fT;
                nrm[i] = n;
                fsum[i] = fN + fT;
            }
            if (record)
                for (int i = 0; i < N; i++)
                    for (int d = 0; d < 3; d++) tool.force_acc[d] += double(float(fsum[i][d]));
            if (record)
                for (int d = 0; d < 3; d++) tool.force[d] = float(tool.force_acc[d]);
        }
    }

    // ---- fric heat, BCs, tool particle move (actions_gpu.cu:55-68,192-220,451-487) ----
    void finish() {
        if (twp.eta != 0 && !tools.empty()) {
            V3<R> vt = tools[0].vel;
            for (int i = 0; i < N; i++) {
                if (blanked[i] == 1 || tool_p[i] == 1) continue;
                V3<R> f = ft[i];
                R fm = std::sqrt(f.x * f.x + f.y * f.y + f.z * f.z);
                if (fm == 0) continue;
                V3<R> d = vel[i] - vt;
                R dn = dot(d, nrm[i]);
                V3<R> vr(d.x - dn, d.y - dn, d.z - dn);
                R vm = std::sqrt(vr.x * vr.x + vr.y * vr.y + vr.z * vr.z);
                T[i] += R(twp.eta) * dt * fm * vm / (R(twp.cp) * R(phys.mass));
            }
        }
        for (int i = 0; i < N; i++) {
            if (blanked[i] == 1 || tool_p[i] == 1) continue;
            if (fixed[i] != 0) {
                vel[i] = vel_bc[i];
                fc[i] = V3<R>();
                pos_t[i] = V3<R>();
                vel_t[i] = V3<R>();
            }
        }
        if (thermal())
            for (int i = 0; i < N; i++)
                if (fixed[i] == 1) T[i] = twp.T_init;
        V3<R> vt = tools.empty() ? V3<R>() : tools[0].vel;
        for (int i = 0; i < Ninit; i++) {
            if (tool_p[i] != 1) continue;
            pos[i] = pos[i] + vt * dt;
        }
    }

    int step(bool record) {
        if (!grid_set) return MFREE_ERR_ARG;
        if (blank_set) blanking();
        int st = sort_and_cells();
        if (st) return st;
        predict();
        eos_artstress();
        interactions();
        if (opt.conduction == MFREE_COND_PSE) heat_pse();
        rates();
        correct();
        plasticity();
        contact(record);
        finish();
        t = t + dt;
        return MFREE_OK;
    }
};

struct Handle {
    int prec;
    std::unique_ptr<Sim<double>> d;
    std::unique_ptr<Sim<float>> f;
    std::string err;
};

}  // namespace orc

using orc::Handle;

template <class F> static auto with_sim(Handle *h, F &&fn) {
    if (h->prec == 64) return fn(*h->d);
    return fn(*h->f);
}

extern "C" {

// ---- lifecycle ------------------------------------------------------------
void *orc_create(int prec, int n, const float *pos4, const float *vel4, const float *rho, const float *T,
                 const float *h, const float *fixed, const float *tool_p) {
    auto *H = new Handle();
    H->prec = prec == 32 ? 32 : 64;
    if (H->prec == 64) H->d.reset(new orc::Sim<double>());
    else H->f.reset(new orc::Sim<float>());
    with_sim(H, [&](auto &s) {
        s.init(n, pos4, vel4, rho, T, h, fixed, tool_p);
        s.opt.max_secant_iter = 100;
        return 0;
    });
    return H;
}
void orc_destroy(void *h) { delete (Handle *)h; }
int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_set_params(void *hp, const mfree_phys *phys, const mfree_corr *corr, const mfree_joco *joco,
                   const mfree_trml *twp, const mfree_trml *ttool, const mfree_options *opt) {
    Handle *H = (Handle *)hp;
    return with_sim(H, [&](auto &s) {
        if (phys) s.phys = *phys;
        if (corr) s.corr = *corr;
        if (joco) {
            s.jc = orc::JC{joco->A, joco->B, joco->C, joco->n, joco->m, joco->Tmelt, joco->Tref, joco->eps_dot_ref,
                           joco->clamp_temp};
            s.plastic = true;
        }
        if (twp) s.twp = *twp;
        if (ttool) s.ttool = *ttool;
        if (opt) {
            s.opt = *opt;
            if (s.opt.max_secant_iter <= 0) s.opt.max_secant_iter = 100;
        }
        return 0;
    });
}
int orc_set_grid(void *hp, const float *bbmin, const float *bbmax, float h) {
    return with_sim((Handle *)hp, [&](auto &s) { s.set_grid(bbmin, bbmax, h); return 0; });
}
int orc_set_grid_adaptive(void *hp, long max_cell) {
    return with_sim((Handle *)hp, [&](auto &s) { s.set_grid_adaptive(max_cell); return 0; });
}
int orc_set_grid_velocity(void *hp, const float *v) {
    return with_sim((Handle *)hp, [&](auto &s) { s.g_vel = {v[0], v[1], v[2]}; return 0; });
}
int orc_set_blanking(void *hp, const float *bbmin, const float *bbmax, const float *bbvel, float max_vel) {
    return with_sim((Handle *)hp, [&](auto &s) {
        using R = decltype(s.t);
        s.b_min = s.b_min0 = {R(bbmin[0]), R(bbmin[1]), R(bbmin[2])};
        s.b_max = s.b_max0 = {R(bbmax[0]), R(bbmax[1]), R(bbmax[2])};
        s.b_vel = bbvel ? orc::V3<R>(bbvel[0], bbvel[1], bbvel[2]) : orc::V3<R>(0, 0, 0);
        s.b_vmax2 = R(max_vel) * R(max_vel);
        s.blank_set = true;
        return 0;
    });
}
int orc_set_time(void *hp, double dt, double t) {
    return with_sim((Handle *)hp, [&](auto &s) {
        using R = decltype(s.t);
        s.dt = R(dt);
        s.t = R(t);
        return 0;
    });
}
double orc_get_time(void *hp) {
    return with_sim((Handle *)hp, [&](auto &s) { return double(s.t); });
}
int orc_add_tool(void *hp, const float *verts, int nv, const int *tris, int nt, const float *vel, float alpha,
                 float mu, int algo) {
    Handle *H = (Handle *)hp;
    return with_sim(H, [&](auto &s) {
        using R = decltype(s.t);
        orc::Tool<R> tool;
        if (!orc::build_tool(tool, verts, nv, tris, nt, H->err)) return -1;
        tool.vel = orc::V3<R>(vel[0], vel[1], vel[2]);
        tool.alpha = alpha;
        tool.mu = mu;
        tool.algo = algo;
        s.tools.push_back(tool);
        return int(s.tools.size()) - 1;
    });
}
int orc_tool_info(void *hp, int k, int *num_tris, int *num_boxed, int *n3, float *bbmin, float *bbmax, float *dx) {
    return with_sim((Handle *)hp, [&](auto &s) {
        if (k < 0 || k >= int(s.tools.size())) return -1;
        auto &t = s.tools[k];
        *num_tris = int(t.tris.size());
        *num_boxed = int(t.boxed.size());
        n3[0] = int(t.nx); n3[1] = int(t.ny); n3[2] = int(t.nz);
        for (int d = 0; d < 3; d++) { bbmin[d] = float(t.bbmin[d]); bbmax[d] = float(t.bbmax[d]); }
        *dx = float(t.dx);
        return 0;
    });
}
// 7 float3 per triangle: n, np1, np2, np3, ne1, ne2, ne3
int orc_tool_normals(void *hp, int k, double *out) {
    return with_sim((Handle *)hp, [&](auto &s) {
        if (k < 0 || k >= int(s.tools.size())) return -1;
        auto &t = s.tools[k];
        for (size_t i = 0; i < t.tris.size(); i++) {
            auto &tr = t.tris[i];
            decltype(tr.n) v[7] = {tr.n, tr.np1, tr.np2, tr.np3, tr.ne1, tr.ne2, tr.ne3};
            for (int a = 0; a < 7; a++)
                for (int d = 0; d < 3; d++) out[i * 21 + a * 3 + d] = double(v[a][d]);
        }
        return 0;
    });
}
// boxed triangle index lists: cells (num_cell+1) and the input index of each boxed triangle
int orc_tool_cells(void *hp, int k, int *cells, int *boxed_src) {
    return with_sim((Handle *)hp, [&](auto &s) {
        if (k < 0 || k >= int(s.tools.size())) return -1;
        auto &t = s.tools[k];
        for (size_t c = 0; c < t.cells.size(); c++) cells[c] = int(t.cells[c]);
        for (size_t b = 0; b < t.boxed.size(); b++) {
            int src = -1;
            for (size_t i = 0; i < t.tris.size(); i++)
                if (t.tris[i].i1 == t.boxed[b].i1 && t.tris[i].i2 == t.boxed[b].i2 && t.tris[i].i3 == t.boxed[b].i3) {
                    src = int(i);
                    break;
                }
            boxed_src[b] = src;
        }
        return 0;
    });
}
int orc_tool_forces(void *hp, float *out3) {
    return with_sim((Handle *)hp, [&](auto &s) {
        for (size_t k = 0; k < s.tools.size(); k++)
            for (int d = 0; d < 3; d++) out3[3 * k + d] = s.tools[k].force[d];
        return int(s.tools.size());
    });
}

int orc_step(void *hp, int record) {
    return with_sim((Handle *)hp, [&](auto &s) { return s.step(record != 0); });
}
int orc_counts(void *hp, int *n, int *ninit) {
    return with_sim((Handle *)hp, [&](auto &s) { *n = s.N; *ninit = s.Ninit; return 0; });
}
long orc_secant_failures(void *hp) {
    return with_sim((Handle *)hp, [&](auto &s) { return long(s.secant_fail); });
}
int orc_grid(void *hp, long *n3, double *bbmin, double *dx) {
    return with_sim((Handle *)hp, [&](auto &s) {
        n3[0] = s.g_nx; n3[1] = s.g_ny; n3[2] = s.g_nz;
        for (int d = 0; d < 3; d++) bbmin[d] = double(s.g_bbmin[d]);
        *dx = double(s.g_dx);
        return 0;
    });
}
int orc_cells(void *hp, int *cs, int *ce) {
    return with_sim((Handle *)hp, [&](auto &s) {
        std::copy(s.cell_start.begin(), s.cell_start.end(), cs);
        std::copy(s.cell_end.begin(), s.cell_end.end(), ce);
        return 0;
    });
}

// field export in the reference layout, as doubles (ints for the index fields)
int orc_get_field(void *hp, int field, double *out) {
    return with_sim((Handle *)hp, [&](auto &s) {
        int n = s.Ninit;
        auto v4 = [&](const auto &v) { for (int i = 0; i < n; i++) { out[4*i] = v[i].x; out[4*i+1] = v[i].y; out[4*i+2] = v[i].z; out[4*i+3] = 0; } };
        auto v3 = [&](const auto &v) { for (int i = 0; i < n; i++) { out[3*i] = v[i].x; out[3*i+1] = v[i].y; out[3*i+2] = v[i].z; } };
        auto s1 = [&](const auto &v) { for (int i = 0; i < n; i++) out[i] = double(v[i]); };
        auto m9 = [&](const auto &v) { for (int i = 0; i < n; i++) for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++) out[9*i + 3*c + r] = v[i][c][r]; };
        switch (field) {
            case MFREE_POS: v4(s.pos); break;
            case MFREE_VEL: v4(s.vel); break;
            case MFREE_VEL_BC: v4(s.vel_bc); break;
            case MFREE_H: s1(s.h); break;
            case MFREE_RHO: s1(s.rho); break;
            case MFREE_P: s1(s.p); break;
            case MFREE_S: m9(s.S); break;
            case MFREE_R: m9(s.Rs); break;
            case MFREE_FC: v3(s.fc); break;
            case MFREE_FT: v3(s.ft); break;
            case MFREE_NRM: v3(s.nrm); break;
            case MFREE_FIXED: s1(s.fixed); break;
            case MFREE_BLANKED: s1(s.blanked); break;
            case MFREE_TOOL_PARTICLE: s1(s.tool_p); break;
            case MFREE_EPS_PL: s1(s.eps); break;
            case MFREE_EPS_PL_DOT: s1(s.epsd); break;
            case MFREE_T: s1(s.T); break;
            case MFREE_POS_T: v3(s.pos_t); break;
            case MFREE_VEL_T: v3(s.vel_t); break;
            case MFREE_RHO_T: s1(s.rho_t); break;
            case MFREE_S_T: m9(s.S_t); break;
            case MFREE_T_T: s1(s.T_t); break;
            case MFREE_NUM_NBH: s1(s.nnb); break;
            case MFREE_IDX: s1(s.idx); break;
            case MFREE_HASH: s1(s.hash); break;
            case MFREE_ID: s1(s.id); break;
            case MFREE_POS_HALF: v4(s.pos_half); break;
            default: return -1;
        }
        return 0;
    });
}
// overwrite a field (doubles in the reference layout); used to seed a step
// from a state exported by the CUDA path
int orc_set_field(void *hp, int field, const double *in) {
    return with_sim((Handle *)hp, [&](auto &s) {
        using R = decltype(s.t);
        int n = s.Ninit;
        auto v4 = [&](auto &v) { for (int i = 0; i < n; i++) v[i] = {R(in[4*i]), R(in[4*i+1]), R(in[4*i+2])}; };
        auto v3 = [&](auto &v) { for (int i = 0; i < n; i++) v[i] = {R(in[3*i]), R(in[3*i+1]), R(in[3*i+2])}; };
        auto s1 = [&](auto &v) { for (int i = 0; i < n; i++) v[i] = R(in[i]); };
        auto m9 = [&](auto &v) { for (int i = 0; i < n; i++) for (int c = 0; c < 3; c++) for (int r = 0; r < 3; r++) v[i][c][r] = R(in[9*i + 3*c + r]); };
        switch (field) {
            case MFREE_POS: v4(s.pos); break;
            case MFREE_VEL: v4(s.vel); break;
            case MFREE_VEL_BC: v4(s.vel_bc); break;
            case MFREE_H: s1(s.h); break;
            case MFREE_RHO: s1(s.rho); break;
            case MFREE_S: m9(s.S); break;
            case MFREE_FC: v3(s.fc); break;
            case MFREE_FT: v3(s.ft); break;
            case MFREE_FIXED: s1(s.fixed); break;
            case MFREE_BLANKED: s1(s.blanked); break;
            case MFREE_TOOL_PARTICLE: s1(s.tool_p); break;
            case MFREE_EPS_PL: s1(s.eps); break;
            case MFREE_EPS_PL_DOT: s1(s.epsd); break;
            case MFREE_T: s1(s.T); break;
            case MFREE_POS_T: v3(s.pos_t); break;
            case MFREE_VEL_T: v3(s.vel_t); break;
            case MFREE_RHO_T: s1(s.rho_t); break;
            case MFREE_S_T: m9(s.S_t); break;
            case MFREE_T_T: s1(s.T_t); break;
            case MFREE_ID: for (int i = 0; i < n; i++) s.id[i] = int(in[i]); break;
            default: return -1;
        }
        return 0;
    });
}
const char *orc_last_error(void *hp) { return ((Handle *)hp)->err.c_str(); }

// ---- FP32 integer pipeline of the reference, for the bit-exact checks ----
// compute_hashes (grid_gpu_base.cu:41-63); blanked -> INT_MAX
void orc_hash_fp32(int n, const float *pos4, const float *blanked, const float *bbmin, float dx, long nx, long ny,
                   long nz, int *out) {
    for (int i = 0; i < n; i++) {
        if (blanked && blanked[i] == 1.f) { out[i] = INT_MAX; continue; }
        int ix = int((pos4[4 * i] - bbmin[0]) / dx);
        int iy = int((pos4[4 * i + 1] - bbmin[1]) / dx);
        int iz = int((pos4[4 * i + 2] - bbmin[2]) / dx);
        out[i] = int(long(ix) * ny * nz + long(iy) * nz + long(iz));
    }
}
// stable sort_by_key of (hash, 0..n-1) and find_cell_start over the first
// n_active entries (grid_gpu_green.cu:24-70,265-297)
void orc_sort_cells(int n, const int *hash, int n_active, long num_cell, int *idx_out, int *sorted_hash,
                    int *cell_start, int *cell_end) {
    std::vector<int> idx(n);
    for (int i = 0; i < n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return hash[a] < hash[b]; });
    for (int i = 0; i < n; i++) { idx_out[i] = idx[i]; sorted_hash[i] = hash[idx[i]]; }
    for (long c = 0; c < num_cell; c++) { cell_start[c] = -1; cell_end[c] = -1; }
    for (int i = 0; i < n_active; i++) {
        int hs = sorted_hash[i];
        if (hs < 0 || hs >= num_cell) continue;
        if (i == 0 || hs != sorted_hash[i - 1]) {
            cell_start[hs] = i;
            if (i > 0 && sorted_hash[i - 1] >= 0 && sorted_hash[i - 1] < num_cell) cell_end[sorted_hash[i - 1]] = i;
        }
        if (i == n_active - 1) cell_end[hs] = i + 1;
    }
}
// neighbour count: j in the 5x5x5 stencil of i's cell with 1e-8 <= r^2 < 4 h_i^2
// (the support of cubic_spline, kernels.cuh:41), positions in FP32
void orc_neighbor_counts_fp32(int n_active, const float *pos4, const float *h, const int *sorted_hash,
                              const int *cell_start, const int *cell_end, long nx, long ny, long nz, int *out) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n_active; i++) {
        int hs = sorted_hash[i];
        long gi = hs / (nz * ny), gj = (hs - gi * ny * nz) / nz, gk = hs % nz;
        long li = std::max(gi - 2, 0L), lj = std::max(gj - 2, 0L), lk = std::max(gk - 2, 0L);
        long hi = std::min(gi + 3, nx), hj = std::min(gj + 3, ny), hk = std::min(gk + 3, nz);
        int cnt = 0;
        float xi = pos4[4 * i], yi = pos4[4 * i + 1], zi = pos4[4 * i + 2], hh = h[i];
        for (long a = li; a < hi; a++)
            for (long b = lj; b < hj; b++)
                for (long c = lk; c < hk; c++) {
                    long cell = a * ny * nz + b * nz + c;
                    if (cell_start[cell] == -1) continue;
                    for (int j = cell_start[cell]; j < cell_end[cell]; j++) {
                        float dx = xi - pos4[4 * j], dy = yi - pos4[4 * j + 1], dz = zi - pos4[4 * j + 2];
                        float r2 = dx * dx + dy * dy + dz * dz;
                        if (orc::in_support<float>(r2, hh)) cnt++;
                    }
                }
        out[i] = cnt;
    }
}

// ---- single-function checks (against the reference functions) ----
void orc_cubic_spline(int prec, const double *pi, const double *pj, double h, double *w4) {
    if (prec == 32) {
        auto w = orc::cubic_spline<float>(float(pi[0]), float(pi[1]), float(pi[2]), float(pj[0]), float(pj[1]),
                                          float(pj[2]), float(h));
        w4[0] = w.w; w4[1] = w.wx; w4[2] = w.wy; w4[3] = w.wz;
    } else {
        auto w = orc::cubic_spline<double>(pi[0], pi[1], pi[2], pj[0], pj[1], pj[2], h);
        w4[0] = w.w; w4[1] = w.wx; w4[2] = w.wy; w4[3] = w.wz;
    }
}
double orc_lapl_pse(int prec, const double *pi, const double *pj, double h) {
    if (prec == 32)
        return orc::lapl_pse<float>(float(pi[0]), float(pi[1]), float(pi[2]), float(pj[0]), float(pj[1]),
                                    float(pj[2]), float(h));
    return orc::lapl_pse<double>(pi[0], pi[1], pi[2], pj[0], pj[1], pj[2], h);
}
// a[6] = a00 a01 a02 a11 a12 a22; out[12] = eval(3), e1, e2, e3
void orc_solve_eigen(int prec, const double *a, double *out) {
    auto put = [&](auto e) {
        decltype(e.eval) v[4] = {e.eval, e.e1, e.e2, e.e3};
        for (int k = 0; k < 4; k++) for (int d = 0; d < 3; d++) out[3 * k + d] = double(v[k][d]);
    };
    if (prec == 32) put(orc::solve_eigen<float>(float(a[0]), float(a[1]), float(a[2]), float(a[3]), float(a[4]), float(a[5])));
    else put(orc::solve_eigen<double>(a[0], a[1], a[2], a[3], a[4], a[5]));
}
// Johnson-Cook: jc[9] = A B C n m Tmelt Tref eps_dot_ref clamp_temp
double orc_sigma_yield(int prec, const double *jcv, double eps, double epsd, double T) {
    orc::JC jc{jcv[0], jcv[1], jcv[2], jcv[3], jcv[4], jcv[5], jcv[6], jcv[7], jcv[8]};
    return orc::sigma_yield(jc, eps, epsd, T, prec == 32);
}
double orc_solve_secant(int prec, const double *jcv, double init, double tol, double normS, double eps0, double T,
                        double dt, double mu, int max_iter, int *failed) {
    orc::JC jc{jcv[0], jcv[1], jcv[2], jcv[3], jcv[4], jcv[5], jcv[6], jcv[7], jcv[8]};
    bool f = false;
    double r = orc::solve_secant(jc, init, tol, normS, eps0, T, dt, mu, max_iter, prec == 32, f);
    *failed = f;
    return r;
}

}  // extern "C"
