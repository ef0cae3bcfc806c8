// glm/glm.hpp -- TEST INFRASTRUCTURE: a small GLM-compatible vector and
// matrix header, written for this project, under which the reference
// (iwf_mfree_gpu_3d) compiles unchanged.  The reference names GLM as its only
// dependency (README.md:21) without vendoring it or pinning a version, and
// GLM is not installed here.  This header is NOT GLM: it implements the part of
// GLM's documented interface that the reference uses, from the mathematical
// definitions and GLM's documented conventions:
//
//  * vec2/vec3/dvec2/dvec3 with x, y, z members, componentwise arithmetic,
//    scalar broadcasting, exact == / !=, and operator[] by component;
//  * mat3x3/dmat3x3 stored column-major: m[c] is column c and m[c][r] the
//    entry in row r of column c; the scalar constructor builds s*I (so
//    mat3x3(0.) is zero and mat3x3(1.) the identity); the nine-scalar
//    constructor fills column 0 first, then column 1, then column 2;
//    the default constructor gives the identity;
//  * m * v treats v as a column vector, v * m as a row vector, and m1 * m2 is
//    the matrix product (column c of the result is m1 applied to column c of
//    m2);
//  * dot, cross, length = sqrt(dot(v, v)), normalize = v * (1 / sqrt(dot(v, v)))
//    (GLM's normalize goes through its inversesqrt),
//    transpose, determinant (cofactor expansion along the first row) and
//    inverse (adjugate divided by the determinant).
//
// The reference uses these through its types.h (mat3x3_t, vec3_t, vec2_t),
// actions_gpu.cu:103-129,171-187, interactions_gpu.cu:217-293,
// tool_3d_gpu.cu, surface_tri_mesh.cpp, grid_cpu_tri.cpp, tool_3d.cpp,
// geometry_utils.cpp and the readers.  Sums are evaluated left to right in the
// order written below; where GLM orders a sum differently, results differ in
// the last bits only.  With nvcc every function is __host__ __device__.
#ifndef REF_GLM_COMPAT_HPP
#define REF_GLM_COMPAT_HPP

#include <cmath>
#include <cstddef>

#if defined(__CUDACC__)
#define REFGLM_FN __host__ __device__ inline
#else
#define REFGLM_FN inline
#endif

namespace glm {

template <typename T>
struct tvec2 {
    T x, y;
    REFGLM_FN tvec2() : x(0), y(0) {}
    REFGLM_FN explicit tvec2(T s) : x(s), y(s) {}
    template <typename A, typename B>
    REFGLM_FN tvec2(A a, B b) : x(static_cast<T>(a)), y(static_cast<T>(b)) {}
    template <typename U>
    REFGLM_FN tvec2(const tvec2<U> &o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)) {}
    REFGLM_FN T &operator[](int i) { return i == 0 ? x : y; }
    REFGLM_FN const T &operator[](int i) const { return i == 0 ? x : y; }
};

template <typename T>
struct tvec3 {
    T x, y, z;
    REFGLM_FN tvec3() : x(0), y(0), z(0) {}
    REFGLM_FN explicit tvec3(T s) : x(s), y(s), z(s) {}
    template <typename A, typename B, typename C>
    REFGLM_FN tvec3(A a, B b, C c) : x(static_cast<T>(a)), y(static_cast<T>(b)), z(static_cast<T>(c)) {}
    template <typename U>
    REFGLM_FN tvec3(const tvec3<U> &o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
    REFGLM_FN T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    REFGLM_FN const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }

    REFGLM_FN tvec3 &operator+=(const tvec3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    REFGLM_FN tvec3 &operator-=(const tvec3 &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    REFGLM_FN tvec3 &operator*=(const tvec3 &o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
    REFGLM_FN tvec3 &operator/=(const tvec3 &o) { x /= o.x; y /= o.y; z /= o.z; return *this; }
    template <typename S>
    REFGLM_FN tvec3 &operator*=(S s) { x *= static_cast<T>(s); y *= static_cast<T>(s); z *= static_cast<T>(s); return *this; }
    template <typename S>
    REFGLM_FN tvec3 &operator/=(S s) { x /= static_cast<T>(s); y /= static_cast<T>(s); z /= static_cast<T>(s); return *this; }
};

// ------------------------------------------------------------ vec2 ops --
template <typename T> REFGLM_FN tvec2<T> operator+(const tvec2<T> &a, const tvec2<T> &b) { return tvec2<T>(a.x + b.x, a.y + b.y); }
template <typename T> REFGLM_FN tvec2<T> operator-(const tvec2<T> &a, const tvec2<T> &b) { return tvec2<T>(a.x - b.x, a.y - b.y); }
template <typename T> REFGLM_FN tvec2<T> operator*(const tvec2<T> &a, T s) { return tvec2<T>(a.x * s, a.y * s); }
template <typename T> REFGLM_FN tvec2<T> operator*(T s, const tvec2<T> &a) { return tvec2<T>(s * a.x, s * a.y); }
template <typename T> REFGLM_FN bool operator==(const tvec2<T> &a, const tvec2<T> &b) { return a.x == b.x && a.y == b.y; }
template <typename T> REFGLM_FN bool operator!=(const tvec2<T> &a, const tvec2<T> &b) { return !(a == b); }

// ------------------------------------------------------------ vec3 ops --
template <typename T> REFGLM_FN tvec3<T> operator-(const tvec3<T> &a) { return tvec3<T>(-a.x, -a.y, -a.z); }
template <typename T> REFGLM_FN tvec3<T> operator+(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T> REFGLM_FN tvec3<T> operator-(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> REFGLM_FN tvec3<T> operator*(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x * b.x, a.y * b.y, a.z * b.z); }
template <typename T> REFGLM_FN tvec3<T> operator/(const tvec3<T> &a, const tvec3<T> &b) { return tvec3<T>(a.x / b.x, a.y / b.y, a.z / b.z); }
template <typename T> REFGLM_FN tvec3<T> operator+(const tvec3<T> &a, T s) { return tvec3<T>(a.x + s, a.y + s, a.z + s); }
template <typename T> REFGLM_FN tvec3<T> operator-(const tvec3<T> &a, T s) { return tvec3<T>(a.x - s, a.y - s, a.z - s); }
template <typename T> REFGLM_FN tvec3<T> operator*(const tvec3<T> &a, T s) { return tvec3<T>(a.x * s, a.y * s, a.z * s); }
template <typename T> REFGLM_FN tvec3<T> operator/(const tvec3<T> &a, T s) { return tvec3<T>(a.x / s, a.y / s, a.z / s); }
template <typename T> REFGLM_FN tvec3<T> operator+(T s, const tvec3<T> &a) { return tvec3<T>(s + a.x, s + a.y, s + a.z); }
template <typename T> REFGLM_FN tvec3<T> operator-(T s, const tvec3<T> &a) { return tvec3<T>(s - a.x, s - a.y, s - a.z); }
template <typename T> REFGLM_FN tvec3<T> operator*(T s, const tvec3<T> &a) { return tvec3<T>(s * a.x, s * a.y, s * a.z); }
template <typename T> REFGLM_FN tvec3<T> operator/(T s, const tvec3<T> &a) { return tvec3<T>(s / a.x, s / a.y, s / a.z); }
template <typename T> REFGLM_FN bool operator==(const tvec3<T> &a, const tvec3<T> &b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
template <typename T> REFGLM_FN bool operator!=(const tvec3<T> &a, const tvec3<T> &b) { return !(a == b); }

template <typename T> REFGLM_FN T dot(const tvec3<T> &a, const tvec3<T> &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> REFGLM_FN T dot(const tvec2<T> &a, const tvec2<T> &b) { return a.x * b.x + a.y * b.y; }
template <typename T> REFGLM_FN tvec3<T> cross(const tvec3<T> &a, const tvec3<T> &b) {
    return tvec3<T>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template <typename T> REFGLM_FN T length(const tvec3<T> &a) { using std::sqrt; return sqrt(dot(a, a)); }
template <typename T> REFGLM_FN T length(const tvec2<T> &a) { using std::sqrt; return sqrt(dot(a, a)); }
// GLM normalizes through its inverse square root, 1 / sqrt(x): v * (1 / |v|)
template <typename T> REFGLM_FN tvec3<T> normalize(const tvec3<T> &a) {
    using std::sqrt;
    return a * (T(1) / sqrt(dot(a, a)));
}

// ------------------------------------------------------------- mat3x3 --
template <typename T>
struct tmat3x3 {
    tvec3<T> value[3];  // columns

    REFGLM_FN tmat3x3() {
        value[0] = tvec3<T>(1, 0, 0);
        value[1] = tvec3<T>(0, 1, 0);
        value[2] = tvec3<T>(0, 0, 1);
    }
    REFGLM_FN explicit tmat3x3(T s) {
        value[0] = tvec3<T>(s, 0, 0);
        value[1] = tvec3<T>(0, s, 0);
        value[2] = tvec3<T>(0, 0, s);
    }
    template <typename X1, typename Y1, typename Z1, typename X2, typename Y2, typename Z2,
              typename X3, typename Y3, typename Z3>
    REFGLM_FN tmat3x3(X1 x1, Y1 y1, Z1 z1, X2 x2, Y2 y2, Z2 z2, X3 x3, Y3 y3, Z3 z3) {
        value[0] = tvec3<T>(x1, y1, z1);
        value[1] = tvec3<T>(x2, y2, z2);
        value[2] = tvec3<T>(x3, y3, z3);
    }
    REFGLM_FN tmat3x3(const tvec3<T> &c0, const tvec3<T> &c1, const tvec3<T> &c2) {
        value[0] = c0; value[1] = c1; value[2] = c2;
    }
    template <typename U>
    REFGLM_FN tmat3x3(const tmat3x3<U> &o) {
        value[0] = tvec3<T>(o[0]); value[1] = tvec3<T>(o[1]); value[2] = tvec3<T>(o[2]);
    }
    REFGLM_FN tvec3<T> &operator[](int c) { return value[c]; }
    REFGLM_FN const tvec3<T> &operator[](int c) const { return value[c]; }

    REFGLM_FN tmat3x3 &operator+=(const tmat3x3 &o) { value[0] += o[0]; value[1] += o[1]; value[2] += o[2]; return *this; }
    REFGLM_FN tmat3x3 &operator-=(const tmat3x3 &o) { value[0] -= o[0]; value[1] -= o[1]; value[2] -= o[2]; return *this; }
    template <typename S>
    REFGLM_FN tmat3x3 &operator*=(S s) { value[0] *= s; value[1] *= s; value[2] *= s; return *this; }
};

template <typename T> REFGLM_FN tmat3x3<T> operator-(const tmat3x3<T> &m) { return tmat3x3<T>(-m[0], -m[1], -m[2]); }
template <typename T> REFGLM_FN tmat3x3<T> operator+(const tmat3x3<T> &a, const tmat3x3<T> &b) { return tmat3x3<T>(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
template <typename T> REFGLM_FN tmat3x3<T> operator-(const tmat3x3<T> &a, const tmat3x3<T> &b) { return tmat3x3<T>(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
template <typename T> REFGLM_FN tmat3x3<T> operator*(const tmat3x3<T> &m, T s) { return tmat3x3<T>(m[0] * s, m[1] * s, m[2] * s); }
template <typename T> REFGLM_FN tmat3x3<T> operator*(T s, const tmat3x3<T> &m) { return tmat3x3<T>(s * m[0], s * m[1], s * m[2]); }
template <typename T> REFGLM_FN tmat3x3<T> operator/(const tmat3x3<T> &m, T s) { return tmat3x3<T>(m[0] / s, m[1] / s, m[2] / s); }

// column vector: sum over columns weighted by the vector's components
template <typename T> REFGLM_FN tvec3<T> operator*(const tmat3x3<T> &m, const tvec3<T> &v) {
    return tvec3<T>(m[0].x * v.x + m[1].x * v.y + m[2].x * v.z,
                    m[0].y * v.x + m[1].y * v.y + m[2].y * v.z,
                    m[0].z * v.x + m[1].z * v.y + m[2].z * v.z);
}
// row vector: component c is the row vector times column c
template <typename T> REFGLM_FN tvec3<T> operator*(const tvec3<T> &v, const tmat3x3<T> &m) {
    return tvec3<T>(dot(v, m[0]), dot(v, m[1]), dot(v, m[2]));
}
template <typename T> REFGLM_FN tmat3x3<T> operator*(const tmat3x3<T> &a, const tmat3x3<T> &b) {
    return tmat3x3<T>(a * b[0], a * b[1], a * b[2]);
}
template <typename T> REFGLM_FN bool operator==(const tmat3x3<T> &a, const tmat3x3<T> &b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; }

template <typename T> REFGLM_FN tmat3x3<T> transpose(const tmat3x3<T> &m) {
    return tmat3x3<T>(m[0][0], m[1][0], m[2][0],
                      m[0][1], m[1][1], m[2][1],
                      m[0][2], m[1][2], m[2][2]);
}

// entry (row r, column c) of the mathematical matrix is m[c][r]; expansion
// along row 0: a00 (a11 a22 - a12 a21) - a01 (a10 a22 - a12 a20) + a02 (a10 a21 - a11 a20)
template <typename T> REFGLM_FN T determinant(const tmat3x3<T> &m) {
    return m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
         - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
         + m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
}

// inverse = adjugate / det: entry (r, c) of the inverse is the cofactor of
// entry (c, r) divided by the determinant
template <typename T> REFGLM_FN tmat3x3<T> inverse(const tmat3x3<T> &m) {
    const T d = determinant(m);
    tmat3x3<T> r(T(0));
    // row r, column c of the inverse is stored at [c][r]
    r[0][0] = (m[1][1] * m[2][2] - m[2][1] * m[1][2]) / d;
    r[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) / d;
    r[2][0] = (m[1][0] * m[2][1] - m[2][0] * m[1][1]) / d;
    r[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) / d;
    r[1][1] = (m[0][0] * m[2][2] - m[2][0] * m[0][2]) / d;
    r[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) / d;
    r[0][2] = (m[0][1] * m[1][2] - m[1][1] * m[0][2]) / d;
    r[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) / d;
    r[2][2] = (m[0][0] * m[1][1] - m[1][0] * m[0][1]) / d;
    return r;
}

typedef tvec2<float> vec2;
typedef tvec3<float> vec3;
typedef tvec2<double> dvec2;
typedef tvec3<double> dvec3;
typedef tmat3x3<float> mat3x3;
typedef tmat3x3<double> dmat3x3;
typedef tmat3x3<float> mat3;
typedef tmat3x3<double> dmat3;

}  // namespace glm

#endif
