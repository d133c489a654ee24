// Project-written stand-in for the subset of the GLM vector-math API that the
// reference tracer uses (its glm submodule is not vendored). This is test
// infrastructure: it exists only so the reference's own C++ sources can be
// compiled as a CPU oracle. Semantics follow GLM's public documentation:
//  - vec<L,T,Q>: L in {2,3}, members x,y(,z), element-wise arithmetic with
//    vectors and scalars, explicit scalar-broadcast constructor.
//  - mat<2,2,T,Q>: column-major, m[col][row]; mat(s) = s*I;
//    mat(x0,y0,x1,y1) fills column 0 then column 1.
//  - dot = sum of products left to right; length = sqrt(dot(v,v));
//    cross, distance, transpose, determinant, row as in linear algebra.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstddef>

namespace glm {

enum qualifier { defaultp = 0 };

template<int L, typename T, qualifier Q = defaultp> struct vec;

template<typename T, qualifier Q> struct vec<2, T, Q> {
    T x, y;
    vec() : x(0), y(0) {}
    explicit vec(T s) : x(s), y(s) {}
    vec(T a, T b) : x(a), y(b) {}
    template<typename U, qualifier P> explicit vec(const vec<2, U, P> &o)
        : x(static_cast<T>(o.x)), y(static_cast<T>(o.y))
    {}
    T &operator[](int i) { return i == 0 ? x : y; }
    const T &operator[](int i) const { return i == 0 ? x : y; }
    vec &operator+=(const vec &o) { x += o.x; y += o.y; return *this; }
    vec &operator-=(const vec &o) { x -= o.x; y -= o.y; return *this; }
    vec &operator*=(const vec &o) { x *= o.x; y *= o.y; return *this; }
    vec &operator/=(const vec &o) { x /= o.x; y /= o.y; return *this; }
    template<typename S> vec &operator*=(S s) { x *= T(s); y *= T(s); return *this; }
    template<typename S> vec &operator/=(S s) { x /= T(s); y /= T(s); return *this; }
    template<typename S> vec &operator+=(S s) { x += T(s); y += T(s); return *this; }
    template<typename S> vec &operator-=(S s) { x -= T(s); y -= T(s); return *this; }
};

template<typename T, qualifier Q> struct vec<3, T, Q> {
    T x, y, z;
    vec() : x(0), y(0), z(0) {}
    explicit vec(T s) : x(s), y(s), z(s) {}
    vec(T a, T b, T c) : x(a), y(b), z(c) {}
    vec(const vec<2, T, Q> &xy, T c) : x(xy.x), y(xy.y), z(c) {}
    template<typename U, qualifier P> explicit vec(const vec<3, U, P> &o)
        : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z))
    {}
    T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const T &operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    vec &operator+=(const vec &o) { x += o.x; y += o.y; z += o.z; return *this; }
    vec &operator-=(const vec &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    vec &operator*=(const vec &o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
    vec &operator/=(const vec &o) { x /= o.x; y /= o.y; z /= o.z; return *this; }
    template<typename S> vec &operator*=(S s) { x *= T(s); y *= T(s); z *= T(s); return *this; }
    template<typename S> vec &operator/=(S s) { x /= T(s); y /= T(s); z /= T(s); return *this; }
    template<typename S> vec &operator+=(S s) { x += T(s); y += T(s); z += T(s); return *this; }
    template<typename S> vec &operator-=(S s) { x -= T(s); y -= T(s); z -= T(s); return *this; }
};

// ---- vec2 operators
#define GLMSHIM_V2BIN(OP) \
    template<typename T, qualifier Q> inline vec<2, T, Q> operator OP( \
        const vec<2, T, Q> &a, const vec<2, T, Q> &b) \
    { \
        return vec<2, T, Q>(a.x OP b.x, a.y OP b.y); \
    } \
    template<typename T, qualifier Q, typename S> inline vec<2, T, Q> operator OP( \
        const vec<2, T, Q> &a, S s) \
    { \
        return vec<2, T, Q>(a.x OP T(s), a.y OP T(s)); \
    } \
    template<typename T, qualifier Q, typename S> inline vec<2, T, Q> operator OP( \
        S s, const vec<2, T, Q> &a) \
    { \
        return vec<2, T, Q>(T(s) OP a.x, T(s) OP a.y); \
    }
GLMSHIM_V2BIN(+)
GLMSHIM_V2BIN(-)
GLMSHIM_V2BIN(*)
GLMSHIM_V2BIN(/)
#undef GLMSHIM_V2BIN
template<typename T, qualifier Q> inline vec<2, T, Q> operator-(const vec<2, T, Q> &a)
{
    return vec<2, T, Q>(-a.x, -a.y);
}
template<typename T, qualifier Q> inline bool operator==(
    const vec<2, T, Q> &a, const vec<2, T, Q> &b)
{
    return a.x == b.x && a.y == b.y;
}
template<typename T, qualifier Q> inline bool operator!=(
    const vec<2, T, Q> &a, const vec<2, T, Q> &b)
{
    return !(a == b);
}

// ---- vec3 operators
#define GLMSHIM_V3BIN(OP) \
    template<typename T, qualifier Q> inline vec<3, T, Q> operator OP( \
        const vec<3, T, Q> &a, const vec<3, T, Q> &b) \
    { \
        return vec<3, T, Q>(a.x OP b.x, a.y OP b.y, a.z OP b.z); \
    } \
    template<typename T, qualifier Q, typename S> inline vec<3, T, Q> operator OP( \
        const vec<3, T, Q> &a, S s) \
    { \
        return vec<3, T, Q>(a.x OP T(s), a.y OP T(s), a.z OP T(s)); \
    } \
    template<typename T, qualifier Q, typename S> inline vec<3, T, Q> operator OP( \
        S s, const vec<3, T, Q> &a) \
    { \
        return vec<3, T, Q>(T(s) OP a.x, T(s) OP a.y, T(s) OP a.z); \
    }
GLMSHIM_V3BIN(+)
GLMSHIM_V3BIN(-)
GLMSHIM_V3BIN(*)
GLMSHIM_V3BIN(/)
#undef GLMSHIM_V3BIN
template<typename T, qualifier Q> inline vec<3, T, Q> operator-(const vec<3, T, Q> &a)
{
    return vec<3, T, Q>(-a.x, -a.y, -a.z);
}
template<typename T, qualifier Q> inline bool operator==(
    const vec<3, T, Q> &a, const vec<3, T, Q> &b)
{
    return a.x == b.x && a.y == b.y && a.z == b.z;
}
template<typename T, qualifier Q> inline bool operator!=(
    const vec<3, T, Q> &a, const vec<3, T, Q> &b)
{
    return !(a == b);
}

// ---- 2x2 matrix, column-major: m[col][row]
template<int C, int R, typename T, qualifier Q = defaultp> struct mat;

template<typename T, qualifier Q> struct mat<2, 2, T, Q> {
    typedef vec<2, T, Q> col_type;
    col_type value[2];
    mat() : value{col_type(T(1), T(0)), col_type(T(0), T(1))} {}
    explicit mat(T s) : value{col_type(s, T(0)), col_type(T(0), s)} {}
    mat(T x0, T y0, T x1, T y1) : value{col_type(x0, y0), col_type(x1, y1)} {}
    mat(const col_type &c0, const col_type &c1) : value{c0, c1} {}
    col_type &operator[](int i) { return value[i]; }
    const col_type &operator[](int i) const { return value[i]; }
    template<typename S> mat &operator*=(S s)
    {
        value[0] *= s;
        value[1] *= s;
        return *this;
    }
    mat &operator+=(const mat &o)
    {
        value[0] += o.value[0];
        value[1] += o.value[1];
        return *this;
    }
    mat &operator-=(const mat &o)
    {
        value[0] -= o.value[0];
        value[1] -= o.value[1];
        return *this;
    }
};

template<typename T, qualifier Q> inline mat<2, 2, T, Q> operator+(
    const mat<2, 2, T, Q> &a, const mat<2, 2, T, Q> &b)
{
    return mat<2, 2, T, Q>(a[0] + b[0], a[1] + b[1]);
}
template<typename T, qualifier Q> inline mat<2, 2, T, Q> operator-(
    const mat<2, 2, T, Q> &a, const mat<2, 2, T, Q> &b)
{
    return mat<2, 2, T, Q>(a[0] - b[0], a[1] - b[1]);
}
template<typename T, qualifier Q> inline mat<2, 2, T, Q> operator-(const mat<2, 2, T, Q> &a)
{
    return mat<2, 2, T, Q>(-a[0], -a[1]);
}
template<typename T, qualifier Q, typename S> inline mat<2, 2, T, Q> operator*(
    const mat<2, 2, T, Q> &a, S s)
{
    return mat<2, 2, T, Q>(a[0] * T(s), a[1] * T(s));
}
template<typename T, qualifier Q, typename S> inline mat<2, 2, T, Q> operator*(
    S s, const mat<2, 2, T, Q> &a)
{
    return mat<2, 2, T, Q>(T(s) * a[0], T(s) * a[1]);
}
template<typename T, qualifier Q, typename S> inline mat<2, 2, T, Q> operator/(
    const mat<2, 2, T, Q> &a, S s)
{
    return mat<2, 2, T, Q>(a[0] / T(s), a[1] / T(s));
}
// matrix product: (A B)[c][r] = sum_k A[k][r] * B[c][k]
template<typename T, qualifier Q> inline mat<2, 2, T, Q> operator*(
    const mat<2, 2, T, Q> &a, const mat<2, 2, T, Q> &b)
{
    return mat<2, 2, T, Q>(
        a[0][0] * b[0][0] + a[1][0] * b[0][1], a[0][1] * b[0][0] + a[1][1] * b[0][1],
        a[0][0] * b[1][0] + a[1][0] * b[1][1], a[0][1] * b[1][0] + a[1][1] * b[1][1]);
}
// matrix times column vector
template<typename T, qualifier Q> inline vec<2, T, Q> operator*(
    const mat<2, 2, T, Q> &a, const vec<2, T, Q> &v)
{
    return vec<2, T, Q>(a[0][0] * v.x + a[1][0] * v.y, a[0][1] * v.x + a[1][1] * v.y);
}
// row vector times matrix
template<typename T, qualifier Q> inline vec<2, T, Q> operator*(
    const vec<2, T, Q> &v, const mat<2, 2, T, Q> &a)
{
    return vec<2, T, Q>(v.x * a[0][0] + v.y * a[0][1], v.x * a[1][0] + v.y * a[1][1]);
}

typedef vec<2, float, defaultp> vec2f_;
typedef mat<2, 2, double, defaultp> mat2x2;
typedef mat<2, 2, double, defaultp> dmat2x2;

// ---- geometric functions
template<typename T, qualifier Q> inline T dot(const vec<2, T, Q> &a, const vec<2, T, Q> &b)
{
    return a.x * b.x + a.y * b.y;
}
template<typename T, qualifier Q> inline T dot(const vec<3, T, Q> &a, const vec<3, T, Q> &b)
{
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template<int L, typename T, qualifier Q> inline T length(const vec<L, T, Q> &v)
{
    return std::sqrt(dot(v, v));
}
template<int L, typename T, qualifier Q> inline T distance(
    const vec<L, T, Q> &a, const vec<L, T, Q> &b)
{
    return length(b - a);
}
template<typename T, qualifier Q> inline vec<3, T, Q> cross(
    const vec<3, T, Q> &a, const vec<3, T, Q> &b)
{
    return vec<3, T, Q>(
        a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
template<typename T, qualifier Q> inline mat<2, 2, T, Q> transpose(const mat<2, 2, T, Q> &m)
{
    return mat<2, 2, T, Q>(m[0][0], m[1][0], m[0][1], m[1][1]);
}
template<typename T, qualifier Q> inline T determinant(const mat<2, 2, T, Q> &m)
{
    return m[0][0] * m[1][1] - m[1][0] * m[0][1];
}
template<typename T, qualifier Q> inline vec<2, T, Q> row(const mat<2, 2, T, Q> &m, int i)
{
    return vec<2, T, Q>(m[0][i], m[1][i]);
}
template<typename T, qualifier Q> inline vec<2, T, Q> column(const mat<2, 2, T, Q> &m, int i)
{
    return m[i];
}

} // namespace glm
