// Small device math helpers: 2-vectors and complex numbers in the bulk real
// type R (float in the mixed-precision tracer, double in the FP64 tracer).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace bhcb {

template<typename T> struct V2 {
    T x, y;
};
template<typename T> __device__ __forceinline__ V2<T> mk2(T x, T y) { return V2<T>{x, y}; }
template<typename T> __device__ __forceinline__ V2<T> add2(V2<T> a, V2<T> b) { return {a.x + b.x, a.y + b.y}; }
template<typename T> __device__ __forceinline__ V2<T> sub2(V2<T> a, V2<T> b) { return {a.x - b.x, a.y - b.y}; }
template<typename T> __device__ __forceinline__ V2<T> scl2(T s, V2<T> a) { return {s * a.x, s * a.y}; }
template<typename T> __device__ __forceinline__ V2<T> div2(V2<T> a, T s) { return {a.x / s, a.y / s}; }
template<typename T> __device__ __forceinline__ T dot2(V2<T> a, V2<T> b) { return a.x * b.x + a.y * b.y; }
template<typename T, typename U> __device__ __forceinline__ V2<T> cvt2(V2<U> a)
{
    return {(T)a.x, (T)a.y};
}

template<typename T> struct Cx {
    T r, i;
};
template<typename T> __device__ __forceinline__ Cx<T> cx(T r, T i) { return Cx<T>{r, i}; }
template<typename T> __device__ __forceinline__ Cx<T> cadd(Cx<T> a, Cx<T> b) { return {a.r + b.r, a.i + b.i}; }
template<typename T> __device__ __forceinline__ Cx<T> csub(Cx<T> a, Cx<T> b) { return {a.r - b.r, a.i - b.i}; }
template<typename T> __device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b)
{
    return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r};
}
template<typename T> __device__ __forceinline__ Cx<T> cscl(T s, Cx<T> a) { return {s * a.r, s * a.i}; }
// complex division by Smith's method (scales by the larger component, exact
// for a purely real divisor)
template<typename T> __device__ __forceinline__ Cx<T> cdiv(Cx<T> a, Cx<T> b)
{
    if(fabs(b.r) >= fabs(b.i)) {
        T rat = b.i / b.r, den = b.r + b.i * rat;
        return {(a.r + a.i * rat) / den, (a.i - a.r * rat) / den};
    } else {
        T rat = b.r / b.i, den = b.r * rat + b.i;
        return {(a.r * rat + a.i) / den, (a.i * rat - a.r) / den};
    }
}
template<typename T> __device__ __forceinline__ Cx<T> rdivc(T a, Cx<T> b)
{
    return cdiv(Cx<T>{a, (T)0}, b);
}
template<typename T> __device__ __forceinline__ T cabs_(Cx<T> a) { return hypot(a.r, a.i); }
// principal square root
template<typename T> __device__ __forceinline__ Cx<T> csqrt_(Cx<T> z)
{
    T m = hypot(z.r, z.i);
    if(m == (T)0) return {(T)0, z.i};
    if(z.r >= (T)0) {
        T t = sqrt((m + z.r) * (T)0.5);
        return {t, z.i / (t + t)};
    }
    T t = sqrt((m - z.r) * (T)0.5);
    return {fabs(z.i) / (t + t), copysign(t, z.i)};
}

// Hardware approximations (PTX .approx.ftz forms) for the mixed-precision
// contribution math; arguments of sin/cos are range-reduced by the caller.
__device__ __forceinline__ float ex2_ftz(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_ftz(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_ftz(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sin_ftz(float x)
{
    float y;
    asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float cos_ftz(float x)
{
    float y;
    asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ double spacing_d(double v)
{
    return fabs(nextafter(v, 0.0) - v);
}

} // namespace bhcb
