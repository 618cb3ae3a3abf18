// cplx.cuh -- complex arithmetic on float2 / double2 for the device code.
#pragma once
#include <cuda_runtime.h>

template <typename R> struct CT;
template <> struct CT<float> { typedef float2 T; };
template <> struct CT<double> { typedef double2 T; };

template <typename R> using cplx = typename CT<R>::T;

template <typename R> __host__ __device__ __forceinline__ cplx<R> mkc(R x, R y) {
    cplx<R> r;
    r.x = x;
    r.y = y;
    return r;
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
__host__ __device__ __forceinline__ double2 cconjmul(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cconjmul(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// acc + a * b
__host__ __device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 acc) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}
__host__ __device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc - a * b
__host__ __device__ __forceinline__ float2 cfms(float2 a, float2 b, float2 acc) {
    acc.x = fmaf(-a.x, b.x, acc.x);
    acc.x = fmaf(a.y, b.y, acc.x);
    acc.y = fmaf(-a.x, b.y, acc.y);
    acc.y = fmaf(-a.y, b.x, acc.y);
    return acc;
}
__host__ __device__ __forceinline__ double2 cfms(double2 a, double2 b, double2 acc) {
    acc.x = fma(-a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float cabs2(float2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
// 1 / a, scaled to avoid overflow in |a|^2
__device__ __forceinline__ float2 cinv(float2 a) {
    float s = fmaxf(fabsf(a.x), fabsf(a.y));
    float ax = a.x / s, ay = a.y / s;
    float d = s * (ax * ax + ay * ay);
    return make_float2(ax / d, -ay / d);
}
__device__ __forceinline__ double2 cinv(double2 a) {
    double s = fmax(fabs(a.x), fabs(a.y));
    double ax = a.x / s, ay = a.y / s;
    double d = s * (ax * ax + ay * ay);
    return make_double2(ax / d, -ay / d);
}

template <typename To, typename From> __device__ __forceinline__ To cvt(From a);
template <> __device__ __forceinline__ float2 cvt<float2, double2>(double2 a) {
    return make_float2((float)a.x, (float)a.y);
}
template <> __device__ __forceinline__ double2 cvt<double2, float2>(float2 a) {
    return make_double2((double)a.x, (double)a.y);
}
template <> __device__ __forceinline__ double2 cvt<double2, double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 cvt<float2, float2>(float2 a) { return a; }

__device__ __forceinline__ float2 shfl_c(float2 v, int src) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    return v;
}
__device__ __forceinline__ double2 shfl_c(double2 v, int src) {
    v.x = __shfl_sync(0xffffffffu, v.x, src);
    v.y = __shfl_sync(0xffffffffu, v.y, src);
    return v;
}

// 1 / pv for a nonzero pivot with |pv| in [2^-126, 2^127) (the block
// factors' Gauss-Jordan steps): pv is scaled by the power of two s that
// brings its larger component into [1, 2) (exact), and 1 / |pv s|^2 (in
// [1/8, 1]) is the hardware's approximate reciprocal (rcp.approx, relative
// error within 2^-22); 1 / pv = s^2 conj(pv) / |pv s|^2.
__device__ __forceinline__ float2 pivot_inv(float2 pv) {
    const float m = fmaxf(fabsf(pv.x), fabsf(pv.y));
    const float s = __uint_as_float((254u - (__float_as_uint(m) >> 23)) << 23);
    const float ax = pv.x * s, ay = pv.y * s;
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(ax * ax + ay * ay));
    const float rd = s * r;
    return make_float2(ax * rd, -ay * rd);
}
