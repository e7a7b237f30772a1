// Common device helpers: complex arithmetic for double2/float2, launch checks.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fpb
{

template <typename T> struct Cplx;
template <> struct Cplx<double>
{
    typedef double2 type;
};
template <> struct Cplx<float>
{
    typedef float2 type;
};

template <typename T2> __host__ __device__ __forceinline__ T2 mk(decltype(T2::x) a, decltype(T2::x) b)
{
    T2 r;
    r.x = a;
    r.y = b;
    return r;
}
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2  operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2  operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b)
{
    return mk<T2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T2> __device__ __forceinline__ T2 cconj(T2 a) { return mk<T2>(a.x, -a.y); }
template <typename T2, typename T> __device__ __forceinline__ T2 cscale(T2 a, T s) { return mk<T2>(a.x * s, a.y * s); }
// multiply by -i
template <typename T2> __device__ __forceinline__ T2 mul_mi(T2 a) { return mk<T2>(a.y, -a.x); }

}  // namespace fpb
