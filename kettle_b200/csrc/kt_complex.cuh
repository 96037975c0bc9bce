// kt_complex.cuh — complex arithmetic on interleaved (re, im) vector types and
// index bit helpers used by every kernel.
#pragma once

#ifdef __CUDACC_RTC__
// compiled at run time (generated block kernels): no host headers
typedef signed char int8_t;
typedef unsigned char uint8_t;
typedef short int16_t;
typedef unsigned short uint16_t;
typedef int int32_t;
typedef unsigned int uint32_t;
typedef long long int64_t;
typedef unsigned long long uint64_t;
#else
#include <cuda_runtime.h>

#include <cstdint>
#endif

namespace kt
{

// Generators of the parameterised gates: RX/RY/RZ (and CRX/CRY/CRZ) are
// exp(-i theta G / 2) with G = X, Y, Z; P (and CP) is diag(1, e^(i theta)).
enum Generator : int32_t
{
    GEN_X = 0,
    GEN_Y = 1,
    GEN_Z = 2,
    GEN_P = 3,
};

template <typename T>
struct CxT;
template <>
struct CxT<double>
{
    using type = double2;
};
template <>
struct CxT<float>
{
    using type = float2;
};

template <typename T>
__host__ __device__ __forceinline__ typename CxT<T>::type make_cx(T re, T im)
{
    typename CxT<T>::type v;
    v.x = re;
    v.y = im;
    return v;
}

template <typename C>
__device__ __forceinline__ C cmul(C a, C b)
{
    C r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

// acc + a * b
template <typename C>
__device__ __forceinline__ C cfma(C a, C b, C acc)
{
    C r;
    r.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
    r.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
    return r;
}

template <typename C>
__device__ __forceinline__ C cadd(C a, C b)
{
    C r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}

// conj(a) * b
template <typename C>
__device__ __forceinline__ C cconjmul(C a, C b)
{
    C r;
    r.x = a.x * b.x + a.y * b.y;
    r.y = a.x * b.y - a.y * b.x;
    return r;
}

// Insert a 0 bit at position b of k: bits below b stay, bits at and above b move up by one.
__host__ __device__ __forceinline__ uint64_t insert_zero_bit(uint64_t k, int b)
{
    const uint64_t lo = k & ((uint64_t {1} << b) - 1);
    return ((k ^ lo) << 1) | lo;
}

__device__ __forceinline__ double2 to_d2(double2 v)
{
    return v;
}
__device__ __forceinline__ double2 to_d2(float2 v)
{
    return make_double2(static_cast<double>(v.x), static_cast<double>(v.y));
}

// FP64 value -> the storage type (round to nearest for complex64)
template <typename C>
__device__ __forceinline__ C from_d2(double2 v);
template <>
__device__ __forceinline__ double2 from_d2<double2>(double2 v)
{
    return v;
}
template <>
__device__ __forceinline__ float2 from_d2<float2>(double2 v)
{
    return make_float2(static_cast<float>(v.x), static_cast<float>(v.y));
}

}  // namespace kt
