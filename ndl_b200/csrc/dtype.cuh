// dtype.cuh -- element loads/stores with the reference's conversion rules.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "internal.h"

namespace ndlgpu {

// Border maps of mathHelpers.h:23-25 as applied per axis by
// detail::kernelTapCoord (image/detail.h:178-194): one wrap / one reflection
// only (the host rejects taps that would need more for Wrap and Reflect).
__device__ __forceinline__ int64_t map_border(int border, int64_t M, int64_t x)
{
    if (x >= 0 && x < M) return x;
    if (border == NDLGPU_WRAP) return x < 0 ? x + M : x - M;
    if (border == NDLGPU_REFLECT) return x < 0 ? -x - 1 : 2 * M - x - 1;
    return x < 0 ? 0 : M - 1;
}
__device__ __forceinline__ int map_border32(int border, int M, int x)
{
    if (x >= 0 && x < M) return x;
    if (border == NDLGPU_WRAP) return x < 0 ? x + M : x - M;
    if (border == NDLGPU_REFLECT) return x < 0 ? -x - 1 : 2 * M - x - 1;
    return x < 0 ? 0 : M - 1;
}

// Loads element i of a buffer of dtype dt converted to the accumulator type.
// Integer -> double conversions round to nearest like static_cast<double>
// (convolution.h:68); they are exact for every type of at most 32 bits.
template <class T>
__device__ __forceinline__ T load_as(const char* base, int dt, int64_t i);

template <>
__device__ __forceinline__ double load_as<double>(const char* b, int dt, int64_t i)
{
    switch (dt) {
    case NDLGPU_U8: return (double)((const uint8_t*)b)[i];
    case NDLGPU_I8: return (double)((const int8_t*)b)[i];
    case NDLGPU_U16: return (double)((const uint16_t*)b)[i];
    case NDLGPU_I16: return (double)((const int16_t*)b)[i];
    case NDLGPU_I32: return (double)((const int32_t*)b)[i];
    case NDLGPU_U32: return (double)((const uint32_t*)b)[i];
    case NDLGPU_I64: return __ll2double_rn(((const long long*)b)[i]);
    case NDLGPU_U64: return __ull2double_rn(((const unsigned long long*)b)[i]);
    case NDLGPU_F32: return (double)((const float*)b)[i];
    case NDLGPU_F64: return ((const double*)b)[i];
    case NDLGPU_F16: return (double)__half2float(((const __half*)b)[i]);
    default: return (double)__bfloat162float(((const __nv_bfloat16*)b)[i]);
    }
}

template <>
__device__ __forceinline__ float load_as<float>(const char* b, int dt, int64_t i)
{
    switch (dt) {
    case NDLGPU_U8: return (float)((const uint8_t*)b)[i];
    case NDLGPU_I8: return (float)((const int8_t*)b)[i];
    case NDLGPU_U16: return (float)((const uint16_t*)b)[i];
    case NDLGPU_I16: return (float)((const int16_t*)b)[i];
    case NDLGPU_I32: return __int2float_rn(((const int32_t*)b)[i]);
    case NDLGPU_U32: return __uint2float_rn(((const uint32_t*)b)[i]);
    case NDLGPU_I64: return __ll2float_rn(((const long long*)b)[i]);
    case NDLGPU_U64: return __ull2float_rn(((const unsigned long long*)b)[i]);
    case NDLGPU_F32: return ((const float*)b)[i];
    case NDLGPU_F64: return __double2float_rn(((const double*)b)[i]);
    case NDLGPU_F16: return __half2float(((const __half*)b)[i]);
    default: return __bfloat162float(((const __nv_bfloat16*)b)[i]);
    }
}

template <>
__device__ __forceinline__ int32_t load_as<int32_t>(const char* b, int dt, int64_t i)
{
    switch (dt) {
    case NDLGPU_U8: return ((const uint8_t*)b)[i];
    case NDLGPU_I8: return ((const int8_t*)b)[i];
    case NDLGPU_U16: return ((const uint16_t*)b)[i];
    case NDLGPU_I16: return ((const int16_t*)b)[i];
    default: return ((const int32_t*)b)[i];
    }
}

// Truncation toward zero into 64 bits; out-of-range and NaN give INT64_MIN,
// the value x86-64's cvttsd2si produces (the reference's cast is undefined
// there; in range every choice agrees).
__device__ __forceinline__ long long trunc_i64(double v)
{
    if (!(v > -9.2233720368547758e18 && v < 9.2233720368547758e18)) return (long long)0x8000000000000000ull;
    return (long long)v;
}

__device__ __forceinline__ void store_int_bits(char* b, int dt, int64_t i, long long v)
{
    switch (dt) {
    case NDLGPU_U8: ((uint8_t*)b)[i] = (uint8_t)v; break;
    case NDLGPU_I8: ((int8_t*)b)[i] = (int8_t)(uint8_t)v; break;
    case NDLGPU_U16: ((uint16_t*)b)[i] = (uint16_t)v; break;
    case NDLGPU_I16: ((int16_t*)b)[i] = (int16_t)(uint16_t)v; break;
    case NDLGPU_I32: ((int32_t*)b)[i] = (int32_t)(uint32_t)v; break;
    case NDLGPU_U32: ((uint32_t*)b)[i] = (uint32_t)v; break;
    default: ((long long*)b)[i] = v; break;
    }
}

// Stores a double total as DstT (convolution.h:69 / :184).
__device__ __forceinline__ void store_from(char* b, int dt, int64_t i, double v, int mode)
{
    switch (dt) {
    case NDLGPU_F32: ((float*)b)[i] = __double2float_rn(v); return;
    case NDLGPU_F64: ((double*)b)[i] = v; return;
    case NDLGPU_F16: ((__half*)b)[i] = __double2half(v); return;
    case NDLGPU_BF16: ((__nv_bfloat16*)b)[i] = __double2bfloat16(v); return;
    case NDLGPU_U64: {
        if (mode == STORE_ROUND) v = round(v);
        unsigned long long u = (v >= 9.2233720368547758e18)
            ? (unsigned long long)trunc_i64(v - 9.2233720368547758e18) + 0x8000000000000000ull
            : (unsigned long long)trunc_i64(v);
        ((unsigned long long*)b)[i] = u;
        return;
    }
    default:
        if (mode == STORE_ROUND) v = round(v);
        store_int_bits(b, dt, i, trunc_i64(v));
        return;
    }
}

__device__ __forceinline__ void store_from(char* b, int dt, int64_t i, float v, int mode)
{
    switch (dt) {
    case NDLGPU_F32: ((float*)b)[i] = v; return;
    case NDLGPU_F64: ((double*)b)[i] = (double)v; return;
    case NDLGPU_F16: ((__half*)b)[i] = __float2half_rn(v); return;
    case NDLGPU_BF16: ((__nv_bfloat16*)b)[i] = __float2bfloat16_rn(v); return;
    default: store_from(b, dt, i, (double)v, mode); return;
    }
}

// Integer accumulator with a dyadic scale: value = acc / 2^shift, exact.
__device__ __forceinline__ long long int_scaled(long long acc, int shift, int mode)
{
    if (shift == 0) return acc;
    const long long half = 1ll << (shift - 1);
    if (mode == STORE_ROUND)
        return acc >= 0 ? (acc + half) >> shift : -((-acc + half) >> shift);
    return acc >= 0 ? acc >> shift : -((-acc) >> shift);
}

__device__ __forceinline__ void store_from(char* b, int dt, int64_t i, int32_t acc, int mode, int shift)
{
    if (mode == STORE_RAW) { ((int32_t*)b)[i] = acc; return; }
    long long v = int_scaled(acc, shift, mode);
    if (dt == NDLGPU_F32 || dt == NDLGPU_F64 || dt == NDLGPU_F16 || dt == NDLGPU_BF16) {
        store_from(b, dt, i, ldexp((double)acc, -shift), STORE_CAST);
        return;
    }
    store_int_bits(b, dt, i, v);
}

}  // namespace ndlgpu
