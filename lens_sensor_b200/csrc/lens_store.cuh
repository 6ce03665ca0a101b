// Field storage access of the batched 2D kernels (sm_100a): FP32, FP16 or BF16
// values read and written in groups of four consecutive elements, arithmetic
// in FP32.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lens_common.cuh"

template <typename T>
struct St;
// Storage access of VEC = 4 consecutive values (16 bytes FP32, 8 bytes FP16/BF16;
// every access starts at a multiple of 4 elements).  Conversions round to
// nearest even per element.
template <>
struct St<float> {
    static __device__ __forceinline__ float4 ld4(const void *p, size_t o) {
        return *reinterpret_cast<const float4 *>(static_cast<const float *>(p) + o);
    }
    static __device__ __forceinline__ void st4(void *p, size_t o, float4 v) {
        *reinterpret_cast<float4 *>(static_cast<float *>(p) + o) = v;
    }
    static __device__ __forceinline__ float ld(const void *p, size_t o) { return static_cast<const float *>(p)[o]; }
};
template <>
struct St<__half> {
    static __device__ __forceinline__ float4 ld4(const void *p, size_t o) {
        const uint2 u = *reinterpret_cast<const uint2 *>(static_cast<const __half *>(p) + o);
        const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    static __device__ __forceinline__ void st4(void *p, size_t o, float4 v) {
        const __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
        uint2 u;
        u.x = *reinterpret_cast<const unsigned *>(&a);
        u.y = *reinterpret_cast<const unsigned *>(&b);
        *reinterpret_cast<uint2 *>(static_cast<__half *>(p) + o) = u;
    }
    static __device__ __forceinline__ float ld(const void *p, size_t o) {
        return __half2float(static_cast<const __half *>(p)[o]);
    }
};
template <>
struct St<__nv_bfloat16> {
    static __device__ __forceinline__ float4 ld4(const void *p, size_t o) {
        const uint2 u = *reinterpret_cast<const uint2 *>(static_cast<const __nv_bfloat16 *>(p) + o);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u.y));
        return make_float4(a.x, a.y, b.x, b.y);
    }
    static __device__ __forceinline__ void st4(void *p, size_t o, float4 v) {
        const __nv_bfloat162 a = __floats2bfloat162_rn(v.x, v.y), b = __floats2bfloat162_rn(v.z, v.w);
        uint2 u;
        u.x = *reinterpret_cast<const unsigned *>(&a);
        u.y = *reinterpret_cast<const unsigned *>(&b);
        *reinterpret_cast<uint2 *>(static_cast<__nv_bfloat16 *>(p) + o) = u;
    }
    static __device__ __forceinline__ float ld(const void *p, size_t o) {
        return __bfloat162float(static_cast<const __nv_bfloat16 *>(p)[o]);
    }
};

__device__ __forceinline__ void f4_to(const float4 v, float *a) { a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w; }
__device__ __forceinline__ float4 to_f4(const float *a) { return make_float4(a[0], a[1], a[2], a[3]); }

