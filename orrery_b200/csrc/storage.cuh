// Population storage forms of the device solvers.
//
//   float          f - w in binary32, binary32 arithmetic (the plain form)
//   __half         f - w in binary16, binary32 arithmetic.  No extra scale:
//                  a scale (as in FP16S, Lehmann et al. 2022) only refines
//                  values below binary16's normal range (6e-5), whose
//                  absolute errors are already far below those of the
//                  1e-2-sized deviations that dominate, and would cost a
//                  multiply per load and store
//   __nv_bfloat16  f - w in bfloat16, binary32 arithmetic
//   double         f unshifted in binary64, binary64 arithmetic following the
//                  reference CPU solver's operation order (the FP64 device
//                  oracle)
//
// Storing f - w keeps the O(1e-2) deviations that carry the flow out of the
// rounding error of the O(1) weights (src/aero/lbm3d/lbm3d_gpu.cpp:1-7).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace orr {

template <class S> struct Storage;

template <> struct Storage<float> {
    using A = float;
    static constexpr bool kShifted = true;
    __device__ __forceinline__ static A load(const float* p) { return __ldg(p); }
    __device__ __forceinline__ static A value(float v) { return v; }
    __device__ __forceinline__ static void store(float* p, A v) { *p = v; }
    __host__ __device__ static float encode(double shifted) { return static_cast<float>(shifted); }
    __host__ __device__ static double decode(float s) { return static_cast<double>(s); }
};

template <> struct Storage<__half> {
    using A = float;
    static constexpr bool kShifted = true;
    __device__ __forceinline__ static A load(const __half* p) {
        return __half2float(__ldg(p));
    }
    __device__ __forceinline__ static A value(__half v) { return __half2float(v); }
    __device__ __forceinline__ static void store(__half* p, A v) {
        *p = __float2half_rn(v);
    }
    // Two neighbouring values as one aligned 32-bit word (lower address in
    // the low half).
    __device__ __forceinline__ static A lo(uint32_t w) {
        return __half2float(__ushort_as_half(static_cast<unsigned short>(w & 0xffffu)));
    }
    __device__ __forceinline__ static A hi(uint32_t w) {
        return __half2float(__ushort_as_half(static_cast<unsigned short>(w >> 16)));
    }
    __device__ __forceinline__ static uint32_t pack(A a, A b) {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
    __device__ static __half encode(double shifted) {
        return __float2half_rn(static_cast<float>(shifted));
    }
    __device__ static double decode(__half s) {
        return static_cast<double>(__half2float(s));
    }
};

template <> struct Storage<__nv_bfloat16> {
    using A = float;
    static constexpr bool kShifted = true;
    __device__ __forceinline__ static A load(const __nv_bfloat16* p) {
        return __bfloat162float(__ldg(p));
    }
    __device__ __forceinline__ static A value(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, A v) {
        *p = __float2bfloat16_rn(v);
    }
    __device__ __forceinline__ static A lo(uint32_t w) {
        return __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(w & 0xffffu)));
    }
    __device__ __forceinline__ static A hi(uint32_t w) {
        return __bfloat162float(__ushort_as_bfloat16(static_cast<unsigned short>(w >> 16)));
    }
    __device__ __forceinline__ static uint32_t pack(A a, A b) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const uint32_t*>(&h);
    }
    __device__ static __nv_bfloat16 encode(double shifted) {
        return __float2bfloat16_rn(static_cast<float>(shifted));
    }
    __device__ static double decode(__nv_bfloat16 s) {
        return static_cast<double>(__bfloat162float(s));
    }
};

template <> struct Storage<double> {
    using A = double;
    static constexpr bool kShifted = false;
    __device__ __forceinline__ static A load(const double* p) { return __ldg(p); }
    __device__ __forceinline__ static A value(double v) { return v; }
    __device__ __forceinline__ static void store(double* p, A v) { *p = v; }
    __host__ __device__ static double encode(double unshifted) { return unshifted; }
    __host__ __device__ static double decode(double s) { return s; }
};

} // namespace orr
