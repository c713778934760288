// Shared helpers for the cospdnn_b200 CUDA sources (sm_100a only).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/cospdnn_b200.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ != 1000)
#error "cospdnn_b200 is built for sm_100a only"
#endif

namespace cospdnn {

// Records the calling thread's last error message (cospdnn_last_error).
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t err, const char *what);

#define CSP_CUDA(call)                                              \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ::cospdnn::cuda_fail(_e, #call); \
    } while (0)

#define CSP_CHECK(cond, code, msg)                   \
    do {                                             \
        if (!(cond)) return ::cospdnn::fail(code, msg); \
    } while (0)

// ---- activation storage types ------------------------------------------
template <typename T>
struct act_traits;
template <>
struct act_traits<float> {
    static __device__ __forceinline__ float to_f(float x) { return x; }
    static __device__ __forceinline__ float from_f(float x) { return x; }
    static __device__ __forceinline__ double to_d(float x) { return (double)x; }
    static __device__ __forceinline__ float from_d(double x) { return __double2float_rn(x); }
};
template <>
struct act_traits<__half> {
    static __device__ __forceinline__ float to_f(__half x) { return __half2float(x); }
    static __device__ __forceinline__ __half from_f(float x) { return __float2half_rn(x); }
    static __device__ __forceinline__ double to_d(__half x) { return (double)__half2float(x); }
    static __device__ __forceinline__ __half from_d(double x) { return __double2half(x); }
};
template <>
struct act_traits<__nv_bfloat16> {
    static __device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
    static __device__ __forceinline__ __nv_bfloat16 from_f(float x) { return __float2bfloat16_rn(x); }
    static __device__ __forceinline__ double to_d(__nv_bfloat16 x) { return (double)__bfloat162float(x); }
    static __device__ __forceinline__ __nv_bfloat16 from_d(double x) {
        return __float2bfloat16_rn(__double2float_rn(x));
    }
};

// Order-preserving map float -> uint32 (for atomicMax on possibly negative floats).
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t o) {
    uint32_t b = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return __uint_as_float(b);
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float clamp32(float z) { return fminf(fmaxf(z, 0.0f), 32.0f); }
__device__ __forceinline__ double clamp32d(double z) { return z < 0.0 ? 0.0 : (z > 32.0 ? 32.0 : z); }

}  // namespace cospdnn
