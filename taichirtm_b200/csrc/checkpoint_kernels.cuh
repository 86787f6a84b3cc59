// Compressed wavefield checkpoints: the 5 P-SV state fields of every shot
// stored as FP16 or BF16 with one scale per (checkpoint, field, shot).
//
// pack:   amax = max |x| over the shot's block of the field (absmax kernel),
//         h = round(x * 32752 / amax)   (FP16: the largest magnitude maps to
//         2^15 - 16, well inside the 65504 range; BF16 uses the same scale)
// unpack: x = float(h) * amax / 32752
// A field that is all zero has amax = 0 and is restored as zeros.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "step_kernels.cuh"

namespace rtm {

constexpr float CKPT_RANGE = 32752.0f;

struct CkptParams {
    const float *src[5];   // FP32 fields (pack) / unused (unpack)
    float *dst[5];         // FP32 fields (unpack)
    void *half;            // 5 consecutive fields of `sf` elements of T
    unsigned int *amax;    // [5][nshots] max |x| as float bits
    const ShotDev *shots;
    int nshots;
    int pitch;
    size_t sf;             // elements per field
};

template <typename T>
__device__ __forceinline__ T to_low(float x);
template <>
__device__ __forceinline__ __half to_low<__half>(float x) { return __float2half_rn(x); }
template <>
__device__ __forceinline__ __nv_bfloat16 to_low<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
__device__ __forceinline__ float from_low(__half h) { return __half2float(h); }
__device__ __forceinline__ float from_low(__nv_bfloat16 h) { return __bfloat162float(h); }

// grid: (chunks, nshots, 5)
static __global__ void ckpt_absmax_kernel(CkptParams cp) {
    const int s = blockIdx.y, f = blockIdx.z;
    const ShotDev sh = cp.shots[s];
    const long long n = (long long)(sh.nx + 2) * cp.pitch;
    const float *x = cp.src[f] + sh.state_off;
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(cp.amax + f * cp.nshots + s, __float_as_uint(m));
}

template <typename T>
static __global__ void ckpt_pack_kernel(CkptParams cp) {
    const int s = blockIdx.y, f = blockIdx.z;
    const ShotDev sh = cp.shots[s];
    const long long n = (long long)(sh.nx + 2) * cp.pitch;
    const float *x = cp.src[f] + sh.state_off;
    T *h = static_cast<T *>(cp.half) + (size_t)f * cp.sf + sh.state_off;
    const float amax = __uint_as_float(cp.amax[f * cp.nshots + s]);
    const float inv = amax > 0.f ? CKPT_RANGE / amax : 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        h[i] = to_low<T>(x[i] * inv);
}

template <typename T>
static __global__ void ckpt_unpack_kernel(CkptParams cp) {
    const int s = blockIdx.y, f = blockIdx.z;
    const ShotDev sh = cp.shots[s];
    const long long n = (long long)(sh.nx + 2) * cp.pitch;
    const T *h = static_cast<const T *>(cp.half) + (size_t)f * cp.sf + sh.state_off;
    float *x = cp.dst[f] + sh.state_off;
    const float scale = __uint_as_float(cp.amax[f * cp.nshots + s]) / CKPT_RANGE;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        x[i] = from_low(h[i]) * scale;
}

}  // namespace rtm
