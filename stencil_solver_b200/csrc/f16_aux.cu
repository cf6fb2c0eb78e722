// Element-wise helpers of the FP16-storage path and its device-side
// renormalisation.
//
//   pack   : h[i] = fp16(f[i] * scale)          (round to nearest even)
//   unpack : f[i] = float(h[i]) / scale
//   k_bf16 : K[i] = bf16(vel2[i] * dt^2 / dx^2) (round to nearest even)
//   renorm : picks the storage scale for the next window of steps from the FP64
//            statistics of the current field -- a_new = 2^floor(log2(target /
//            (max|p| + source bound))) -- and records r = a_new / a_old.
// All are grid-stride kernels on the caller's stream; renorm is one thread so a
// captured CUDA graph can replay it without a host round trip.
#include <cuda_fp16.h>

#include <cmath>

#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {

__global__ void pack_kernel(const float* __restrict__ f, uint16_t* __restrict__ h, int64_t n,
                            float scale) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        h[i] = __half_as_ushort(__float2half_rn(f[i] * scale));
}

__global__ void unpack_kernel(const uint16_t* __restrict__ h, float* __restrict__ f, int64_t n,
                              float inv_scale) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        f[i] = __half2float(__ushort_as_half(h[i])) * inv_scale;
}

// Round-to-nearest-even float -> bf16 on the bit pattern (NaN kept quiet).
__device__ __forceinline__ uint16_t to_bf16(float x) {
    const uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x007fffffu))
        return static_cast<uint16_t>((u >> 16) | 0x40u);
    return static_cast<uint16_t>((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

__global__ void k_bf16_kernel(const float* __restrict__ vel2, uint16_t* __restrict__ k, int64_t n,
                              float dt2_over_dx2) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x)
        k[i] = to_bf16(vel2[i] * dt2_over_dx2);
}

__global__ void renorm_kernel(const double* stats3, F16Scale* scale, const float* bound,
                              const int* step, float bound_host, float target) {
    const double a_old = scale->a;
    const double m = stats3[1] / a_old;  // stats were taken in stored units
    const double b = bound ? double(bound[*step]) : double(bound_host);
    double a_new = a_old;
    if (m + b > 0.0) {
        const int e = static_cast<int>(floor(log2(double(target) / (m + b))));
        a_new = ldexp(1.0, max(-120, min(120, e)));
    }
    scale->r = static_cast<float>(a_new / a_old);
    scale->a = static_cast<float>(a_new);
}

unsigned grid_for(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return static_cast<unsigned>(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace

cudaError_t launch_f16_pack(const float* f, uint16_t* h, int64_t n, float scale,
                            cudaStream_t st) {
    pack_kernel<<<grid_for(n), 256, 0, st>>>(f, h, n, scale);
    return cudaGetLastError();
}

cudaError_t launch_f16_unpack(const uint16_t* h, float* f, int64_t n, float scale,
                              cudaStream_t st) {
    unpack_kernel<<<grid_for(n), 256, 0, st>>>(h, f, n, 1.0f / scale);
    return cudaGetLastError();
}

cudaError_t launch_k_bf16(const float* vel2, uint16_t* k, int64_t n, float dt2_over_dx2,
                          cudaStream_t st) {
    k_bf16_kernel<<<grid_for(n), 256, 0, st>>>(vel2, k, n, dt2_over_dx2);
    return cudaGetLastError();
}

cudaError_t launch_f16_renorm(const double* stats3, F16Scale* scale, const float* bound,
                              const int* step, float bound_host, float target, cudaStream_t st) {
    renorm_kernel<<<1, 1, 0, st>>>(stats3, scale, bound, step, bound_host, target);
    return cudaGetLastError();
}

}  // namespace sb200
