// FP64 reductions over a field's interior: sum of squares, largest magnitude and
// the number of non-finite values, for the stability monitor and for choosing
// the power-of-two storage scale of the FP16 path.
//
// Two launches on the caller's stream: pass 1 has every block reduce a strided
// share of the interior rows into three doubles in a scratch array; pass 2 (one
// block) folds the partials into out[3].  Each row of the interior is contiguous
// in memory, so a warp reads coalesced runs of x.  The accumulations are in
// double; a value of the field is read once (8 B/point of FP32 traffic less than
// the stencil step it accompanies).
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {

constexpr int kStatsThreads = 256;

template <typename T>
__device__ __forceinline__ float load_value(const T* f, int64_t i);

template <>
__device__ __forceinline__ float load_value<float>(const float* f, int64_t i) {
    return f[i];
}

template <>
__device__ __forceinline__ float load_value<__half>(const __half* f, int64_t i) {
    return __half2float(f[i]);
}

__device__ __forceinline__ void block_reduce3(double& s, double& m, double& bad) {
    __shared__ double red[3][kStatsThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        bad += __shfl_down_sync(0xffffffffu, bad, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = s;
        red[1][warp] = m;
        red[2][warp] = bad;
    }
    __syncthreads();
    if (warp == 0) {
        constexpr int nw = kStatsThreads / 32;
        s = lane < nw ? red[0][lane] : 0.0;
        m = lane < nw ? red[1][lane] : 0.0;
        bad = lane < nw ? red[2][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o);
            m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
            bad += __shfl_down_sync(0xffffffffu, bad, o);
        }
    }
}

// Pass 1: block b reduces interior rows b, b + gridDim.x, ... (a row is one
// (y, z) pair) into partials[3*b .. 3*b+2].
template <typename T>
__global__ void __launch_bounds__(kStatsThreads)
    stats_partial_kernel(const T* f, int64_t nx, int64_t ny, int64_t nz, float inv_scale,
                         double* partials) {
    const int64_t ix = nx - 2 * R, iy = ny - 2 * R, iz = nz - 2 * R;
    const int64_t rows = iy * iz;
    double s = 0.0, m = 0.0, bad = 0.0;
    for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
        const int64_t y = R + r % iy, z = R + r / iy;
        const int64_t base = (z * ny + y) * nx + R;
        for (int64_t x = threadIdx.x; x < ix; x += blockDim.x) {
            const float v = load_value<T>(f, base + x) * inv_scale;
            if (isfinite(v)) {
                const double d = static_cast<double>(v);
                s = fma(d, d, s);
                m = fmax(m, fabs(d));
            } else {
                bad += 1.0;
            }
        }
    }
    block_reduce3(s, m, bad);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x + 0] = s;
        partials[3 * blockIdx.x + 1] = m;
        partials[3 * blockIdx.x + 2] = bad;
    }
}

// Pass 2: one block folds nparts partials into out[3] (sum in a fixed order,
// so repeated runs give identical bits).
__global__ void __launch_bounds__(kStatsThreads)
    stats_final_kernel(const double* partials, int nparts, double* out) {
    double s = 0.0, m = 0.0, bad = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        s += partials[3 * i + 0];
        m = fmax(m, partials[3 * i + 1]);
        bad += partials[3 * i + 2];
    }
    block_reduce3(s, m, bad);
    if (threadIdx.x == 0) {
        out[0] = s;
        out[1] = m;
        out[2] = bad;
    }
}

}  // namespace

int stats_blocks(const GridDesc& g) {
    const int64_t rows = (g.ny - 2 * R) * (g.nz - 2 * R);
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(rows, kMaxStatsBlocks)));
}

cudaError_t launch_field_stats(const void* field, bool half, const GridDesc& g, float scale,
                               double* out3, double* scratch, cudaStream_t stream) {
    const int nb = stats_blocks(g);
    const float inv = 1.0f / scale;
    if (half)
        stats_partial_kernel<__half><<<nb, kStatsThreads, 0, stream>>>(
            static_cast<const __half*>(field), g.nx, g.ny, g.nz, inv, scratch);
    else
        stats_partial_kernel<float><<<nb, kStatsThreads, 0, stream>>>(
            static_cast<const float*>(field), g.nx, g.ny, g.nz, inv, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    stats_final_kernel<<<1, kStatsThreads, 0, stream>>>(scratch, nb, out3);
    return cudaGetLastError();
}

}  // namespace sb200
