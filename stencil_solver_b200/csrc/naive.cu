// Naive one-thread-per-point kernels.
//
// These restate the reference's launch_naive arithmetic (src/kernels/stencil_naive.cu:49-89)
// in exactly the order of its CPU branch (stencil_naive.cu:151-169): every product and sum
// goes through __fmul_rn / __fadd_rn, so nvcc cannot contract them into FMAs and the
// result is bit-identical to the oracle's FP32 restatement built with -ffp-contract=off.
// They serve as launch_naive, as the fallback for grids the TMA pencil kernels cannot map
// (row pitch not a multiple of 16 bytes, unaligned base pointers), and as an in-repo
// cross-check of the pencil kernels.
#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {

struct NaiveArgs {
    const float* cur;
    const float* prev;  // wave: p at t-dt; heat: unused
    const float* vel2;  // wave: v^2 field; heat: unused
    float* next;
    int64_t nx, ny, nz;
    float inv_dx2, inv_dy2, inv_dz2;
    float k;  // wave: dt^2; heat: alpha*dt
    int64_t src;  // flat source index or -1
    float src_w;  // wavelet sample for this step (when wavelet == nullptr)
    const float* wavelet;  // device samples: wavelet[*step + step_off]
    const int* step;
    int step_off;
    float* trace;  // value at the source after the step, at [(*step or 0) + step_off]
};

template <bool kHeat>
__global__ void __launch_bounds__(256) naive_kernel(NaiveArgs a) {
    const int64_t ix = R + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t iy = R + static_cast<int64_t>(blockIdx.y) * blockDim.y + threadIdx.y;
    const int64_t iz = R + static_cast<int64_t>(blockIdx.z) * blockDim.z + threadIdx.z;
    if (ix >= a.nx - R || iy >= a.ny - R || iz >= a.nz - R) return;

    const int64_t sy = a.nx;
    const int64_t sz = a.nx * a.ny;
    const int64_t c = iz * sz + iy * sy + ix;
    const float* p = a.cur;
    const float cf[R + 1] = {C0, C1, C2, C3, C4};

    const float pc = p[c];
    float lx = __fmul_rn(__fmul_rn(cf[0], pc), a.inv_dx2);
    float ly = __fmul_rn(__fmul_rn(cf[0], pc), a.inv_dy2);
    float lz = __fmul_rn(__fmul_rn(cf[0], pc), a.inv_dz2);
#pragma unroll
    for (int r = 1; r <= R; ++r) {
        lx = __fadd_rn(lx, __fmul_rn(__fmul_rn(cf[r], __fadd_rn(p[c + r], p[c - r])), a.inv_dx2));
        ly = __fadd_rn(ly, __fmul_rn(__fmul_rn(cf[r], __fadd_rn(p[c + r * sy], p[c - r * sy])),
                                     a.inv_dy2));
        lz = __fadd_rn(lz, __fmul_rn(__fmul_rn(cf[r], __fadd_rn(p[c + r * sz], p[c - r * sz])),
                                     a.inv_dz2));
    }
    const float lap = __fadd_rn(__fadd_rn(lx, ly), lz);
    float out;
    if (kHeat) {
        // 2u - u is exact, so the reference's heat arithmetic reduces to u + k*lap.
        out = __fadd_rn(pc, __fmul_rn(a.k, lap));
    } else {
        const float kv = __fmul_rn(a.k, a.vel2[c]);
        out = __fadd_rn(__fsub_rn(__fmul_rn(2.0f, pc), a.prev[c]), __fmul_rn(kv, lap));
        if (c == a.src) {
            const float w = a.wavelet ? a.wavelet[*a.step + a.step_off] : a.src_w;
            out = __fadd_rn(out, __fmul_rn(kv, w));
            if (a.trace) a.trace[(a.step ? *a.step : 0) + a.step_off] = out;
        }
    }
    a.next[c] = out;
}

NaiveArgs make_args(const float* cur, const float* prev, const float* vel2, float* next,
                    const GridDesc& g, float k, int64_t src, float src_w) {
    NaiveArgs a{};
    a.cur = cur;
    a.prev = prev;
    a.vel2 = vel2;
    a.next = next;
    a.nx = g.nx;
    a.ny = g.ny;
    a.nz = g.nz;
    // Host-side reciprocals in float, as the reference launcher computes them
    // (stencil_naive.cu:96-99).
    a.inv_dx2 = 1.0f / (g.dx * g.dx);
    a.inv_dy2 = 1.0f / (g.dy * g.dy);
    a.inv_dz2 = 1.0f / (g.dz * g.dz);
    a.k = k;
    a.src = src;
    a.src_w = src_w;
    return a;
}

dim3 naive_grid(const GridDesc& g, dim3 block) {
    const int64_t ix = g.nx - 2 * R, iy = g.ny - 2 * R, iz = g.nz - 2 * R;
    return dim3(static_cast<unsigned>((ix + block.x - 1) / block.x),
                static_cast<unsigned>((iy + block.y - 1) / block.y),
                static_cast<unsigned>((iz + block.z - 1) / block.z));
}

}  // namespace

cudaError_t launch_wave_naive(const float* cur, const float* prev, const float* vel2,
                              float* next, const GridDesc& g, const SourceDesc& src,
                              cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const float dt2 = g.dt * g.dt;
    const dim3 block(32, 4, 2);
    NaiveArgs a = make_args(cur, prev, vel2, next, g, dt2, src.idx, src.w);
    a.wavelet = src.wavelet;
    a.step = src.step;
    a.step_off = src.step_offset;
    a.trace = src.trace;
    naive_kernel<false><<<naive_grid(g, block), block, 0, stream>>>(a);
    return cudaGetLastError();
}

namespace {
__global__ void set_int_kernel(int* dst, int value) { *dst = value; }
}  // namespace

cudaError_t launch_set_int(int* dst, int value, cudaStream_t stream) {
    set_int_kernel<<<1, 1, 0, stream>>>(dst, value);
    return cudaGetLastError();
}

cudaError_t launch_heat_naive(const float* u, float* u_next, const GridDesc& g, float alpha_dt,
                              cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const dim3 block(32, 4, 2);
    naive_kernel<true><<<naive_grid(g, block), block, 0, stream>>>(
        make_args(u, nullptr, nullptr, u_next, g, alpha_dt, -1, 0.0f));
    return cudaGetLastError();
}

}  // namespace sb200
