// Shared device helpers for the sm_100a stencil kernels: the radius-4 coefficients,
// the folded per-axis weights, PTX wrappers for mbarriers and TMA, and the bounded
// waits every spin in this library goes through.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sb200 {

constexpr int R = 4;  // stencil radius (8th order), include/stencil/types.hpp:42-44 of the reference

// FDCoeffs<4> of the reference (include/stencil/types.hpp:175-181): the same
// double-precision quotients rounded once to float, so host and device agree.
constexpr float C0 = static_cast<float>(-205.0 / 72.0);
constexpr float C1 = static_cast<float>(8.0 / 5.0);
constexpr float C2 = static_cast<float>(-1.0 / 5.0);
constexpr float C3 = static_cast<float>(8.0 / 315.0);
constexpr float C4 = static_cast<float>(-1.0 / 560.0);

// Laplacian weights with the grid spacing (and the time-step factor) folded in,
// computed on the host once per launch.  Per axis a:
//   lap_a = ca*p + sum_r aa[r]*(p[+r] + p[-r]),   lap = (lap_x + lap_y) + lap_z,
// evaluated so that each axis' large centre term cancels against its r = 1 pair
// in one fused step, as the reference's per-axis sums do.
struct Weights {
    float cx, cy, cz;
    float ax[R], ay[R], az[R];
};

// Codes a kernel writes to the library's device error word (a __device__ int
// defined in capi.cu whose address every launch passes in) when a bounded wait
// gives up.  The host reads and clears it with sb200_device_error().
enum DeviceError : int {
    kDevOk = 0,
    kDevWaitTimeout = 1,
};

// Upper bound for any spin in device code, in SM clock cycles (about one second
// at the B200's boost clock).
constexpr long long kWaitLimitCycles = 2000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Rounds a pointer into dynamic shared memory up to A bytes (A a power of two) by
// pointer arithmetic on the pointer itself: a round trip through an integer
// would hide the shared address space from the compiler and turn every access
// through the result into a generic load or store.
template <unsigned A>
__device__ __forceinline__ unsigned char* smem_align(unsigned char* p) {
    return p + ((A - (smem_u32(p) & (A - 1u))) & (A - 1u));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Invalidates a barrier whose phases have all completed, before it is
// initialised again.
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the barrier phase with the given parity; gives up after
// kWaitLimitCycles and returns false (the caller records the error and exits).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > kWaitLimitCycles) return false;
    }
    return true;
}

// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
// The innermost coordinate x must be a multiple of 16 bytes / element size;
// callers guarantee it (tile origins are multiples of 4 floats / 8 halves).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Streaming 128-bit global accesses: read-only inputs bypass L1, outputs are
// marked evict-first.
__device__ __forceinline__ float4 ldg_stream(const float* p) {
    float4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
}

// Coherent streaming load, for inputs the same launch may overwrite in place
// (p_prev when p_next aliases it): each element is read once, then written by
// the same thread, so no other reader can observe a stale line.
__device__ __forceinline__ float4 ldg_cs(const float* p) {
    float4 v;
    asm volatile("ld.global.cs.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

__device__ __forceinline__ uint4 ldg_cs_u4(const void* p) {
    uint4 v;
    asm volatile("ld.global.cs.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

__device__ __forceinline__ void stg_stream(float* p, float4 v) {
    asm volatile("st.global.cs.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y),
                 "f"(v.z), "f"(v.w)
                 : "memory");
}

__device__ __forceinline__ uint4 ldg_stream_u4(const void* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

__device__ __forceinline__ void stg_stream_u4(void* p, uint4 v) {
    asm volatile("st.global.cs.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x), "r"(v.y),
                 "r"(v.z), "r"(v.w)
                 : "memory");
}

__device__ __forceinline__ float4 lds128(const float* p) {
    return *reinterpret_cast<const float4*>(p);
}

__device__ __forceinline__ void record_error(int* err, int code) {
    if (err) atomicCAS(err, 0, code);
}

__device__ __forceinline__ float f4get(const float4& v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Packed FP32 pairs (sm_100 f32x2 instructions): each lane is rounded exactly
// as the scalar fmaf / + / * would round it, so packed and scalar code give the
// same bits.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 dup2(float s) { return make_float2(s, s); }
// Pair h (0: lanes 0-1, 1: lanes 2-3) of a float4.
__device__ __forceinline__ float2 pair_of(const float4& v, int h) {
    return h == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
}

}  // namespace sb200
