// Device pieces of the learned correction shared by the correction kernels
// (mlp.cu) and the fused coarse step (learned_step.cu): the network's shape and
// parameter layout, the feature row of a 25-point star, and the tcgen05 /
// shared-memory-descriptor helpers.
//
// Features (no reference counterpart): the star of p around a point in a
// difference basis computed in FP32 before the BF16 rounding -- for axis x, y, z
// and r = 1..4 the pair (p_+r - p_-r, p_+r + p_-r - 2 p_c), then p_c, all / s,
// then the local Courant number sqrt(vel2) dt / dx, padded to 32 -- where s is
// the smallest power of two above the star's largest magnitude (0 for an all-zero
// star).  Every kernel scales by 1/s (exact: a power of two) before the BF16
// rounding; rounding the unscaled differences instead gives other bits where
// they are FP32 or BF16 subnormals (the decaying tail ahead of a wave front).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "sb200_common.cuh"

namespace sb200 {
namespace mlp {

constexpr int H = 32;    // hidden width
constexpr int F = 32;    // padded input width
constexpr int NIN = 26;  // real inputs
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + H * F;
constexpr int OFF_W2 = OFF_B1 + H;
constexpr int OFF_B2 = OFF_W2 + H * H;
constexpr int OFF_W3 = OFF_B2 + H;
constexpr int OFF_B3 = OFF_W3 + H;
constexpr int NPARAM = OFF_B3 + 1;  // 2145
constexpr int NSLOT = NPARAM + 1;   // + loss

__device__ __forceinline__ uint32_t pack_bf2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ uint16_t bf16_bits(float x) {
    return static_cast<uint16_t>(pack_bf2(x, 0.f) & 0xffffu);
}
__device__ __forceinline__ uint32_t relu_bf2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// s = the smallest power of two above m = max|star| (m = 0: s = 0), and 1 / s.
// Exponent arithmetic on the bits: m's exponent field plus one (a subnormal m
// counts as 2^-126; m is clamped below 2^126 so that 1 / s stays normal).
__device__ __forceinline__ void pow2_scale(float m, float& s, float& inv) {
    uint32_t e = __float_as_uint(m) & 0x7f800000u;
    e = e < 0x00800000u ? 0x00800000u : (e > 0x7e000000u ? 0x7e000000u : e);
    const uint32_t sb = e + 0x00800000u;
    s = m > 0.f ? __uint_as_float(sb) : 0.f;
    inv = m > 0.f ? __uint_as_float((254u << 23) - sb) : 0.f;
}

// The 25-point star of p around c (centre, then x-4..x-1, x+1..x+4, then y and
// z likewise) and its scale s.  A star whose largest magnitude is below `floor`
// (the network's correction floor; 0 admits every nonzero star) gets s = 0, so
// its correction is exactly zero: ahead of a wavefront the field holds values
// that only underflow if nothing keeps feeding them.
struct Star {
    float v[25];
    float s;
};

__device__ __forceinline__ void gather_star(Star& st, const float* __restrict__ p, int64_t c,
                                            int64_t sy, int64_t sz, float floor = 0.f) {
    st.v[0] = p[c];
    int k = 1;
#pragma unroll
    for (int r = -4; r <= 4; ++r)
        if (r) st.v[k++] = p[c + r];
#pragma unroll
    for (int r = -4; r <= 4; ++r)
        if (r) st.v[k++] = p[c + r * sy];
#pragma unroll
    for (int r = -4; r <= 4; ++r)
        if (r) st.v[k++] = p[c + r * sz];
    float m = 0.f;
#pragma unroll
    for (int j = 0; j < 25; ++j) m = fmaxf(m, fabsf(st.v[j]));
    float inv;
    pow2_scale(m >= floor ? m : 0.f, st.s, inv);
}

// Feature row (32 BF16) of a star (see the file comment): word 4a + r - 1 holds
// axis a's difference and second difference at radius r, word 12 the centre
// and the Courant number, words 13..15 zeros.
__device__ __forceinline__ void feature_row(uint32_t* row, const Star& st, float courant) {
    const float inv = st.s > 0.f ? 1.f / st.s : 0.f;  // exact: s is a power of two
    const float c = st.v[0];
    float f[26];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int r = 1; r <= 4; ++r) {
            const float up = st.v[1 + 8 * a + 3 + r];  // +r: slot 4 + r - 1 of the axis' 8
            const float dn = st.v[1 + 8 * a + 4 - r];  // -r: slot 4 - r
            f[2 * (4 * a + r - 1)] = (up - dn) * inv;
            f[2 * (4 * a + r - 1) + 1] = ((up + dn) - 2.f * c) * inv;
        }
    f[24] = c * inv;
    f[25] = courant;
#pragma unroll
    for (int j = 0; j < 13; ++j) row[j] = pack_bf2(f[2 * j], f[2 * j + 1]);
#pragma unroll
    for (int j = 13; j < 16; ++j) row[j] = 0u;
}

// ── tcgen05 ──────────────────────────────────────────────────────────────────
// Instruction descriptor of an M = 128, N = 32 MMA with BF16 A and B (both
// K-major) and an FP32 accumulator.
constexpr uint32_t kTcIdesc = (1u << 4)                     // D: FP32
                              | (1u << 7) | (1u << 10)      // A, B: BF16 (both K-major)
                              | (uint32_t(32 >> 3) << 17)   // N = 32
                              | (uint32_t(128 >> 4) << 24);  // M = 128

// Byte offset of element (row, k) of a K-major BF16 operand in the no-swizzle
// canonical layout: 8-row x 16-byte core matrices, the 4 K-chunks of a row
// group 128 B apart (leading byte offset), row groups 512 B apart (stride byte
// offset).  A K = 16 step starts 256 B further.
__device__ __forceinline__ uint32_t core_off(int row, int k) {
    return uint32_t((row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return uint64_t((saddr >> 4) & 0x3FFFu)  // start address
           | (uint64_t(128 >> 4) << 16)      // leading byte offset
           | (uint64_t(512 >> 4) << 32)      // stride byte offset
           | (uint64_t(1) << 46);            // descriptor version; no swizzle
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
    const uint32_t mask = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate), "r"(mask)
        : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// One feature / activation row (16 words = 32 BF16) into a K-major operand tile.
__device__ __forceinline__ void store_row(unsigned char* tile, int row, const uint32_t (&w)[16]) {
#pragma unroll
    for (int kc = 0; kc < 4; ++kc)
        *reinterpret_cast<uint4*>(tile + core_off(row, 8 * kc)) =
            make_uint4(w[4 * kc], w[4 * kc + 1], w[4 * kc + 2], w[4 * kc + 3]);
}

}  // namespace mlp
}  // namespace sb200
