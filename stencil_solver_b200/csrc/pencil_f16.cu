// FP16-storage acoustic pencil kernel for sm_100a.
//
// Storage: p and p_prev in FP16, both holding a * p for one power-of-two scale
// a (kept in a device-side F16Scale); K = vel2 * dt^2 / dx^2 in BF16.  All
// arithmetic is FP32 and the output is rounded to FP16 once.  DRAM traffic: 8 B
// per interior point (read p, p_prev, K; write p_next in place over p_prev).
//
// Layout of a CTA's work is the FP32 kernel's (pencil_f32.cu) with 2-byte
// elements: each thread owns 8 consecutive x (one 16-byte chunk) of one row.
// Because the interior starts at x = 4 (byte 8), tiles are aligned to x = 8k
// and the p box starts 8 halves left of the tile (16-byte aligned TMA origin,
// box TX + 16 wide); points of a chunk outside the interior are never stored.
//
// The kernel is bound by the FP32 pipe that also executes the FP16 -> FP32
// conversions, so every choice below is about issuing fewer of them:
//   * y neighbours come from the staged FP16 plane; each pair (up, down) costs
//     one conversion and one mixed FP16 + FP32 add (add.f32.f16), not two
//     conversions and an add.
//   * the z queue is split by role.  The centre plane and the four planes above
//     it stay FP16 in registers (the up operand of a z pair enters through the
//     mixed add); the four planes below the centre are FP32 -- each plane is
//     converted once, when it is the centre (the x window converts it anyway),
//     and is then the down operand of four z pairs.  Both register rings have 4
//     slots (plane index mod 4) and the plane loop is unrolled by 4, so every
//     slot is a compile-time register and nothing is shifted.
//   * arithmetic on point pairs uses the packed f32x2 instructions; the
//     Laplacian is two FMA chains (x and y from the combined centre term, z from
//     its first pair) added once.
//
// Renormalisation (driven by the FP64 statistics every few dozen steps): a
// renorm step (PHASE 1) scales its output by r = a_new / a_old; the step after
// it (PHASE 2) scales p_prev, still at a_old, by r; other steps (PHASE 0) carry
// no scale arithmetic.  Powers of two make every rescale exact.
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>

#include "batch.h"
#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {


template <int TX, int TY, int S, int AUX>
struct ShapeH {
    static_assert(TX % 8 == 0, "TX must be a multiple of 8 halves (16-byte chunks)");
    static_assert(S >= 8 && S % 4 == 0 && 4 % AUX == 0, "rings (the plane loop is unrolled by 4)");
    static constexpr int SX = TX + 16;  // halves per staged row: 8 left, TX, 8 right
    static constexpr int SY = TY + 2 * R;
    static_assert(SX <= 256 && SY <= 256, "TMA box extent is at most 256");
    static constexpr int TPR = TX / 8;
    static constexpr int NT = TPR * TY;
    static constexpr uint32_t PLANE_BYTES = SX * SY * 2u;
    static constexpr int PLANE = int(((PLANE_BYTES + 127u) / 128u) * 64u);  // stride, halves
    static constexpr uint32_t TILE_BYTES = TX * TY * 2u;
    static constexpr int TILE = int(((TILE_BYTES + 127u) / 128u) * 64u);
    static constexpr size_t SMEM = size_t(S) * PLANE * 2 + size_t(AUX) * 2 * TILE * 2 + 128;
    static constexpr int MINB = (512 / NT) > 0 ? (512 / NT) : 1;
};

__device__ __forceinline__ float bf2f(uint32_t word, int hi) {
    return __uint_as_float(hi ? (word & 0xffff0000u) : (word << 16));
}

__device__ __forceinline__ uint32_t get_word(const uint4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

__device__ __forceinline__ uint32_t pack_h2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// Both halves of a word as FP32 (exact), taken apart with a register-pair move.
__device__ __forceinline__ float2 h2f2(uint32_t w) {
    float a, b;
    asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\t"
        "cvt.f32.f16 %0, lo;\n\tcvt.f32.f16 %1, hi;\n\t}"
        : "=f"(a), "=f"(b)
        : "r"(w));
    return make_float2(a, b);
}

// f32(half) + b for both halves of a word (the sm_100 mixed-precision add).
__device__ __forceinline__ float2 addhf2(uint32_t w, float2 b) {
    float x, y;
    asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\t"
        "add.rn.f32.f16 %0, lo, %3;\n\tadd.rn.f32.f16 %1, hi, %4;\n\t}"
        : "=f"(x), "=f"(y)
        : "r"(w), "f"(b.x), "f"(b.y));
    return make_float2(x, y);
}

__device__ __forceinline__ uint2 lds64(const uint16_t* p) {
    return *reinterpret_cast<const uint2*>(p);
}
__device__ __forceinline__ uint4 lds128h(const uint16_t* p) {
    return *reinterpret_cast<const uint4*>(p);
}

// Streaming stores under a predicate (no branch: the three store shapes of a
// chunk -- whole, upper half, lower half -- are issued with per-thread predicates).
__device__ __forceinline__ void stg_stream_u4_if(void* p, uint4 v, bool pred) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t"
        "@q st.global.cs.v4.u32 [%0], {%1, %2, %3, %4};\n\t}" ::"l"(p),
        "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(static_cast<uint32_t>(pred))
        : "memory");
}
__device__ __forceinline__ void stg_stream_u2_if(void* p, uint2 v, bool pred) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t"
        "@q st.global.cs.v2.u32 [%0], {%1, %2};\n\t}" ::"l"(p),
        "r"(v.x), "r"(v.y), "r"(static_cast<uint32_t>(pred))
        : "memory");
}

// b - f32(half) for both halves of a word: the sm_100 mixed-precision FMA
// f32(half) * (-1) + b, whose product is exact, so one rounding of b - half.
__device__ __forceinline__ float2 rsubhf2(uint32_t w, float2 b) {
    float x, y;
    asm("{\n\t.reg .b16 lo, hi, m1;\n\tmov.b32 {lo, hi}, %2;\n\tmov.b16 m1, 0xBC00;\n\t"
        "fma.rn.f32.f16 %0, lo, m1, %3;\n\tfma.rn.f32.f16 %1, hi, m1, %4;\n\t}"
        : "=f"(x), "=f"(y)
        : "r"(w), "f"(b.x), "f"(b.y));
    return make_float2(x, y);
}

// c + f32(half `hi` of word w) * f32(half m): the sm_100 mixed-precision FMA (the
// product of two halves is exact in FP32, so one rounding, as an FP32 FMA of the
// same values).
__device__ __forceinline__ float fmahf(uint32_t w, int hi, uint16_t m, float c) {
    float d;
    if (hi)
        asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %1;\n\t"
            "fma.rn.f32.f16 %0, hi, %2, %3;\n\t}"
            : "=f"(d)
            : "r"(w), "h"(m), "f"(c));
    else
        asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %1;\n\t"
            "fma.rn.f32.f16 %0, lo, %2, %3;\n\t}"
            : "=f"(d)
            : "r"(w), "h"(m), "f"(c));
    return d;
}

// The y weights of an isotropic x-y grid scaled by 5040, the least common
// multiple of the coefficients' denominators: 8064, -1008, 128, -9, all exact
// halves (FDCoeffs<4> c_1..c_4 = 8/5, -1/5, 8/315, -1/560).
__host__ __device__ constexpr uint16_t y_weight5040(int r) {  // r = 1..4
    return r == 1 ? 0x6FE0u : r == 2 ? 0xE3E0u : r == 3 ? 0x5800u : 0xC880u;
}
constexpr float kInv5040 = 1.0f / 5040.0f;

// f32(half `hi` of word w) + c (the mixed add on one point).
__device__ __forceinline__ float addhf(uint32_t w, int hi, float c) {
    float d;
    if (hi)
        asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %1;\n\tadd.rn.f32.f16 %0, hi, %2;\n\t}"
            : "=f"(d)
            : "r"(w), "f"(c));
    else
        asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %1;\n\tadd.rn.f32.f16 %0, lo, %2;\n\t}"
            : "=f"(d)
            : "r"(w), "f"(c));
    return d;
}

// x pair sum x[e+r] + x[e-r] for point e of a chunk: own points as FP32 (c,
// 8 values), the 4 halves left (lf) and right (rt) of the chunk as FP16.  No pair
// reaches both sides (r <= 4), so a pair with a side value takes it through the
// mixed add and the side halves are never converted; the sum is the same FP32
// add either way.
__device__ __forceinline__ float xsum1(const float (&c)[8], uint2 lf, uint2 rt, int e, int r) {
    const int up = e + r, dn = e - r;
    if (up >= 8) {
        const int k = up - 8;  // right half k: word k / 2, half k % 2
        return addhf(k < 2 ? rt.x : rt.y, k & 1, c[dn]);
    }
    if (dn < 0) {
        const int k = dn + 4;  // left half k
        return addhf(k < 2 ? lf.x : lf.y, k & 1, c[up]);
    }
    return c[up] + c[dn];
}

// Ring position a persistent CTA carries from one tile to the next: the
// sequence numbers of the next p plane and the next aux iteration.  Stage =
// seq % ring size, phase parity = (seq / ring size) & 1, so its mbarriers are
// initialised once and their phases continue across the tiles it sweeps.
struct RingH {
    uint32_t p = 0;
    uint32_t aux = 0;
};

// Update formulas of the step (template parameter UPD):
//   kUpdConvert:  p_prev converted to FP32, then fma(K, lap, fma(-m_q, pq, 2c));
//   kUpdMixedSub: u = fma(K, lap, 2c), then u - pq in one mixed-precision FMA
//                 (pq x -1 + u) that converts p_prev on the way;
//                 PHASE 2 (p_prev rescaled) uses kUpdConvert.
// and, as a flag, the y pairs:
//   kUpdExactY:   on a grid with dx == dy each y neighbour enters through one
//                 mixed-precision FMA with the 5040-scaled weights (no conversion,
//                 no pair add), accumulated apart and scaled by 1/5040 once;
//                 without it a y pair costs a conversion, a mixed add and an FMA.
constexpr int kUpdConvert = 0, kUpdMixedSub = 1, kUpdExactY = 2;

// One tile: columns [tx TX, tx TX + TX) x rows [4 + ty TY, ...) of the interior,
// marched over z chunk zc.  All threads of the CTA call it; `sm`, `full` and
// `auxf` are the CTA's rings.  CARRY false: their mbarriers are freshly
// initialised (phase 0 on every stage) and the ring positions are compile-time;
// CARRY true: `ring` gives the positions (advanced on return).  Every copy it
// issues has landed when it returns; false means a bounded wait gave up (the
// error is recorded).
template <int TX, int TY, int S, int AUX, int PHASE, int UNR, bool CARRY, int UPD>
__device__ __forceinline__ bool pencil_f16_tile(const CUtensorMap* pmap, const CUtensorMap* qmap,
                                                const CUtensorMap* kmap, const F16Args& a,
                                                int tx, int ty, int zc, uint16_t* sm,
                                                uint64_t* full, uint64_t* auxf, RingH& ring) {
    using P = ShapeH<TX, TY, S, AUX>;
    const uint32_t pb = CARRY ? ring.p : 0u;    // sequence number of plane 0
    const uint32_t ab = CARRY ? ring.aux : 0u;  // sequence number of aux iteration 0
    uint16_t* aux = sm + S * P::PLANE;  // AUX stages of [p_prev tile | K tile]

    const int tid = threadIdx.x;
    const int lx = tid % P::TPR;
    const int ly = tid / P::TPR;
    const int xa = tx * TX;      // first x of the tile (multiple of 8)
    const int y0 = R + ty * TY;  // first interior row of the tile
    const int zb = R + zc * a.zlen;
    const int ze = min(zb + a.zlen, a.nz - R);
    const int nint = ze - zb;
    const int nplanes = nint + 2 * R;

    if (tid == 0) {
        prefetch_tmap(pmap);
        prefetch_tmap(qmap);
        prefetch_tmap(kmap);
    }
    int issued_hi = -1, aux_issued_hi = -1;
    auto issue_plane = [&](int j) {  // thread 0 only
        const uint32_t st = (pb + j) % S;
        mbar_arrive_expect_tx(&full[st], P::PLANE_BYTES);
        tma_load_3d(sm + st * P::PLANE, pmap, &full[st], xa - 8, y0 - R, zb - R + j);
        issued_hi = j;
    };
    auto issue_aux = [&](int it) {  // thread 0 only
        const uint32_t sa = (ab + it) % AUX;
        uint16_t* st = aux + sa * 2 * P::TILE;
        mbar_arrive_expect_tx(&auxf[sa], 2 * P::TILE_BYTES);
        tma_load_3d(st, qmap, &auxf[sa], xa, y0, zb + it);
        tma_load_3d(st + P::TILE, kmap, &auxf[sa], xa, y0, zb + it);
        aux_issued_hi = it;
    };
    auto wait_plane = [&](int j) { return mbar_wait(&full[(pb + j) % S], ((pb + j) / S) & 1u); };
    auto wait_aux = [&](int it) {
        return mbar_wait(&auxf[(ab + it) % AUX], ((ab + it) / AUX) & 1u);
    };
    if (tid == 0) {
        for (int s = 0; s < S && s < nplanes; ++s) issue_plane(s);
        for (int it = 0; it < AUX && it < nint; ++it) issue_aux(it);
    }

    const int gx = xa + 8 * lx;  // first x of this thread's chunk
    const int gy = y0 + ly;
    // With nx % 8 == 0 a chunk is wholly interior, wholly halo, or (at the two x
    // edges) half and half: x = 0..7 stores its upper 4 points, x = nx-8..nx-1
    // its lower 4.
    const bool xfull = gx >= R && gx + 8 <= a.nx - R;
    const bool xany = gx + 8 > R && gx < a.nx - R;
    const bool rin = xany && gy < a.ny - R;
    const bool st_full = rin && xfull;           // the whole chunk is interior
    const bool st_upper = rin && !xfull && gx < R;  // first chunk: x = 4..7
    const bool st_lower = rin && !xfull && gx >= R;  // last chunk: x = nx-8 .. nx-5
    const int soff = (ly + R) * P::SX + 8 + 8 * lx;
    const int aoff = ly * TX + 8 * lx;
    int64_t goff = static_cast<int64_t>(zb) * a.sz + static_cast<int64_t>(gy) * a.sy + gx;

    // Source: a CTA-uniform test first (tile and plane), then the owning thread.
    const bool src_tile = a.src_z >= zb && a.src_z < ze && a.src_y >= y0 && a.src_y < y0 + TY &&
                          a.src_x >= xa && a.src_x < xa + TX;
    const bool src_mine = src_tile && a.src_x >= gx && a.src_x < gx + 8 && a.src_y == gy;
    const int src_e = a.src_x - gx;
    const int src_i = a.src_z - zb;

    float2 ax2[R], ay2[R], az2[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        ax2[r] = dup2(a.w.ax[r]);
        ay2[r] = dup2(a.w.ay[r]);
        az2[r] = dup2(a.w.az[r]);
    }
    const float2 cxy2 = dup2(a.w.cx + a.w.cy + a.w.cz);  // combined centre weight
    float m_out = 1.f, m_q = 1.f;
    if (PHASE == 1) m_out = a.scale->r;
    if (PHASE == 2) m_q = a.scale->r;
    const float2 nmq2 = dup2(-m_q), mout2 = dup2(m_out);

    // Plane index p (z = zb - 4 + p) lives in slot p % 4 of both rings.
    uint4 hq[4];      // FP16: centre and the planes above it
    float2 dq[4][4];  // FP32: the four planes below the centre, as point pairs
    bool bad = false;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        if (!wait_plane(p)) bad = true;
        const uint4 v = lds128h(sm + ((pb + p) % S) * P::PLANE + soff);
        if (p < R) {
#pragma unroll
            for (int h = 0; h < 4; ++h) dq[p][h] = h2f2(get_word(v, h));
        } else {
            hq[p - R] = v;
        }
    }
    bool abort_run = __syncthreads_or(bad) != 0;
    if (!abort_run && tid == 0) {
#pragma unroll
        for (int p = 0; p < R; ++p)  // planes 0..3 are consumed: refill their stages
            if (p + S < nplanes) issue_plane(p + S);
    }

    // The plane loop is unrolled by UNR (4 or 8).  i0 is a multiple of 4 and so
    // is S: the fed plane's stage is a block base + u, wrapping at most once
    // (UNR = 8), and its phase is a block constant or flips with the wrap; the aux
    // ring (AUX | 4) has compile-time stages and a block-constant phase.
    static_assert(UNR == 4 || UNR == 8, "unroll");
    static_assert(UNR == 4 || S == 8, "an unroll of 8 needs an 8-stage ring");
    for (int i0 = 0; i0 < nint && !abort_run; i0 += UNR) {
        // (CARRY: the same block bases offset by the carried sequence numbers)
        const int cbase = (pb + i0 + 4) % S, fbase = (pb + i0 + 8) % S;
        const uint32_t fpar = ((pb + i0 + 8) / S) & 1u, apar = (i0 / AUX) & 1u;
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int i = i0 + u;
            if (i < nint && !abort_run) {
                // Centre plane i + 4 (slot u); it was waited for when it was fed.
                const int cst = (cbase + u) % S, fst = (fbase + u) % S;
                const uint32_t fph = fpar ^ (fbase + u >= S ? 1u : 0u);
                const uint16_t* pc = sm + cst * P::PLANE + soff;
                // x window: 4 halves left and right of the chunk stay FP16; the
                // own 8 points (the centre) are converted once.
                const uint2 lf = lds64(pc - 4);
                const uint2 rt = lds64(pc + 8);
                // feed: plane i + 8 (z + 4) replaces the centre in slot u; the z pair
                // of radius 4 is formed at once, so plane z - 4 (FP32 slot u) is dead
                // before the centre is converted into that slot -- the two never
                // hold registers at the same time and the slots need no copies.
                const uint4 c16 = hq[u % 4];
                if (!mbar_wait(&full[fst], fph)) bad = true;
                hq[u % 4] = lds128h(sm + fst * P::PLANE + soff);
                float2 z4[4];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    z4[h] = addhf2(get_word(hq[u % 4], h), dq[u % 4][h]);
                    dq[u % 4][h] = h2f2(get_word(c16, h));
                }
                const float2(&cv)[4] = dq[u % 4];  // the centre, FP32
                const float cf[8] = {cv[0].x, cv[0].y, cv[1].x, cv[1].y,
                                     cv[2].x, cv[2].y, cv[3].x, cv[3].y};
                uint4 yu[R], yd[R];  // staged rows y +- d of the centre plane
#pragma unroll
                for (int d = 1; d <= R; ++d) {
                    yu[d - 1] = lds128h(pc + d * P::SX);
                    yd[d - 1] = lds128h(pc - d * P::SX);
                }
                // lap = c (cx+cy+cz) + sum_r (ax_r sx_r [+ ay_r sy_r] + az_r sz_r) in one
                // chain (+ sy5040 / 5040 with exact y), pair sums s = p[+r] + p[-r];
                // up operands of y and z enter FP16.
                // z pair of radius r: up plane (slot (u + r) % 4) + down plane
                auto zpair = [&](int r, int h) {
                    return r == R ? z4[h]
                                  : addhf2(get_word(hq[(u + r) % 4], h), dq[(u + 4 - r) % 4][h]);
                };
                float2 lap[4];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const float2 c = cv[h];
                    // one chain: centre, then per radius the x pair and the z pair
                    // (and the y pair without exact y); 5040 x the y pairs apart
                    float2 txy = mul2(cxy2, c);
                    float2 ty = make_float2(0.f, 0.f);  // kUpdExactY: 5040 x the y pairs
#pragma unroll
                    for (int r = 1; r <= R; ++r) {
                        // an aligned pair of own points (even r) adds as one pair
                        const bool own2 = r % 2 == 0 && 2 * h - r >= 0 && 2 * h + 1 + r <= 7;
                        const float2 sx = own2 ? add2(cv[h + r / 2], cv[h - r / 2])
                                               : make_float2(xsum1(cf, lf, rt, 2 * h, r),
                                                             xsum1(cf, lf, rt, 2 * h + 1, r));
                        txy = fma2(ax2[r - 1], sx, txy);
                        if (UPD & kUpdExactY) {
                            const uint16_t wy = y_weight5040(r);
                            ty.x = fmahf(get_word(yu[r - 1], h), 0, wy, ty.x);
                            ty.y = fmahf(get_word(yu[r - 1], h), 1, wy, ty.y);
                            ty.x = fmahf(get_word(yd[r - 1], h), 0, wy, ty.x);
                            ty.y = fmahf(get_word(yd[r - 1], h), 1, wy, ty.y);
                        } else {
                            txy = fma2(ay2[r - 1],
                                       addhf2(get_word(yu[r - 1], h), h2f2(get_word(yd[r - 1], h))),
                                       txy);
                        }
                        // up: plane z + r (FP16, slot (u + r) % 4; r = 4 is the plane
                        // just fed); down: plane z - r (FP32, slot (u + 4 - r) % 4)
                        txy = fma2(az2[r - 1], zpair(r, h), txy);
                    }
                    if (UPD & kUpdExactY) txy = fma2(dup2(kInv5040), ty, txy);
                    lap[h] = txy;
                }

                bool aok;
                const uint16_t* st;
                if (CARRY) {
                    aok = wait_aux(i);
                    st = aux + ((ab + i) % AUX) * 2 * P::TILE + aoff;
                } else {  // compile-time stage, block-constant phase
                    aok = mbar_wait(&auxf[u % AUX], apar ^ ((u / AUX) & 1u));
                    st = aux + (u % AUX) * 2 * P::TILE + aoff;
                }
                if (!aok) bad = true;
                const uint4 qv = lds128h(st);
                const uint4 kv = lds128h(st + P::TILE);
                constexpr bool kMixed = (UPD & kUpdMixedSub) && PHASE != 2;
                float o[8];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    const float2 c = cv[h];
                    const uint32_t kw = get_word(kv, h);
                    const float2 kk = make_float2(__uint_as_float(kw << 16),
                                                  __uint_as_float(kw & 0xffff0000u));
                    float2 ov;
                    if (kMixed) {
                        ov = rsubhf2(get_word(qv, h), fma2(kk, lap[h], add2(c, c)));
                        if (PHASE == 1) ov = mul2(ov, mout2);
                    } else {
                        // 2c - m_q pq in one rounding (2c is exact), then + K lap
                        const float2 pq = h2f2(get_word(qv, h));
                        ov = fma2(kk, lap[h], fma2(nmq2, pq, add2(c, c)));
                        if (PHASE == 1) ov = mul2(ov, mout2);
                    }
                    o[2 * h] = ov.x;
                    o[2 * h + 1] = ov.y;
                }
                if (src_tile && i == src_i) {  // CTA-uniform
                    if (src_mine) {
                        const float wv = a.src_wavelet ? a.src_wavelet[*a.src_step + a.src_off]
                                                       : a.src_w;
                        const float kk = bf2f(get_word(kv, src_e >> 1), src_e & 1);
                        const float sa = a.scale->a;
                        const float add = ((kk * a.dx2) * wv) * sa;
#pragma unroll
                        for (int e = 0; e < 8; ++e)
                            if (e == src_e) {
                                o[e] += add;
                                if (a.trace)
                                    a.trace[(a.src_step ? *a.src_step : 0) + a.src_off] =
                                        __half2float(__float2half_rn(o[e])) / sa;
                            }
                    }
                }
                {
                    uint16_t* dst = a.next + goff;  // used only under the predicates
                    uint4 pk;
                    pk.x = pack_h2(o[0], o[1]);
                    pk.y = pack_h2(o[2], o[3]);
                    pk.z = pack_h2(o[4], o[5]);
                    pk.w = pack_h2(o[6], o[7]);
                    stg_stream_u4_if(dst, pk, st_full);
                    // x = 4..7 of the first chunk; x = nx-8 .. nx-5 of the last
                    stg_stream_u2_if(dst + 4, make_uint2(pk.z, pk.w), st_upper);
                    stg_stream_u2_if(dst, make_uint2(pk.x, pk.y), st_lower);
                }
                goff += a.sz;
                abort_run = __syncthreads_or(bad) != 0;
                if (!abort_run && tid == 0) {
                    if (i + 4 + S < nplanes) issue_plane(i + 4 + S);  // the centre's stage
                    if (i + AUX < nint) issue_aux(i + AUX);
                }
            }
        }
    }

    if (abort_run) {
        if (tid == 0) {
            record_error(a.err, kDevWaitTimeout);
            for (int jj = max(0, issued_hi - S + 1); jj <= issued_hi; ++jj) (void)wait_plane(jj);
            for (int it = max(0, aux_issued_hi - AUX + 1); it <= aux_issued_hi; ++it)
                (void)wait_aux(it);
        }
        return false;
    }
    if (CARRY) {
        ring.p = pb + nplanes;
        ring.aux = ab + nint;
    }
    return true;
}

// Initialises the CTA's ring barriers (thread 0); the caller synchronises.
template <int S, int AUX>
__device__ __forceinline__ void init_rings_f16(uint64_t* full, uint64_t* auxf) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
#pragma unroll
    for (int s = 0; s < AUX; ++s) mbar_init(&auxf[s], 1);
    fence_barrier_init();
}

// One grid: CTA b owns tile (b % tiles_x, (b / tiles_x) % tiles_y) and z chunk
// b / (tiles_x * tiles_y).
template <int TX, int TY, int S, int AUX, int PHASE, int UNR, int UPD>
__global__ void __launch_bounds__(ShapeH<TX, TY, S, AUX>::NT, ShapeH<TX, TY, S, AUX>::MINB)
    pencil_f16_kernel(const __grid_constant__ CUtensorMap pmap,
                      const __grid_constant__ CUtensorMap qmap,
                      const __grid_constant__ CUtensorMap kmap, const F16Args a) {
    extern __shared__ unsigned char dsmem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t auxf[AUX];
    uint16_t* sm = reinterpret_cast<uint16_t*>(smem_align<128>(dsmem));
    if (threadIdx.x == 0) init_rings_f16<S, AUX>(full, auxf);
    __syncthreads();
    int b = blockIdx.x;
    const int tx = b % a.tiles_x;
    b /= a.tiles_x;
    const int ty = b % a.tiles_y;
    b /= a.tiles_y;
    RingH ring;
    (void)pencil_f16_tile<TX, TY, S, AUX, PHASE, UNR, false, UPD>(&pmap, &qmap, &kmap, a, tx, ty,
                                                                  b, sm, full, auxf, ring);
}

// Many grids (shots) in one persistent launch, as batch_f32_kernel: CTAs take
// (shot, tile x, tile y, z chunk) items from the queue; the rings' barriers are
// initialised once and their phases carried from item to item (RingH); the last
// CTA to finish resets the queue and advances the step counter the sources read.
template <int TX, int TY, int S, int AUX, int PHASE, int UNR, int UPD>
__global__ void __launch_bounds__(ShapeH<TX, TY, S, AUX>::NT, ShapeH<TX, TY, S, AUX>::MINB)
    batch_f16_kernel(const ShotF16* __restrict__ shots, const int4* __restrict__ items,
                     int n_items, BatchQueue* queue) {
    extern __shared__ unsigned char dsmem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t auxf[AUX];
    __shared__ int s_item;
    uint16_t* sm = reinterpret_cast<uint16_t*>(smem_align<128>(dsmem));
    if (threadIdx.x == 0) init_rings_f16<S, AUX>(full, auxf);
    RingH ring;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(&queue->next, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();  // every thread has read s_item before it is replaced
        if (it >= n_items) break;
        const int4 w = items[it];
        const ShotF16* sh = shots + w.x;
        const F16Args a = sh->args;
        if (!pencil_f16_tile<TX, TY, S, AUX, PHASE, UNR, true, UPD>(&sh->p, &sh->prev, &sh->k, a,
                                                                    w.y, w.z, w.w, sm, full, auxf,
                                                                    ring))
            break;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&queue->done, 1) == static_cast<int>(gridDim.x) - 1) {
            queue->next = 0;
            queue->done = 0;
            queue->step += 1;
            __threadfence();
        }
    }
}


using LaunchFnH = cudaError_t (*)(const PencilMaps&, const F16Args&, unsigned, int, bool,
                                   cudaStream_t);
using ResidentFnH = int (*)();

// The two update forms every tile is compiled in: kUpdMixedSub, and with
// kUpdExactY on grids with dx == dy (the form follows the grid, not the tile, so
// every tile gives the same bits on a grid).
constexpr int kFormPlain = kUpdMixedSub, kFormExactY = kUpdMixedSub | kUpdExactY;

template <int TX, int TY, int S, int AUX, int UNR, int UPD>
bool set_f16_smem(int smem) {
    return cudaFuncSetAttribute(pencil_f16_kernel<TX, TY, S, AUX, 0, UNR, UPD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
           cudaFuncSetAttribute(pencil_f16_kernel<TX, TY, S, AUX, 1, UNR, UPD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
           cudaFuncSetAttribute(pencil_f16_kernel<TX, TY, S, AUX, 2, UNR, UPD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess;
}

template <int TX, int TY, int S, int AUX, int UNR>
int resident_f16() {
    using P = ShapeH<TX, TY, S, AUX>;
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63] > 0) return cached[dev & 63];
    const int smem = static_cast<int>(P::SMEM);
    int n = 0, n2 = 0;
    if (set_f16_smem<TX, TY, S, AUX, UNR, kFormPlain>(smem) &&
        set_f16_smem<TX, TY, S, AUX, UNR, kFormExactY>(smem) &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, pencil_f16_kernel<TX, TY, S, AUX, 0, UNR, kFormPlain>, P::NT, P::SMEM) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n2, pencil_f16_kernel<TX, TY, S, AUX, 0, UNR, kFormExactY>, P::NT, P::SMEM) ==
            cudaSuccess &&
        std::min(n, n2) > 0) {
        cached[dev & 63] = std::min(n, n2);
        return cached[dev & 63];
    }
    cudaGetLastError();
    return std::max(1, std::min(int((228u * 1024u) / (P::SMEM + 1024u)), 65536 / (P::NT * 128)));
}

template <int TX, int TY, int S, int AUX, int UNR, int UPD>
void launch_f16_form(const PencilMaps& m, const F16Args& a, unsigned ctas, int phase,
                     cudaStream_t stream) {
    using P = ShapeH<TX, TY, S, AUX>;
    if (phase == 1)
        pencil_f16_kernel<TX, TY, S, AUX, 1, UNR, UPD><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                     m.vel2, a);
    else if (phase == 2)
        pencil_f16_kernel<TX, TY, S, AUX, 2, UNR, UPD><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                     m.vel2, a);
    else
        pencil_f16_kernel<TX, TY, S, AUX, 0, UNR, UPD><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                     m.vel2, a);
}

template <int TX, int TY, int S, int AUX, int UNR>
cudaError_t launch_f16(const PencilMaps& m, const F16Args& a, unsigned ctas, int phase,
                       bool exact_y, cudaStream_t stream) {
    resident_f16<TX, TY, S, AUX, UNR>();  // sets the attributes once per device
    if (exact_y)
        launch_f16_form<TX, TY, S, AUX, UNR, kFormExactY>(m, a, ctas, phase, stream);
    else
        launch_f16_form<TX, TY, S, AUX, UNR, kFormPlain>(m, a, ctas, phase, stream);
    return cudaGetLastError();
}

struct VariantH {
    int tx, ty, stages, aux;
    const char* name;
    LaunchFnH launch;
    ResidentFnH resident;
};

#define SB200_VARIANT_H(TX, TY, S, AUX, UNR, NAME)                                         \
    VariantH {                                                                               \
        TX, TY, S, AUX, NAME, &launch_f16<TX, TY, S, AUX, UNR>,                             \
            &resident_f16<TX, TY, S, AUX, UNR>                                               \
    }

// Tile shapes.  Measured at 1024^3 (median of 5 interleaved rounds, random
// fields, h64x16): the update with a separate p_prev conversion 1.86 ms, the
// mixed subtract 1.83-1.86, exact y alone 1.80-1.82, both 1.78-1.80; not kept:
// 64 x 8 tiles (2.08), 32 x 16 (2.12), the plane loop unrolled by 8 (1.82-2.14;
// again 1.92-1.99 against 1.54-1.71 in one interleaved run), the planes above the
// centre converted to FP32 when fed so that each z pair is one FP32 pair add
// (2.39-2.48: 128 registers and spills; unrolled by 8, no spills, 1.98-2.21).
const VariantH kF16[] = {
    SB200_VARIANT_H(64, 16, 8, 4, 4, "h64x16_s8_a4"),
    SB200_VARIANT_H(64, 32, 8, 4, 4, "h64x32_s8_a4"),
    SB200_VARIANT_H(128, 16, 8, 4, 4, "h128x16_s8_a4"),
};
constexpr int kNumF16 = sizeof(kF16) / sizeof(kF16[0]);

}  // namespace

int pencil_f16_variant_count() { return kNumF16; }
const char* pencil_f16_variant_name(int v) {
    return (v >= 0 && v < kNumF16) ? kF16[v].name : nullptr;
}
PencilBoxes pencil_f16_boxes(int v) {
    PencilBoxes b;
    b.halo_x = kF16[v].tx + 16;
    b.halo_y = kF16[v].ty + 2 * R;
    b.tile_x = kF16[v].tx;
    b.tile_y = kF16[v].ty;
    b.aux_tma = true;
    return b;
}
int pencil_f16_resident(int v) { return kF16[v].resident(); }
void pencil_f16_prepare() {
    for (int v = 0; v < kNumF16; ++v) kF16[v].resident();
}
int64_t pencil_f16_ctas(int v, const GridDesc& g, int zchunks) {
    const int tiles_x = static_cast<int>((g.nx - R + kF16[v].tx - 1) / kF16[v].tx);
    const int tiles_y = static_cast<int>((g.ny - 2 * R + kF16[v].ty - 1) / kF16[v].ty);
    const int inz = static_cast<int>(g.nz - 2 * R);
    const int zc = std::max(1, std::min(zchunks, inz));
    const int zlen = (inz + zc - 1) / zc;
    return int64_t(tiles_x) * tiles_y * ((inz + zlen - 1) / zlen);
}

// Whether the exact-y form applies: dx == dy (the 5040-scaled y weights of
// c_r (dx/dy)^2 are exact halves only then).
bool f16_exact_y(const GridDesc& g) { return g.dx == g.dy; }

namespace {

// Sweep arguments of a TX x TY tile shape over grid g split into zchunks z
// chunks: tile counts, weights relative to K, source, scale.
F16Args make_f16_args(int TX, int TY, const GridDesc& g, int zchunks, uint16_t* next,
                      const SourceDesc& src, const F16Scale* scale, int* err) {
    F16Args a{};
    a.next = next;
    a.nx = static_cast<int>(g.nx);
    a.ny = static_cast<int>(g.ny);
    a.nz = static_cast<int>(g.nz);
    a.sy = g.nx;
    a.sz = g.nx * g.ny;
    // x tiles start at 0 and cover every x below nx - 4.
    a.tiles_x = static_cast<int>((g.nx - R + TX - 1) / TX);
    a.tiles_y = static_cast<int>((g.ny - 2 * R + TY - 1) / TY);
    const int inz = static_cast<int>(g.nz - 2 * R);
    const int zc = std::max(1, std::min(zchunks, inz));
    a.zlen = (inz + zc - 1) / zc;
    const double ry = double(g.dx) * g.dx / (double(g.dy) * g.dy);
    const double rz = double(g.dx) * g.dx / (double(g.dz) * g.dz);
    const double c[R + 1] = {C0, C1, C2, C3, C4};
    a.w.cx = static_cast<float>(c[0]);
    a.w.cy = static_cast<float>(c[0] * ry);
    a.w.cz = static_cast<float>(c[0] * rz);
    for (int r = 0; r < R; ++r) {
        a.w.ax[r] = static_cast<float>(c[r + 1]);
        a.w.ay[r] = static_cast<float>(c[r + 1] * ry);
        a.w.az[r] = static_cast<float>(c[r + 1] * rz);
    }
    a.dx2 = g.dx * g.dx;
    a.src_x = a.src_y = a.src_z = -1;
    if (src.idx >= 0) {
        a.src_x = static_cast<int>(src.idx % g.nx);
        a.src_y = static_cast<int>((src.idx / g.nx) % g.ny);
        a.src_z = static_cast<int>(src.idx / (g.nx * g.ny));
        a.src_w = src.w;
        a.src_wavelet = src.wavelet;
        a.src_step = src.step;
        a.src_off = src.step_offset;
        a.trace = src.trace;
    }
    a.scale = scale;
    a.err = err;
    return a;
}

// ── batched FP16 shots ────────────────────────────────────────────────────────

using LaunchFnB16 = cudaError_t (*)(const ShotF16*, const int4*, int, BatchQueue*, unsigned, int,
                                    bool, cudaStream_t);

template <int TX, int TY, int S, int AUX, int UNR, int UPD>
bool set_batch_f16_smem(int smem) {
    return cudaFuncSetAttribute(batch_f16_kernel<TX, TY, S, AUX, 0, UNR, UPD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
           cudaFuncSetAttribute(batch_f16_kernel<TX, TY, S, AUX, 1, UNR, UPD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
           cudaFuncSetAttribute(batch_f16_kernel<TX, TY, S, AUX, 2, UNR, UPD>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess;
}

template <int TX, int TY, int S, int AUX, int UNR>
int resident_batch_f16() {
    using P = ShapeH<TX, TY, S, AUX>;
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63] > 0) return cached[dev & 63];
    const int smem = static_cast<int>(P::SMEM);
    int n = 0, n2 = 0;
    if (set_batch_f16_smem<TX, TY, S, AUX, UNR, kFormPlain>(smem) &&
        set_batch_f16_smem<TX, TY, S, AUX, UNR, kFormExactY>(smem) &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, batch_f16_kernel<TX, TY, S, AUX, 0, UNR, kFormPlain>, P::NT, P::SMEM) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n2, batch_f16_kernel<TX, TY, S, AUX, 0, UNR, kFormExactY>, P::NT, P::SMEM) ==
            cudaSuccess &&
        std::min(n, n2) > 0) {
        cached[dev & 63] = std::min(n, n2);
        return cached[dev & 63];
    }
    cudaGetLastError();
    return std::max(1, std::min(int((228u * 1024u) / (P::SMEM + 1024u)), 65536 / (P::NT * 128)));
}

template <int TX, int TY, int S, int AUX, int UNR, int UPD>
void launch_batch_f16_form(const ShotF16* shots, const int4* items, int n_items,
                           BatchQueue* queue, unsigned ctas, int phase, cudaStream_t stream) {
    using P = ShapeH<TX, TY, S, AUX>;
    if (phase == 1)
        batch_f16_kernel<TX, TY, S, AUX, 1, UNR, UPD><<<ctas, P::NT, P::SMEM, stream>>>(shots, items,
                                                                                    n_items, queue);
    else if (phase == 2)
        batch_f16_kernel<TX, TY, S, AUX, 2, UNR, UPD><<<ctas, P::NT, P::SMEM, stream>>>(shots, items,
                                                                                    n_items, queue);
    else
        batch_f16_kernel<TX, TY, S, AUX, 0, UNR, UPD><<<ctas, P::NT, P::SMEM, stream>>>(shots, items,
                                                                                    n_items, queue);
}

template <int TX, int TY, int S, int AUX, int UNR>
cudaError_t launch_batch_f16_t(const ShotF16* shots, const int4* items, int n_items,
                               BatchQueue* queue, unsigned ctas, int phase, bool exact_y,
                               cudaStream_t stream) {
    resident_batch_f16<TX, TY, S, AUX, UNR>();  // sets the attributes once per device
    if (exact_y)
        launch_batch_f16_form<TX, TY, S, AUX, UNR, kFormExactY>(shots, items, n_items, queue, ctas,
                                                              phase, stream);
    else
        launch_batch_f16_form<TX, TY, S, AUX, UNR, kFormPlain>(shots, items, n_items, queue, ctas,
                                                             phase, stream);
    return cudaGetLastError();
}

struct VariantB16 {
    int tx, ty;
    const char* name;
    LaunchFnB16 launch;
    ResidentFnH resident;
};

const VariantB16 kBatchF16[] = {
    {64, 16, "bh64x16_s8_a4", &launch_batch_f16_t<64, 16, 8, 4, 4>,
     &resident_batch_f16<64, 16, 8, 4, 4>},
    {32, 16, "bh32x16_s8_a4", &launch_batch_f16_t<32, 16, 8, 4, 4>,
     &resident_batch_f16<32, 16, 8, 4, 4>},
    {64, 8, "bh64x8_s8_a4", &launch_batch_f16_t<64, 8, 8, 4, 4>,
     &resident_batch_f16<64, 8, 8, 4, 4>},
};
constexpr int kNumBatchF16 = sizeof(kBatchF16) / sizeof(kBatchF16[0]);

}  // namespace

cudaError_t launch_wave_pencil_f16(const PencilMaps& maps, uint16_t* next, const GridDesc& g,
                                   const SourceDesc& src, const F16Scale* scale, int phase,
                                   const PencilConfig& cfg, int* err, cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const VariantH& v = kF16[cfg.variant];
    const F16Args a = make_f16_args(v.tx, v.ty, g, cfg.zchunks, next, src, scale, err);
    const int inz = static_cast<int>(g.nz - 2 * R);
    const unsigned ctas = static_cast<unsigned>(int64_t(a.tiles_x) * a.tiles_y *
                                                ((inz + a.zlen - 1) / a.zlen));
    return v.launch(maps, a, ctas, phase, f16_exact_y(g), stream);
}

int batch_f16_variant_count() { return kNumBatchF16; }
const char* batch_f16_variant_name(int v) {
    return (v >= 0 && v < kNumBatchF16) ? kBatchF16[v].name : nullptr;
}
PencilBoxes batch_f16_boxes(int v) {
    PencilBoxes b;
    b.halo_x = kBatchF16[v].tx + 16;
    b.halo_y = kBatchF16[v].ty + 2 * R;
    b.tile_x = kBatchF16[v].tx;
    b.tile_y = kBatchF16[v].ty;
    b.aux_tma = true;
    return b;
}
int batch_f16_resident(int v) { return kBatchF16[v].resident(); }
void batch_f16_prepare() {
    for (int v = 0; v < kNumBatchF16; ++v) kBatchF16[v].resident();
}
F16Args batch_f16_shot_args(int v, const GridDesc& g, int zchunks, uint16_t* next,
                            const SourceDesc& src, const F16Scale* scale, int* err) {
    return make_f16_args(kBatchF16[v].tx, kBatchF16[v].ty, g, zchunks, next, src, scale, err);
}
cudaError_t launch_batch_f16(int v, const ShotF16* shots, const int4* items, int n_items,
                             BatchQueue* queue, unsigned ctas, int phase, bool exact_y,
                             cudaStream_t stream) {
    return kBatchF16[v].launch(shots, items, n_items, queue, ctas, phase, exact_y, stream);
}

}  // namespace sb200
