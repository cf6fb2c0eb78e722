// FP16-storage acoustic pencil kernel for sm_100a.
//
// Storage: p and p_prev in FP16, both holding a * p for one power-of-two scale
// a (kept in a device-side F16Scale); K = vel2 * dt^2 / dx^2 in BF16.  All
// arithmetic is FP32: every stored value is converted once at its use, the
// z / x pair sums use the sm_100 mixed-precision add (f16 + f32 -> f32), and
// the output is rounded to FP16 once.  DRAM traffic: 8 B per interior point
// (read p, p_prev, K; write p_next in place over p_prev).
//
// Layout of a CTA's work is the FP32 kernel's (pencil_f32.cu) with 2-byte
// elements: each thread owns 8 consecutive x (one 16-byte chunk) in RPT rows.
// Because the interior starts at x = 4 (byte 8), tiles are aligned to x = 8k
// and the p box starts 8 halves left of the tile (16-byte aligned TMA origin,
// box TX + 16 wide); points of a chunk outside the interior are never stored.
//
// Renormalisation (driven by the FP64 statistics every few dozen steps): a
// renorm step (PHASE 1) scales its output by r = a_new / a_old; the step after
// it (PHASE 2) scales p_prev, still at a_old, by r; other steps (PHASE 0) carry
// no scale arithmetic.  Powers of two make every rescale exact.
#include <cuda_fp16.h>

#include <algorithm>
#include <mutex>

#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {

struct F16Args {
    uint16_t* next;  // p_next (aliases the p_prev buffer read through qmap)
    int nx, ny, nz;
    int64_t sy, sz;
    int tiles_x, tiles_y, zlen;
    Weights w;   // Laplacian weights relative to K: ax = c_r, ay = c_r (dx/dy)^2, ...
    float dx2;   // dx^2: the source term dt^2 vel2 w = K dx^2 w
    int src_x, src_y, src_z;
    float src_w;
    const float* src_wavelet;
    const int* src_step;
    int src_off;
    float* trace;
    const F16Scale* scale;
    int* err;
};

template <int TX, int TY, int RPT, int S, int AUX>
struct ShapeH {
    static_assert(TX % 8 == 0, "TX must be a multiple of 8 halves (16-byte chunks)");
    static_assert(TY % RPT == 0, "TY must be a multiple of RPT");
    static_assert(S >= 8 && AUX >= 1, "rings");
    static constexpr int SX = TX + 16;  // halves per staged row: 8 left, TX, 8 right
    static constexpr int SY = TY + 2 * R;
    static_assert(SX <= 256 && SY <= 256, "TMA box extent is at most 256");
    static constexpr int TPR = TX / 8;
    static constexpr int NT = TPR * (TY / RPT);
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

// UNR = 9: the plane loop is unrolled by 9 so the z queue's slots are
// compile-time registers that never move.  UNR = 1: one plane per iteration and
// the queue shifts by one slot after each plane (36 register moves per row of
// a thread) -- a ninth of the code, for kernels that stall on instruction fetch.
template <int TX, int TY, int RPT, int S, int AUX, int PHASE, int UNR>
__global__ void __launch_bounds__(ShapeH<TX, TY, RPT, S, AUX>::NT, ShapeH<TX, TY, RPT, S, AUX>::MINB)
    pencil_f16_kernel(const __grid_constant__ CUtensorMap pmap,
                      const __grid_constant__ CUtensorMap qmap,
                      const __grid_constant__ CUtensorMap kmap, const F16Args a) {
    using P = ShapeH<TX, TY, RPT, S, AUX>;
    extern __shared__ unsigned char dsmem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t auxf[AUX];
    uint16_t* sm = reinterpret_cast<uint16_t*>((reinterpret_cast<uintptr_t>(dsmem) + 127) &
                                               ~uintptr_t(127));
    uint16_t* aux = sm + S * P::PLANE;  // AUX stages of [p_prev tile | K tile]

    const int tid = threadIdx.x;
    const int lx = tid % P::TPR;
    const int ly = tid / P::TPR;
    int b = blockIdx.x;
    const int tx = b % a.tiles_x;
    b /= a.tiles_x;
    const int ty = b % a.tiles_y;
    b /= a.tiles_y;
    const int xa = tx * TX;      // first x of the tile (multiple of 8)
    const int y0 = R + ty * TY;  // first interior row of the tile
    const int zb = R + b * a.zlen;
    const int ze = min(zb + a.zlen, a.nz - R);
    const int nint = ze - zb;
    const int nplanes = nint + 2 * R;

    if (tid == 0) {
        prefetch_tmap(&pmap);
        prefetch_tmap(&qmap);
        prefetch_tmap(&kmap);
#pragma unroll
        for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
#pragma unroll
        for (int s = 0; s < AUX; ++s) mbar_init(&auxf[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int issued_hi = -1, aux_issued_hi = -1;
    auto issue_aux = [&](int it) {
        uint16_t* st = aux + (it % AUX) * 2 * P::TILE;
        mbar_arrive_expect_tx(&auxf[it % AUX], 2 * P::TILE_BYTES);
        tma_load_3d(st, &qmap, &auxf[it % AUX], xa, y0, zb + it);
        tma_load_3d(st + P::TILE, &kmap, &auxf[it % AUX], xa, y0, zb + it);
        aux_issued_hi = it;
    };
    if (tid == 0) {
        for (int s = 0; s < S && s < nplanes; ++s) {
            mbar_arrive_expect_tx(&full[s], P::PLANE_BYTES);
            tma_load_3d(sm + s * P::PLANE, &pmap, &full[s], xa - 8, y0 - R, zb - R + s);
            issued_hi = s;
        }
        for (int it = 0; it < AUX && it < nint; ++it) issue_aux(it);
    }

    const int gx = xa + 8 * lx;  // first x of this thread's chunk
    const int gy = y0 + RPT * ly;
    // Interior x range of the chunk: [max(gx, 4), min(gx + 8, nx - 4)).
    const int xlo = max(gx, R), xhi = min(gx + 8, a.nx - R);
    const bool xany = xlo < xhi, xfull = gx >= R && gx + 8 <= a.nx - R;
    bool rin[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) rin[j] = xany && (gy + j < a.ny - R);
    const int soff = (RPT * ly + R) * P::SX + 8 + 8 * lx;
    const int aoff = RPT * ly * TX + 8 * lx;
    int64_t goff = static_cast<int64_t>(zb) * a.sz + static_cast<int64_t>(gy) * a.sy + gx;

    int src_j = -1, src_e = -1;
    if (a.src_z >= 0 && a.src_x >= gx && a.src_x < gx + 8 && a.src_y >= gy &&
        a.src_y < gy + RPT) {
        src_j = a.src_y - gy;
        src_e = a.src_x - gx;
    }

    float ax[R], ay[R], az[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        ax[r] = a.w.ax[r];
        ay[r] = a.w.ay[r];
        az[r] = a.w.az[r];
    }
    float m_out = 1.f, m_q = 1.f;
    if (PHASE == 1) m_out = a.scale->r;
    if (PHASE == 2) m_q = a.scale->r;
    float2 ax2[R], ay2[R], az2[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        ax2[r] = make_float2(ax[r], ax[r]);
        ay2[r] = make_float2(ay[r], ay[r]);
        az2[r] = make_float2(az[r], az[r]);
    }
    const float2 cx2 = make_float2(a.w.cx, a.w.cx), cy2 = make_float2(a.w.cy, a.w.cy),
                 cz2 = make_float2(a.w.cz, a.w.cz);
    const float2 nmq2 = make_float2(-m_q, -m_q), mout2 = make_float2(m_out, m_out);

    uint4 q[9][RPT];
    bool bad = false;
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
        if (!mbar_wait(&full[jj % S], (jj / S) & 1)) bad = true;
        const uint16_t* pl = sm + (jj % S) * P::PLANE + soff;
#pragma unroll
        for (int j = 0; j < RPT; ++j) q[jj][j] = lds128h(pl + j * P::SX);
    }
    bool abort_run = __syncthreads_or(bad) != 0;
    if (!abort_run && tid == 0) {
#pragma unroll
        for (int jj = 0; jj < R; ++jj) {
            const int jn = jj + S;
            if (jn < nplanes) {
                mbar_arrive_expect_tx(&full[jj], P::PLANE_BYTES);
                tma_load_3d(sm + jj * P::PLANE, &pmap, &full[jj], xa - 8, y0 - R, zb - R + jn);
                issued_hi = jn;
            }
        }
    }

    static_assert(UNR == 1 || UNR == 9, "the z queue is unrolled by 9 or rolled");
    for (int i0 = 0; i0 < nint && !abort_run; i0 += UNR) {
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const int i = i0 + u;
            if (i < nint && !abort_run) {
                const int cs = (u + 4) % 9;
                {
                    const int jf = i + 8;
                    if (!mbar_wait(&full[jf % S], (jf / S) & 1)) bad = true;
                    const uint16_t* pf = sm + (jf % S) * P::PLANE + soff;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) q[(u + 8) % 9][j] = lds128h(pf + j * P::SX);
                }
                const uint16_t* pc = sm + ((i + 4) % S) * P::PLANE + soff;

                // Pairs of points (halves 2h, 2h+1 of a 16-byte chunk) as packed
                // FP32.  y: row pairs j+d, j-d through the mixed FP16 + FP32 add;
                // farthest pair first, from zero.
                float2 ya[RPT][4];
#pragma unroll
                for (int j = 0; j < RPT; ++j)
#pragma unroll
                    for (int h = 0; h < 4; ++h) ya[j][h] = make_float2(0.f, 0.f);
#pragma unroll
                for (int d = R; d >= 1; --d) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        const int ku = j + d, kd = j - d;
                        const uint4 up = (ku < RPT) ? q[cs][ku] : lds128h(pc + ku * P::SX);
                        const uint4 dn = (kd >= 0) ? q[cs][kd] : lds128h(pc + kd * P::SX);
#pragma unroll
                        for (int h = 0; h < 4; ++h)
                            ya[j][h] = fma2(ay2[d - 1], addhf2(get_word(up, h), h2f2(get_word(dn, h))),
                                            ya[j][h]);
                    }
                }
                // x window halves: [4 left | 8 own | 4 right] per row; z from the queue.
                float2 lap[RPT][4];
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    const uint2 lf = lds64(pc + j * P::SX - 4);
                    const uint2 rt = lds64(pc + j * P::SX + 8);
                    const uint4 own = q[cs][j];
                    const uint32_t win[8] = {lf.x, lf.y, own.x, own.y, own.z, own.w, rt.x, rt.y};
                    float2 xv[8];  // the window's 16 halves as 8 pairs
#pragma unroll
                    for (int w = 0; w < 8; ++w) xv[w] = h2f2(win[w]);
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float2 c = xv[2 + h];
                        float2 tz = mul2(cz2, c);
                        float2 tx = mul2(cx2, c);
#pragma unroll
                        for (int r = 1; r <= R; ++r) {
                            const uint4& upv = q[(u + 4 + r) % 9][j];
                            const uint4& dnv = q[(u + 4 - r + 9) % 9][j];
                            tz = fma2(az2[r - 1], addhf2(get_word(upv, h), h2f2(get_word(dnv, h))), tz);
                            // window halves 4 + 2h +- r and 5 + 2h +- r
                            float2 s;
                            if (r % 2 == 0) {
                                s = add2(xv[2 + h + r / 2], xv[2 + h - r / 2]);
                            } else {
                                const int a0 = 4 + 2 * h + r, b0 = 4 + 2 * h - r;
                                const float ra = (a0 & 1) ? xv[a0 >> 1].y : xv[a0 >> 1].x;
                                const float rb = ((a0 + 1) & 1) ? xv[(a0 + 1) >> 1].y : xv[(a0 + 1) >> 1].x;
                                const float la = (b0 & 1) ? xv[b0 >> 1].y : xv[b0 >> 1].x;
                                const float lb = ((b0 + 1) & 1) ? xv[(b0 + 1) >> 1].y : xv[(b0 + 1) >> 1].x;
                                s = make_float2(ra + la, rb + lb);
                            }
                            tx = fma2(ax2[r - 1], s, tx);
                        }
                        const float2 ty = fma2(cy2, c, ya[j][h]);
                        lap[j][h] = add2(add2(tx, ty), tz);
                    }
                }
                if (!mbar_wait(&auxf[i % AUX], (i / AUX) & 1)) bad = true;
                const uint16_t* st = aux + (i % AUX) * 2 * P::TILE + aoff;
                const int z = zb + i;
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    const uint4 qv = lds128h(st + j * TX);
                    const uint4 kv = lds128h(st + P::TILE + j * TX);
                    const uint4 own = q[cs][j];
                    float o[8];
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const float2 c = h2f2(get_word(own, h));
                        const float2 pq = h2f2(get_word(qv, h));
                        const uint32_t kw = get_word(kv, h);
                        const float2 kk = make_float2(__uint_as_float(kw << 16),
                                                      __uint_as_float(kw & 0xffff0000u));
                        // 2c - m_q pq in one rounding (2c is exact), then + K lap
                        float2 ov = fma2(kk, lap[j][h], fma2(nmq2, pq, add2(c, c)));
                        if (PHASE == 1) ov = mul2(ov, mout2);
                        o[2 * h] = ov.x;
                        o[2 * h + 1] = ov.y;
                    }
                    if (src_j == j && z == a.src_z) {
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
                    if (rin[j]) {
                        uint16_t* dst = a.next + goff + j * a.sy;
                        if (xfull) {
                            uint4 pk;
                            pk.x = pack_h2(o[0], o[1]);
                            pk.y = pack_h2(o[2], o[3]);
                            pk.z = pack_h2(o[4], o[5]);
                            pk.w = pack_h2(o[6], o[7]);
                            stg_stream_u4(dst, pk);
                        } else {  // chunk straddles the halo: store interior points only
#pragma unroll
                            for (int e = 0; e < 8; ++e)
                                if (gx + e >= xlo && gx + e < xhi)
                                    dst[e] = __half_as_ushort(__float2half_rn(o[e]));
                        }
                    }
                }
                goff += a.sz;
                abort_run = __syncthreads_or(bad) != 0;
                if (!abort_run && tid == 0) {
                    const int jr = i + 4;
                    const int jn = jr + S;
                    if (jn < nplanes) {
                        mbar_arrive_expect_tx(&full[jr % S], P::PLANE_BYTES);
                        tma_load_3d(sm + (jr % S) * P::PLANE, &pmap, &full[jr % S], xa - 8,
                                    y0 - R, zb - R + jn);
                        issued_hi = jn;
                    }
                    if (i + AUX < nint) issue_aux(i + AUX);
                }
                if (UNR == 1) {  // slot k holds plane i + 1 + k for the next plane
#pragma unroll
                    for (int k = 0; k < 8; ++k)
#pragma unroll
                        for (int j = 0; j < RPT; ++j) q[k][j] = q[k + 1][j];
                }
            }
        }
    }

    if (abort_run && tid == 0) {
        record_error(a.err, kDevWaitTimeout);
        for (int jj = max(0, issued_hi - S + 1); jj <= issued_hi; ++jj)
            (void)mbar_wait(&full[jj % S], (jj / S) & 1);
        for (int it = max(0, aux_issued_hi - AUX + 1); it <= aux_issued_hi; ++it)
            (void)mbar_wait(&auxf[it % AUX], (it / AUX) & 1);
    }
}

using LaunchFnH = cudaError_t (*)(const PencilMaps&, const F16Args&, unsigned, int, cudaStream_t);
using ResidentFnH = int (*)();

template <int TX, int TY, int RPT, int S, int AUX, int UNR>
int resident_f16() {
    using P = ShapeH<TX, TY, RPT, S, AUX>;
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63] > 0) return cached[dev & 63];
    auto kern = pencil_f16_kernel<TX, TY, RPT, S, AUX, 0, UNR>;
    const int smem = static_cast<int>(P::SMEM);
    int n = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
            cudaSuccess &&
        cudaFuncSetAttribute(pencil_f16_kernel<TX, TY, RPT, S, AUX, 1, UNR>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
        cudaFuncSetAttribute(pencil_f16_kernel<TX, TY, RPT, S, AUX, 2, UNR>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, P::NT, P::SMEM) == cudaSuccess &&
        n > 0) {
        cached[dev & 63] = n;
        return n;
    }
    cudaGetLastError();
    return std::max(1, std::min(int((228u * 1024u) / (P::SMEM + 1024u)), 65536 / (P::NT * 128)));
}

template <int TX, int TY, int RPT, int S, int AUX, int UNR>
cudaError_t launch_f16(const PencilMaps& m, const F16Args& a, unsigned ctas, int phase,
                       cudaStream_t stream) {
    using P = ShapeH<TX, TY, RPT, S, AUX>;
    resident_f16<TX, TY, RPT, S, AUX, UNR>();  // sets the attributes once per device
    if (phase == 1)
        pencil_f16_kernel<TX, TY, RPT, S, AUX, 1, UNR><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                   m.vel2, a);
    else if (phase == 2)
        pencil_f16_kernel<TX, TY, RPT, S, AUX, 2, UNR><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                   m.vel2, a);
    else
        pencil_f16_kernel<TX, TY, RPT, S, AUX, 0, UNR><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                   m.vel2, a);
    return cudaGetLastError();
}

struct VariantH {
    int tx, ty, rpt, stages, aux;
    const char* name;
    LaunchFnH launch;
    ResidentFnH resident;
};

#define SB200_VARIANT_H(TX, TY, RPT, S, AUX, UNR, NAME)                                   \
    VariantH {                                                                              \
        TX, TY, RPT, S, AUX, NAME, &launch_f16<TX, TY, RPT, S, AUX, UNR>,                   \
            &resident_f16<TX, TY, RPT, S, AUX, UNR>                                          \
    }

// "_roll": the z queue shifts one slot per plane instead of the 9x unroll.
const VariantH kF16[] = {
    SB200_VARIANT_H(64, 16, 1, 8, 4, 9, "h64x16_r1_s8_a4"),
    SB200_VARIANT_H(64, 32, 2, 8, 3, 9, "h64x32_r2_s8_a3"),
    SB200_VARIANT_H(128, 16, 2, 8, 3, 9, "h128x16_r2_s8_a3"),
    SB200_VARIANT_H(64, 32, 1, 8, 3, 9, "h64x32_r1_s8_a3"),
    SB200_VARIANT_H(64, 16, 1, 8, 4, 1, "h64x16_r1_s8_a4_roll"),
    SB200_VARIANT_H(64, 32, 2, 8, 3, 1, "h64x32_r2_s8_a3_roll"),
    SB200_VARIANT_H(128, 16, 2, 8, 3, 1, "h128x16_r2_s8_a3_roll"),
    SB200_VARIANT_H(64, 32, 1, 8, 3, 1, "h64x32_r1_s8_a3_roll"),
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

cudaError_t launch_wave_pencil_f16(const PencilMaps& maps, uint16_t* next, const GridDesc& g,
                                   const SourceDesc& src, const F16Scale* scale, int phase,
                                   const PencilConfig& cfg, int* err, cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const VariantH& v = kF16[cfg.variant];
    F16Args a{};
    a.next = next;
    a.nx = static_cast<int>(g.nx);
    a.ny = static_cast<int>(g.ny);
    a.nz = static_cast<int>(g.nz);
    a.sy = g.nx;
    a.sz = g.nx * g.ny;
    // x tiles start at 0 and cover every x below nx - 4.
    a.tiles_x = static_cast<int>((g.nx - R + v.tx - 1) / v.tx);
    a.tiles_y = static_cast<int>((g.ny - 2 * R + v.ty - 1) / v.ty);
    const int inz = static_cast<int>(g.nz - 2 * R);
    const int zc = std::max(1, std::min(cfg.zchunks, inz));
    a.zlen = (inz + zc - 1) / zc;
    const unsigned ctas = static_cast<unsigned>(int64_t(a.tiles_x) * a.tiles_y *
                                                ((inz + a.zlen - 1) / a.zlen));
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
    return v.launch(maps, a, ctas, phase, stream);
}

}  // namespace sb200
