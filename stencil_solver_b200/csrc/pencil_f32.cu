// FP32 z-marching pencil kernels for sm_100a: acoustic leapfrog and explicit heat.
//
// Replaces the reference's kernel_tiled (src/kernels/stencil_tiled.cu:37-145) and
// kernel_naive (src/kernels/stencil_naive.cu:49-89) behind launch_tiled / launch_naive.
//
// Work unit: one CTA owns a TX x TY tile of interior columns and marches z over
// [zb, ze) (the whole interior unless the launch splits z into chunks).
//   * x-y planes of p (with the 4-cell halo: (TX+8) x (TY+8) floats) are fetched by
//     TMA into an S-stage shared-memory ring; each stage has an mbarrier that the
//     copy completes (expect_tx / complete_tx).  Thread 0 refills a stage as soon as
//     the CTA is past its last use, S-4 planes ahead of the first consumer.
//   * Acoustic: the TX x TY tiles of p_prev and vel2 for plane z come by TMA into a
//     second AUX-stage ring, AUX-1 planes ahead of their use (AUX = 0 instead loads
//     them with 128-bit global loads at the start of the plane).
//   * Each thread owns a float4 of x (4 points) in RPT consecutive rows.  Its z
//     neighbours (z-4..z+4) live in a 9-deep register queue; the loop is unrolled
//     by 9 so queue slots are compile-time registers and nothing is shifted.
//   * x and y neighbours come from the staged plane with 128-bit shared loads (a
//     quarter-warp reads 128 contiguous bytes, so no bank conflicts).
//   * p_next is written with 128-bit streaming stores and may alias p_prev (in-place
//     leapfrog: each element of p_prev is read once, before its own update).
// Arithmetic per point: each axis' centre term is cancelled against its r = 1 pair
// in one FMA and the axes are combined as (x + y) + z, which keeps the rounding
// close to the reference's per-axis evaluation.  Heat takes u + lap in two FMA
// chains whose sum meets the centre in one FMA with weight 1 + (cx + cy + cz).
// Modes: acoustic (the leapfrog step), heat (u + alpha dt lap u) and prepass,
// the first half of the coarse step with the two-step composition term
// (sb200_wave_prepass_f32): r = p + beta dt^2 v^2 lap p into `next`, and
// p_prev + 2 beta dt^2 v^2 lap p written over p_prev, so that the plain step of
// (r, p_prev) is 2p - p_prev + dt^2 L p + beta dt^4 L^2 p (L = v^2 lap).
// Algorithmic DRAM traffic: acoustic 16 B / interior point (read p, p_prev, vel2;
// write p_next), heat 8 B (read u, write u_next), prepass 20 B (read p, p_prev,
// vel2; write r, p_prev).
#include <algorithm>
#include <mutex>

#include "batch.h"
#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {

enum Mode : int { kModeAcoustic = 0, kModeHeat = 1, kModePrepass = 2 };

template <int TX, int TY, int RPT, int S, int AUX>
struct Shape {
    static_assert(TX % 4 == 0, "TX must be a multiple of 4 (16-byte TMA origin)");
    static_assert(TY % RPT == 0, "TY must be a multiple of RPT");
    static_assert(S >= 8, "ring must hold the 8 planes the queue start-up reads");
    static constexpr int SX = TX + 2 * R;
    static constexpr int SY = TY + 2 * R;
    static_assert(SX <= 256 && SY <= 256, "TMA box extent is at most 256");
    static constexpr int TPR = TX / 4;
    static constexpr int NT = TPR * (TY / RPT);
    static constexpr uint32_t PLANE_BYTES = SX * SY * 4u;                  // one p box
    static constexpr int PLANE = int(((PLANE_BYTES + 127u) / 128u) * 32u);  // stride (floats)
    static constexpr uint32_t TILE_BYTES = TX * TY * 4u;                    // p_prev / vel2 box
    static constexpr int TILE = int(((TILE_BYTES + 127u) / 128u) * 32u);
    static constexpr size_t SMEM = size_t(S) * PLANE * 4 + size_t(AUX) * 2 * TILE * 4 + 128;
    static constexpr int MINB = (512 / NT) > 0 ? (512 / NT) : 1;  // caps registers at 128
};

// Ring position a CTA carries from one tile to the next: the sequence numbers of
// the next p plane and the next aux iteration.  Stage = seq % ring size, phase
// parity = (seq / ring size) & 1, so the mbarriers are initialised once per CTA
// and their phases simply continue across the tiles a persistent CTA processes.
struct Ring {
    uint32_t p = 0;
    uint32_t aux = 0;
};

// One tile: columns [x0, x0+TX) x [y0, y0+TY) of the interior, marched over the
// z chunk zc.  All threads of the CTA call it; `sm`, `full` and `auxf` are the
// CTA's rings, initialised by the caller.  Returns false when a bounded wait gave
// up: the error is recorded and every copy in flight has landed.
template <int TX, int TY, int RPT, int S, int AUX, int MODE>
__device__ __forceinline__ bool pencil_tile(const CUtensorMap* pmap, const CUtensorMap* qmap,
                                            const CUtensorMap* vmap, const PencilArgs& a,
                                            int tile_x, int tile_y, int zc, float* sm,
                                            uint64_t* full, uint64_t* auxf, Ring& ring) {
    using P = Shape<TX, TY, RPT, S, AUX>;
    constexpr bool HEAT = MODE == kModeHeat;
    constexpr bool PRE = MODE == kModePrepass;
    constexpr bool kAuxTma = !HEAT && AUX > 0;
    constexpr int NAUX = AUX > 0 ? AUX : 1;
    float* aux = sm + S * P::PLANE;  // AUX stages of [p_prev tile | vel2 tile]

    const int tid = threadIdx.x;
    const int lx = tid % P::TPR;
    const int ly = tid / P::TPR;
    const int x0 = R + tile_x * TX;
    const int y0 = R + tile_y * TY;
    const int zb = R + zc * a.zlen;
    const int ze = min(zb + a.zlen, a.nz - R);
    const int nint = ze - zb;          // interior planes this tile computes (>= 1)
    const int nplanes = nint + 2 * R;  // planes of p it reads (>= 9)
    const uint32_t pb = ring.p;        // sequence number of plane 0
    const uint32_t ab = ring.aux;      // sequence number of aux iteration 0

    int issued_hi = -1;      // thread 0: highest p plane handed to TMA
    int aux_issued_hi = -1;  // thread 0: highest aux iteration handed to TMA
    auto issue_plane = [&](int j) {  // thread 0 only
        const uint32_t s = (pb + j) % S;
        mbar_arrive_expect_tx(&full[s], P::PLANE_BYTES);
        tma_load_3d(sm + s * P::PLANE, pmap, &full[s], x0 - R, y0 - R, zb - R + j);
        issued_hi = j;
    };
    auto issue_aux = [&](int it) {  // thread 0 only
        const uint32_t s = (ab + it) % NAUX;
        float* st = aux + s * 2 * P::TILE;
        mbar_arrive_expect_tx(&auxf[s], 2 * P::TILE_BYTES);
        tma_load_3d(st, qmap, &auxf[s], x0, y0, zb + it);
        tma_load_3d(st + P::TILE, vmap, &auxf[s], x0, y0, zb + it);
        aux_issued_hi = it;
    };
    auto wait_plane = [&](int j) {
        return mbar_wait(&full[(pb + j) % S], ((pb + j) / S) & 1);
    };
    auto wait_aux = [&](int it) {
        return mbar_wait(&auxf[(ab + it) % NAUX], ((ab + it) / NAUX) & 1);
    };
    auto plane = [&](int j) -> const float* { return sm + ((pb + j) % S) * P::PLANE; };

    if (tid == 0) {
        prefetch_tmap(pmap);
        if (kAuxTma) {
            prefetch_tmap(qmap);
            prefetch_tmap(vmap);
        }
        for (int s = 0; s < S && s < nplanes; ++s) issue_plane(s);
        if (kAuxTma)
            for (int it = 0; it < NAUX && it < nint; ++it) issue_aux(it);
    }

    const int gx = x0 + 4 * lx;
    const int gy = y0 + RPT * ly;
    const bool xin = gx < a.nx - R;
    bool rin[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) rin[j] = xin && (gy + j < a.ny - R);
    const int soff = (RPT * ly + R) * P::SX + 4 * lx + R;
    const int aoff = RPT * ly * TX + 4 * lx;  // this thread's first point in an aux tile
    int64_t goff = static_cast<int64_t>(zb) * a.sz + static_cast<int64_t>(gy) * a.sy + gx;

    // Source ownership: which (row, lane element) of this thread, if any.
    int src_j = -1, src_i = -1;
    if (MODE == kModeAcoustic && a.src_z >= 0 && a.src_x >= gx && a.src_x < gx + 4 && a.src_y >= gy &&
        a.src_y < gy + RPT && xin) {
        src_j = a.src_y - gy;
        src_i = a.src_x - gx;
    }

    float2 ax2[R], ay2[R], az2[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        ax2[r] = dup2(a.w.ax[r]);
        ay2[r] = dup2(a.w.ay[r]);
        az2[r] = dup2(a.w.az[r]);
    }
    const float2 cx2 = dup2(a.w.cx), cy2 = dup2(a.w.cy), cz2 = dup2(a.w.cz), neg1 = dup2(-1.f);

    float4 q[9][RPT];
    bool bad = false;
    // Start-up: planes 0..7 (z = zb-4 .. zb+3) fill queue slots 0..7.
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
        if (!wait_plane(jj)) bad = true;
        const float* pl = plane(jj) + soff;
#pragma unroll
        for (int j = 0; j < RPT; ++j) q[jj][j] = lds128(pl + j * P::SX);
    }
    bool abort_run = __syncthreads_or(bad) != 0;
    if (!abort_run && tid == 0) {
        // Planes 0..3 are only queue feed: their stages are free again.
#pragma unroll
        for (int jj = 0; jj < R; ++jj)
            if (jj + S < nplanes) issue_plane(jj + S);
    }

    for (int i0 = 0; i0 < nint && !abort_run; i0 += 9) {
#pragma unroll
        for (int u = 0; u < 9; ++u) {
            const int i = i0 + u;
            if (i < nint && !abort_run) {
                const int cs = (u + 4) % 9;  // centre slot (plane z)
                // p_prev / vel2 of this plane (global-load variant).
                float4 pv[RPT], vv[RPT];
                if (!HEAT && !kAuxTma) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        if (rin[j]) {
                            pv[j] = ldg_cs(a.prev + goff + j * a.sy);
                            vv[j] = ldg_stream(a.vel2 + goff + j * a.sy);
                        }
                    }
                }
                // Queue feed: plane z+4.
                {
                    const int jf = i + 8;
                    if (!wait_plane(jf)) bad = true;
                    const float* pf = plane(jf) + soff;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) q[(u + 8) % 9][j] = lds128(pf + j * P::SX);
                }
                const float* pc = plane(i + 4) + soff;

                // y: neighbour rows outside the own block from shared memory, own
                // rows from the queue centre, accumulated from zero in row order
                // (farthest rows, smallest weights, first).
                // Pairs of points (lanes 0-1, 2-3 of a float4) as packed f32x2:
                // per lane exactly the scalar operations in the same order.
                float2 ya[RPT][2];
#pragma unroll
                for (int j = 0; j < RPT; ++j) ya[j][0] = ya[j][1] = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = -R; k < RPT + R; ++k) {
                    const float4 row = (k >= 0 && k < RPT) ? q[cs][k] : lds128(pc + k * P::SX);
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        const int d = k > j ? k - j : j - k;
                        if (d >= 1 && d <= R) {
                            ya[j][0] = fma2(ay2[d - 1], pair_of(row, 0), ya[j][0]);
                            ya[j][1] = fma2(ay2[d - 1], pair_of(row, 1), ya[j][1]);
                        }
                    }
                }
                // Acoustic / prepass: lap per axis (centre cancelled against the
                // r = 1 pair first), combined as (x + y) + z.  Heat: u + lap in two
                // chains -- the y rows plus the x pairs, and the z pairs -- whose
                // sum takes the centre through one FMA with heat_c, so `lap` holds
                // the new value itself.
                float2 lap[RPT][2];
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    const float4 c = q[cs][j];
                    const float4 lf = lds128(pc + j * P::SX - 4);
                    const float4 rt = lds128(pc + j * P::SX + 4);
                    const float win[12] = {lf.x, lf.y, lf.z, lf.w, c.x, c.y,
                                           c.z,  c.w,  rt.x, rt.y, rt.z, rt.w};
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float2 ce = pair_of(c, h);
                        if constexpr (HEAT) {
                            const int e = 4 + 2 * h;  // window index of the pair's first lane
                            float2 txy = ya[j][h];
                            float2 tz = make_float2(0.f, 0.f);
#pragma unroll
                            for (int r = 1; r <= R; ++r) {
                                const float2 up = pair_of(q[(u + 4 + r) % 9][j], h);
                                const float2 dn = pair_of(q[(u + 4 - r + 9) % 9][j], h);
                                tz = r == 1 ? mul2(az2[0], add2(up, dn))
                                            : fma2(az2[r - 1], add2(up, dn), tz);
                                const float2 s = make_float2(win[e + r] + win[e - r],
                                                             win[e + 1 + r] + win[e + 1 - r]);
                                txy = fma2(ax2[r - 1], s, txy);
                            }
                            lap[j][h] = fma2(dup2(a.heat_c), ce, add2(txy, tz));
                        } else {
                            float2 tz = mul2(cz2, ce);
                            float2 tx = mul2(cx2, ce);
#pragma unroll
                            for (int r = 1; r <= R; ++r) {
                                const float2 up = pair_of(q[(u + 4 + r) % 9][j], h);
                                const float2 dn = pair_of(q[(u + 4 - r + 9) % 9][j], h);
                                tz = fma2(az2[r - 1], add2(up, dn), tz);
                                const int e = 4 + 2 * h;  // window index of the pair's first lane
                                const float2 s = make_float2(win[e + r] + win[e - r],
                                                             win[e + 1 + r] + win[e + 1 - r]);
                                tx = fma2(ax2[r - 1], s, tx);
                            }
                            const float2 ty = fma2(cy2, ce, ya[j][h]);
                            lap[j][h] = add2(add2(tx, ty), tz);
                        }
                    }
                }
                if (kAuxTma) {
                    if (!wait_aux(i)) bad = true;
                    const float* st = aux + ((ab + i) % NAUX) * 2 * P::TILE + aoff;
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        pv[j] = lds128(st + j * TX);
                        vv[j] = lds128(st + P::TILE + j * TX);
                    }
                }
                // Update and store.
                const int z = zb + i;
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
                    const float4 c = q[cs][j];
                    float4 o;
                    if (HEAT) {
                        o = make_float4(lap[j][0].x, lap[j][0].y, lap[j][1].x, lap[j][1].y);
                    } else if (PRE) {
                        // weights carry beta dt^2: r = c + vv lap, p_prev += 2 vv lap
                        const float2 v0 = pair_of(vv[j], 0), v1 = pair_of(vv[j], 1);
                        const float2 r0 = fma2(v0, lap[j][0], pair_of(c, 0));
                        const float2 r1 = fma2(v1, lap[j][1], pair_of(c, 1));
                        const float2 q0 = fma2(add2(v0, v0), lap[j][0], pair_of(pv[j], 0));
                        const float2 q1 = fma2(add2(v1, v1), lap[j][1], pair_of(pv[j], 1));
                        o = make_float4(r0.x, r0.y, r1.x, r1.y);
                        if (rin[j])
                            stg_stream(a.prev_out + goff + j * a.sy,
                                       make_float4(q0.x, q0.y, q1.x, q1.y));
                    } else {
                        // fmaf(vv, lap, fmaf(2, c, -pv)): 2c - pv is rounded once (2c is
                        // exact), as fma(-1, pv, c + c)
                        const float2 t0 = fma2(neg1, pair_of(pv[j], 0), add2(pair_of(c, 0), pair_of(c, 0)));
                        const float2 t1 = fma2(neg1, pair_of(pv[j], 1), add2(pair_of(c, 1), pair_of(c, 1)));
                        const float2 o0 = fma2(pair_of(vv[j], 0), lap[j][0], t0);
                        const float2 o1 = fma2(pair_of(vv[j], 1), lap[j][1], t1);
                        o = make_float4(o0.x, o0.y, o1.x, o1.y);
                        if (src_j == j && z == a.src_z) {
                            const float wv = a.src_wavelet
                                                 ? a.src_wavelet[*a.src_step + a.src_off]
                                                 : a.src_w;
                            const float kv = a.dt2 * f4get(vv[j], src_i);
                            const float add = kv * wv;
                            if (src_i == 0) o.x = o.x + add;
                            if (src_i == 1) o.y = o.y + add;
                            if (src_i == 2) o.z = o.z + add;
                            if (src_i == 3) o.w = o.w + add;
                            if (a.trace)
                                a.trace[(a.src_step ? *a.src_step : 0) + a.src_off] =
                                    f4get(o, src_i);
                        }
                    }
                    if constexpr (HEAT) {  // predicated: no branch per row
                        float* dst = a.next + goff + j * a.sy;  // used only if rin[j]
                        asm volatile(
                            "{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t"
                            "@q st.global.cs.v4.f32 [%0], {%1, %2, %3, %4};\n\t}" ::"l"(dst),
                            "f"(o.x), "f"(o.y), "f"(o.z), "f"(o.w),
                            "r"(static_cast<uint32_t>(rin[j]))
                            : "memory");
                    } else if (rin[j]) {
                        stg_stream(a.next + goff + j * a.sy, o);
                    }
                }
                goff += a.sz;
                // The stages of plane z (p) and of iteration i (aux) are free now:
                // refill them S planes / AUX iterations ahead.
                abort_run = __syncthreads_or(bad) != 0;
                if (!abort_run && tid == 0) {
                    if (i + 4 + S < nplanes) issue_plane(i + 4 + S);
                    if (kAuxTma && i + NAUX < nint) issue_aux(i + NAUX);
                }
            }
        }
    }

    if (abort_run) {
        if (tid == 0) {
            record_error(a.err, kDevWaitTimeout);
            // Let every copy still in flight land before the CTA's shared memory
            // is released or reused (each stage has at most one outstanding fill).
            for (int jj = max(0, issued_hi - S + 1); jj <= issued_hi; ++jj) (void)wait_plane(jj);
            if (kAuxTma)
                for (int it = max(0, aux_issued_hi - NAUX + 1); it <= aux_issued_hi; ++it)
                    (void)wait_aux(it);
        }
        return false;
    }
    ring.p = pb + nplanes;
    if (kAuxTma) ring.aux = ab + nint;
    return true;
}

// Shared-memory rings of a CTA: S planes of p, AUX stages of [p_prev | vel2]
// tiles, and their mbarriers (initialised here by thread 0).
template <int TX, int TY, int RPT, int S, int AUX>
__device__ __forceinline__ float* setup_rings(unsigned char* dsmem, uint64_t* full,
                                              uint64_t* auxf) {
    constexpr int NAUX = AUX > 0 ? AUX : 1;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
#pragma unroll
        for (int s = 0; s < NAUX; ++s) mbar_init(&auxf[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    return reinterpret_cast<float*>(smem_align<128>(dsmem));
}

// One grid: CTA b owns tile (b % tiles_x, (b / tiles_x) % tiles_y) and z chunk
// b / (tiles_x * tiles_y).
template <int TX, int TY, int RPT, int S, int AUX, int MODE>
__global__ void __launch_bounds__(Shape<TX, TY, RPT, S, AUX>::NT, Shape<TX, TY, RPT, S, AUX>::MINB)
    pencil_f32_kernel(const __grid_constant__ CUtensorMap pmap,
                      const __grid_constant__ CUtensorMap qmap,
                      const __grid_constant__ CUtensorMap vmap, const PencilArgs a) {
    constexpr int NAUX = AUX > 0 ? AUX : 1;
    extern __shared__ unsigned char dsmem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t auxf[NAUX];
    float* sm = setup_rings<TX, TY, RPT, S, AUX>(dsmem, full, auxf);
    int b = blockIdx.x;
    const int tx = b % a.tiles_x;
    b /= a.tiles_x;
    const int ty = b % a.tiles_y;
    b /= a.tiles_y;
    Ring ring;
    (void)pencil_tile<TX, TY, RPT, S, AUX, MODE>(&pmap, &qmap, &vmap, a, tx, ty, b, sm, full,
                                                 auxf, ring);
}

// Many grids (shots) in one persistent launch.  Each CTA takes work items --
// (shot, tile x, tile y, z chunk) -- from a device queue with an atomic counter
// until the queue is empty; the last CTA to finish resets the queue and advances
// the step counter the sources read, so the next launch (eager or in a CUDA
// graph) starts clean without a host-side reset.
template <int TX, int TY, int RPT, int S, int AUX>
__global__ void __launch_bounds__(Shape<TX, TY, RPT, S, AUX>::NT, Shape<TX, TY, RPT, S, AUX>::MINB)
    batch_f32_kernel(const ShotF32* __restrict__ shots, const int4* __restrict__ items,
                     int n_items, BatchQueue* queue) {
    constexpr int NAUX = AUX > 0 ? AUX : 1;
    extern __shared__ unsigned char dsmem[];
    __shared__ __align__(8) uint64_t full[S];
    __shared__ __align__(8) uint64_t auxf[NAUX];
    __shared__ int s_item;
    float* sm = setup_rings<TX, TY, RPT, S, AUX>(dsmem, full, auxf);
    Ring ring;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(&queue->next, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();  // every thread has read s_item before it is replaced
        if (it >= n_items) break;
        const int4 w = items[it];
        const ShotF32* sh = shots + w.x;
        const PencilArgs a = sh->args;
        if (!pencil_tile<TX, TY, RPT, S, AUX, kModeAcoustic>(&sh->p, &sh->prev, &sh->vel2, a, w.y, w.z,
                                                     w.w, sm, full, auxf, ring))
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

// ── variant tables ────────────────────────────────────────────────────────────

using LaunchFn = cudaError_t (*)(const PencilMaps&, const PencilArgs&, unsigned, cudaStream_t);
using ResidentFn = int (*)();

// CTAs of a variant that fit on one SM: the occupancy calculator when a device
// is present, else the shared-memory / register limits computed here.
template <int TX, int TY, int RPT, int S, int AUX, int MODE>
int resident_variant() {
    using P = Shape<TX, TY, RPT, S, AUX>;
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63] > 0) return cached[dev & 63];
    auto kern = pencil_f32_kernel<TX, TY, RPT, S, AUX, MODE>;
    int n = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(P::SMEM)) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, P::NT, P::SMEM) == cudaSuccess &&
        n > 0) {
        cached[dev & 63] = n;
        return n;
    }
    cudaGetLastError();
    const int by_smem = int((228u * 1024u) / (P::SMEM + 1024u));
    const int by_regs = 65536 / (P::NT * 128);
    return std::max(1, std::min(by_smem, by_regs));
}

template <int TX, int TY, int RPT, int S, int AUX, int MODE>
cudaError_t launch_variant(const PencilMaps& m, const PencilArgs& a, unsigned ctas,
                           cudaStream_t stream) {
    using P = Shape<TX, TY, RPT, S, AUX>;
    // Sets the shared-memory attribute on the first call per device (cached).
    resident_variant<TX, TY, RPT, S, AUX, MODE>();
    pencil_f32_kernel<TX, TY, RPT, S, AUX, MODE><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev,
                                                                                 m.vel2, a);
    return cudaGetLastError();
}

struct Variant {
    int tx, ty, rpt, stages, aux;
    const char* name;
    LaunchFn launch;
    ResidentFn resident;
    LaunchFn launch_prepass;  // acoustic tiles only: the same shape in prepass mode
};

// The prepass launcher of an acoustic tile (heat tiles have none).
template <int TX, int TY, int RPT, int S, int AUX, bool HEAT>
constexpr LaunchFn prepass_launcher() {
    if constexpr (HEAT)
        return nullptr;
    else
        return &launch_variant<TX, TY, RPT, S, AUX, kModePrepass>;
}

#define SB200_VARIANT(TX, TY, RPT, S, AUX, HEAT, NAME)                                       \
    Variant {                                                                                \
        TX, TY, RPT, S, AUX, NAME,                                                           \
            &launch_variant<TX, TY, RPT, S, AUX, HEAT ? kModeHeat : kModeAcoustic>,          \
            &resident_variant<TX, TY, RPT, S, AUX, HEAT ? kModeHeat : kModeAcoustic>,        \
            prepass_launcher<TX, TY, RPT, S, AUX, HEAT>()                                    \
    }

// Index 0 of each table is the default when no tuned choice exists.
const Variant kWave[] = {
    SB200_VARIANT(32, 32, 2, 8, 4, false, "t32x32_r2_s8_a4"),
    SB200_VARIANT(32, 32, 2, 8, 2, false, "t32x32_r2_s8_a2"),
    SB200_VARIANT(32, 32, 2, 8, 0, false, "t32x32_r2_s8_ldg"),
    SB200_VARIANT(64, 16, 2, 8, 3, false, "t64x16_r2_s8_a3"),
    SB200_VARIANT(32, 16, 1, 8, 4, false, "t32x16_r1_s8_a4"),
    SB200_VARIANT(64, 32, 2, 8, 3, false, "t64x32_r2_s8_a3"),
    SB200_VARIANT(32, 64, 2, 8, 3, false, "t32x64_r2_s8_a3"),
};
const Variant kHeat[] = {
    SB200_VARIANT(32, 32, 2, 8, 0, true, "t32x32_r2_s8"),
    SB200_VARIANT(64, 16, 2, 8, 0, true, "t64x16_r2_s8"),
    SB200_VARIANT(32, 16, 1, 8, 0, true, "t32x16_r1_s8"),
    SB200_VARIANT(64, 32, 2, 8, 0, true, "t64x32_r2_s8"),
    SB200_VARIANT(32, 64, 2, 8, 0, true, "t32x64_r2_s8"),
    SB200_VARIANT(128, 16, 2, 8, 0, true, "t128x16_r2_s8"),
};
constexpr int kNumWave = sizeof(kWave) / sizeof(kWave[0]);
constexpr int kNumHeat = sizeof(kHeat) / sizeof(kHeat[0]);

const Variant& variant_of(bool heat, int v) { return heat ? kHeat[v] : kWave[v]; }

PencilArgs base_args(int tile_x, int tile_y, const GridDesc& g, int zchunks, int* err) {
    PencilArgs a{};
    a.nx = static_cast<int>(g.nx);
    a.ny = static_cast<int>(g.ny);
    a.nz = static_cast<int>(g.nz);
    a.sy = g.nx;
    a.sz = g.nx * g.ny;
    a.tiles_x = static_cast<int>((g.nx - 2 * R + tile_x - 1) / tile_x);
    a.tiles_y = static_cast<int>((g.ny - 2 * R + tile_y - 1) / tile_y);
    const int inz = static_cast<int>(g.nz - 2 * R);
    const int zc = std::max(1, std::min(zchunks, inz));
    a.zlen = (inz + zc - 1) / zc;
    a.src_x = a.src_y = a.src_z = -1;
    a.err = err;
    return a;
}

unsigned ctas_of(const PencilArgs& a, const GridDesc& g) {
    const int inz = static_cast<int>(g.nz - 2 * R);
    const int zc = (inz + a.zlen - 1) / a.zlen;
    return static_cast<unsigned>(int64_t(a.tiles_x) * a.tiles_y * zc);
}

}  // namespace

Weights fold_weights(const GridDesc& g, float scale) {
    const float c[R] = {C1, C2, C3, C4};
    const float ix2 = 1.0f / (g.dx * g.dx);
    const float iy2 = 1.0f / (g.dy * g.dy);
    const float iz2 = 1.0f / (g.dz * g.dz);
    Weights w;
    w.cx = static_cast<float>(double(C0) * ix2 * scale);
    w.cy = static_cast<float>(double(C0) * iy2 * scale);
    w.cz = static_cast<float>(double(C0) * iz2 * scale);
    for (int r = 0; r < R; ++r) {
        w.ax[r] = static_cast<float>(double(c[r]) * ix2 * scale);
        w.ay[r] = static_cast<float>(double(c[r]) * iy2 * scale);
        w.az[r] = static_cast<float>(double(c[r]) * iz2 * scale);
    }
    return w;
}


int pencil_f32_variant_count(bool heat) { return heat ? kNumHeat : kNumWave; }

const char* pencil_f32_variant_name(bool heat, int v) {
    return (v >= 0 && v < pencil_f32_variant_count(heat)) ? variant_of(heat, v).name : nullptr;
}

PencilBoxes pencil_f32_boxes(bool heat, int v) {
    const Variant& x = variant_of(heat, v);
    PencilBoxes b;
    b.halo_x = x.tx + 2 * R;
    b.halo_y = x.ty + 2 * R;
    b.tile_x = x.tx;
    b.tile_y = x.ty;
    b.aux_tma = !heat && x.aux > 0;
    return b;
}

int pencil_f32_resident(bool heat, int v) { return variant_of(heat, v).resident(); }

void pencil_f32_prepare() {
    for (int v = 0; v < kNumWave; ++v) kWave[v].resident();
    for (int v = 0; v < kNumHeat; ++v) kHeat[v].resident();
}

int64_t pencil_f32_ctas(bool heat, int v, const GridDesc& g, int zchunks) {
    return ctas_of(base_args(variant_of(heat, v).tx, variant_of(heat, v).ty, g, zchunks, nullptr), g);
}

cudaError_t launch_wave_pencil_f32(const PencilMaps& maps, const float* prev, const float* vel2,
                                   float* next, const GridDesc& g, const SourceDesc& src,
                                   const PencilConfig& cfg, int* err, cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const Variant& v = kWave[cfg.variant];
    PencilArgs a = base_args(v.tx, v.ty, g, cfg.zchunks, err);
    a.prev = prev;
    a.vel2 = vel2;
    a.next = next;
    a.dt2 = g.dt * g.dt;
    a.w = fold_weights(g, a.dt2);
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
    return v.launch(maps, a, ctas_of(a, g), stream);
}

cudaError_t launch_prepass_pencil_f32(const PencilMaps& maps, float* prev, const float* vel2,
                                      float* r, const GridDesc& g, float beta,
                                      const PencilConfig& cfg, int* err, cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const Variant& v = kWave[cfg.variant];
    PencilArgs a = base_args(v.tx, v.ty, g, cfg.zchunks, err);
    a.prev = prev;
    a.prev_out = prev;
    a.vel2 = vel2;
    a.next = r;
    a.w = fold_weights(g, beta * g.dt * g.dt);
    return v.launch_prepass(maps, a, ctas_of(a, g), stream);
}

cudaError_t launch_heat_pencil_f32(const PencilMaps& maps, float* u_next, const GridDesc& g,
                                   float alpha_dt, const PencilConfig& cfg, int* err,
                                   cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    const Variant& v = kHeat[cfg.variant];
    PencilArgs a = base_args(v.tx, v.ty, g, cfg.zchunks, err);
    a.next = u_next;
    a.w = fold_weights(g, alpha_dt);
    a.heat_c = static_cast<float>(
        1.0 + double(C0) * alpha_dt *
                  (1.0 / (double(g.dx) * g.dx) + 1.0 / (double(g.dy) * g.dy) +
                   1.0 / (double(g.dz) * g.dz)));
    return v.launch(maps, a, ctas_of(a, g), stream);
}

// ── batched shots ─────────────────────────────────────────────────────────────

namespace {

template <int TX, int TY, int RPT, int S, int AUX>
int resident_batch() {
    using P = Shape<TX, TY, RPT, S, AUX>;
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63] > 0) return cached[dev & 63];
    auto kern = batch_f32_kernel<TX, TY, RPT, S, AUX>;
    int n = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(P::SMEM)) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, P::NT, P::SMEM) == cudaSuccess &&
        n > 0) {
        cached[dev & 63] = n;
        return n;
    }
    cudaGetLastError();
    const int by_smem = int((228u * 1024u) / (P::SMEM + 1024u));
    const int by_regs = 65536 / (P::NT * 128);
    return std::max(1, std::min(by_smem, by_regs));
}

template <int TX, int TY, int RPT, int S, int AUX>
cudaError_t launch_batch(const ShotF32* shots, const int4* items, int n_items, BatchQueue* q,
                         unsigned ctas, cudaStream_t stream) {
    using P = Shape<TX, TY, RPT, S, AUX>;
    resident_batch<TX, TY, RPT, S, AUX>();
    batch_f32_kernel<TX, TY, RPT, S, AUX><<<ctas, P::NT, P::SMEM, stream>>>(shots, items, n_items,
                                                                           q);
    return cudaGetLastError();
}

struct BatchVariant {
    int tx, ty;
    const char* name;
    cudaError_t (*launch)(const ShotF32*, const int4*, int, BatchQueue*, unsigned, cudaStream_t);
    int (*resident)();
};

#define SB200_BATCH_VARIANT(TX, TY, RPT, S, AUX, NAME) \
    BatchVariant { TX, TY, NAME, &launch_batch<TX, TY, RPT, S, AUX>, &resident_batch<TX, TY, RPT, S, AUX> }

const BatchVariant kBatch[] = {
    SB200_BATCH_VARIANT(32, 32, 2, 8, 4, "b32x32_r2_s8_a4"),
    SB200_BATCH_VARIANT(64, 16, 2, 8, 3, "b64x16_r2_s8_a3"),
    SB200_BATCH_VARIANT(32, 16, 1, 8, 4, "b32x16_r1_s8_a4"),
    SB200_BATCH_VARIANT(64, 32, 2, 8, 3, "b64x32_r2_s8_a3"),
};
constexpr int kNumBatch = sizeof(kBatch) / sizeof(kBatch[0]);

}  // namespace

int batch_f32_variant_count() { return kNumBatch; }

const char* batch_f32_variant_name(int v) {
    return (v >= 0 && v < kNumBatch) ? kBatch[v].name : nullptr;
}

PencilBoxes batch_f32_boxes(int v) {
    PencilBoxes b;
    b.halo_x = kBatch[v].tx + 2 * R;
    b.halo_y = kBatch[v].ty + 2 * R;
    b.tile_x = kBatch[v].tx;
    b.tile_y = kBatch[v].ty;
    b.aux_tma = true;
    return b;
}

int batch_f32_resident(int v) { return kBatch[v].resident(); }

void batch_f32_prepare() {
    for (int v = 0; v < kNumBatch; ++v) kBatch[v].resident();
}

PencilArgs batch_f32_shot_args(int v, const GridDesc& g, int zchunks, float* next,
                               const SourceDesc& src, int* err) {
    PencilArgs a = base_args(kBatch[v].tx, kBatch[v].ty, g, zchunks, err);
    a.prev = next;
    a.next = next;
    a.dt2 = g.dt * g.dt;
    a.w = fold_weights(g, a.dt2);
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
    return a;
}

cudaError_t launch_batch_f32(int v, const ShotF32* shots, const int4* items, int n_items,
                             BatchQueue* queue, unsigned ctas, cudaStream_t stream) {
    return kBatch[v].launch(shots, items, n_items, queue, ctas, stream);
}

}  // namespace sb200
