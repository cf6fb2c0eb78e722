// Two acoustic leapfrog steps per sweep (temporal blocking), FP32, sm_100a.
//
// The one-step pencil kernel (pencil_f32.cu) moves 16 B per interior point and
// step (read p, p_prev, vel2; write p_next) and runs at the copy bandwidth.  This
// kernel advances two steps per pass over the grid and moves 20 B per point for
// the pair (read p, p_prev, vel2; write p at t+dt and at t+2dt): 10 B per point
// and step.  Each per-point operation is the one-step kernel's, in the same order,
// so two steps here give the same bits as two one-step launches.
//
// A CTA owns a TX x TY tile of interior columns and marches z over a chunk:
//   * stage A computes q = p(t+dt) at plane z on the tile widened by the stencil
//     radius, (TX+8) x (TY+8) -- the x-y neighbours stage B needs -- from p
//     planes staged by TMA with an 8-cell halo ((TX+16) x (TY+16)), a 9-deep
//     register queue of p for the z neighbours, and the p_prev / vel2 tiles of the
//     widened region (TMA rings);
//   * stage B computes p(t+2dt) on the tile at plane z-4 from the q planes of the
//     last five iterations (a shared-memory ring, x-y neighbours) and a 9-deep
//     register queue of q for the z neighbours; p_prev of that step is p itself,
//     still in the first queue, and vel2 is still in its ring.
// Each thread owns a float4 of x in RPT (1 or 2) rows of the widened region; the
// threads whose rows lie in the tile run both stages, the others (the 4-cell ring
// around the tile) stage A only.  Points of the widened region outside the grid's
// interior keep p_prev's value (a one-step launch never writes them, and it runs
// in place over p_prev).  The z chunk is widened by 4 planes on each side for
// stage A (q at z-4..z+4 of every output plane), so the chunk reads 16 halo
// planes of p instead of 8.
//
// Inputs and outputs are five distinct buffers: other CTAs read p and p_prev of
// this tile's columns (their widened regions) while this one writes its results.
#include <algorithm>

#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

namespace {

struct Leap2Args {
    float* out1;  // p at t+dt   (interior written)
    float* out2;  // p at t+2dt  (interior written)
    int nx, ny, nz;
    int64_t sy, sz;
    int tiles_x, tiles_y, zlen;
    Weights w;  // weights * dt^2
    float dt2;
    int src_x, src_y, src_z;  // -1 when there is no source
    float src_w0, src_w1;     // host samples of the two steps (no wavelet table)
    const float* src_wavelet;
    const int* src_step;
    int src_off;  // steps s and s+1 read wavelet[*src_step + src_off (+1)]
    float* trace;
    int* err;
};

template <int TX, int TY, int RPT, int S, int AQ, int AV>
struct Shape2 {
    static_assert(RPT == 1 || RPT == 2, "one or two rows per thread");
    static_assert(TX % 4 == 0 && TY % RPT == 0, "float4 columns, RPT-row tasks");
    static_assert(S >= 8, "the p ring holds the 8 planes the queue start-up reads");
    static_assert(AV >= 6, "vel2 stays staged for stage B, 4 iterations later");
    static_assert(AQ >= 2, "p_prev ring");
    static constexpr int EX = TX + 2 * R, EY = TY + 2 * R;  // widened region
    static constexpr int SX0 = TX + 4 * R, SY0 = TY + 4 * R;  // p box
    static_assert(SX0 <= 256 && SY0 <= 256, "TMA box extent is at most 256");
    static constexpr int CX = EX / 4;                 // float4 columns of the widened region
    static constexpr int NB = (TX / 4) * (TY / RPT);  // tasks in the tile (both stages)
    static constexpr int NT = CX * (EY / RPT);        // threads: every task of the widened region
    static constexpr uint32_t P_BYTES = SX0 * SY0 * 4u;
    static constexpr int PST = int(((P_BYTES + 127u) / 128u) * 32u);  // stage stride, floats
    static constexpr uint32_t E_BYTES = EX * EY * 4u;
    static constexpr int EST = int(((E_BYTES + 127u) / 128u) * 32u);
    static constexpr int QS = 5;  // q planes kept for stage B (z-4 .. z)
    static constexpr size_t SMEM = (size_t(S) * PST + size_t(AQ + AV + QS) * EST) * 4 + 128;
};

__device__ __forceinline__ void sts128(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

// The one-step kernel's per-point arithmetic on RPT rows of a float4 column
// (pencil_f32.cu, acoustic mode): y rows accumulated in row order, x and z pairs
// with the centre cancelled first, combined as (x + y) + z; the update rounds
// 2c - p_prev once, then adds vel2 * lap.  Packed f32x2 lanes round as scalars.
struct Leap2Math {
    float2 ax2[R], ay2[R], az2[R], cx2, cy2, cz2, neg1;
    __device__ explicit Leap2Math(const Weights& w) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            ax2[r] = dup2(w.ax[r]);
            ay2[r] = dup2(w.ay[r]);
            az2[r] = dup2(w.az[r]);
        }
        cx2 = dup2(w.cx);
        cy2 = dup2(w.cy);
        cz2 = dup2(w.cz);
        neg1 = dup2(-1.f);
    }
    // pc: the task's first point in a staged plane of row stride SX; c: its own
    // RPT rows; up(r, row) / dn(r, row): the z neighbours at +-r.
    template <int RPT, class Up, class Dn>
    __device__ __forceinline__ void laplacian(const float* pc, int SX, const float4 (&c)[RPT],
                                              Up&& up, Dn&& dn, float2 (&lap)[RPT][2]) const {
        float2 ya[RPT][2];
#pragma unroll
        for (int j = 0; j < RPT; ++j) ya[j][0] = ya[j][1] = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = -R; k < RPT + R; ++k) {
            const float4 row = (k >= 0 && k < RPT) ? c[k] : lds128(pc + k * SX);
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                const int d = k > j ? k - j : j - k;
                if (d >= 1 && d <= R) {
                    ya[j][0] = fma2(ay2[d - 1], pair_of(row, 0), ya[j][0]);
                    ya[j][1] = fma2(ay2[d - 1], pair_of(row, 1), ya[j][1]);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const float4 cc = c[j];
            const float4 lf = lds128(pc + j * SX - 4);
            const float4 rt = lds128(pc + j * SX + 4);
            const float win[12] = {lf.x, lf.y, lf.z, lf.w, cc.x, cc.y,
                                   cc.z, cc.w, rt.x, rt.y, rt.z, rt.w};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float2 ce = pair_of(cc, h);
                float2 tz = mul2(cz2, ce);
                float2 tx = mul2(cx2, ce);
#pragma unroll
                for (int r = 1; r <= R; ++r) {
                    tz = fma2(az2[r - 1], add2(pair_of(up(r, j), h), pair_of(dn(r, j), h)), tz);
                    const int e = 4 + 2 * h;
                    const float2 s = make_float2(win[e + r] + win[e - r],
                                                 win[e + 1 + r] + win[e + 1 - r]);
                    tx = fma2(ax2[r - 1], s, tx);
                }
                const float2 ty = fma2(cy2, ce, ya[j][h]);
                lap[j][h] = add2(add2(tx, ty), tz);
            }
        }
    }
    __device__ __forceinline__ float4 update(const float4& c, const float4& pv, const float4& vv,
                                             const float2 (&lap)[2]) const {
        const float2 t0 = fma2(neg1, pair_of(pv, 0), add2(pair_of(c, 0), pair_of(c, 0)));
        const float2 t1 = fma2(neg1, pair_of(pv, 1), add2(pair_of(c, 1), pair_of(c, 1)));
        const float2 o0 = fma2(pair_of(vv, 0), lap[0], t0);
        const float2 o1 = fma2(pair_of(vv, 1), lap[1], t1);
        return make_float4(o0.x, o0.y, o1.x, o1.y);
    }
    // element e of o += (dt2 vel2[e]) * w, rounded as the one-step kernel rounds it
    __device__ __forceinline__ static void add_source(float4& o, const float4& vv, float dt2,
                                                      float w, int e) {
        const float add = (dt2 * f4get(vv, e)) * w;
        if (e == 0) o.x = o.x + add;
        if (e == 1) o.y = o.y + add;
        if (e == 2) o.z = o.z + add;
        if (e == 3) o.w = o.w + add;
    }
};

// Source sample k (0: step s, 1: step s+1) and the trace record of that step.
__device__ __forceinline__ float source_sample(const Leap2Args& a, int k) {
    return a.src_wavelet ? a.src_wavelet[*a.src_step + a.src_off + k]
                         : (k == 0 ? a.src_w0 : a.src_w1);
}
__device__ __forceinline__ void record_trace(const Leap2Args& a, int k, float v) {
    if (a.trace) a.trace[(a.src_step ? *a.src_step : 0) + a.src_off + k] = v;
}

// Thread t -> its task: float4 column ex and first row ey (of RPT) of the widened
// region.  Threads [0, NB) take the tile row-major; the rest take the ring: the
// 4 rows above the tile, the 4 below, then the left / right column of each task
// row beside it.
template <int TX, int TY, int RPT>
__device__ __forceinline__ void task_of(int t, int& ex, int& ey) {
    constexpr int CX = (TX + 2 * R) / 4, EY = TY + 2 * R, NB = (TX / 4) * (TY / RPT);
    if (t < NB) {
        ex = 1 + t % (TX / 4);
        ey = R + RPT * (t / (TX / 4));
        return;
    }
    int k = t - NB;
    constexpr int band = (R / RPT) * CX;  // the 4 rows above (below) the tile
    if (k < band) {
        ex = k % CX;
        ey = RPT * (k / CX);
        return;
    }
    k -= band;
    if (k < band) {
        ex = k % CX;
        ey = EY - R + RPT * (k / CX);
        return;
    }
    k -= band;
    ex = (k & 1) ? CX - 1 : 0;
    ey = R + RPT * (k >> 1);
}

template <int TX, int TY, int RPT, int S, int AQ, int AV>
__global__ void __launch_bounds__(Shape2<TX, TY, RPT, S, AQ, AV>::NT, 1)
    leap2_kernel(const __grid_constant__ CUtensorMap pmap, const __grid_constant__ CUtensorMap qmap,
                 const __grid_constant__ CUtensorMap vmap, const Leap2Args a) {
    using P = Shape2<TX, TY, RPT, S, AQ, AV>;
    extern __shared__ unsigned char dsmem[];
    __shared__ __align__(8) uint64_t fullp[S];
    __shared__ __align__(8) uint64_t fullq[AQ];
    __shared__ __align__(8) uint64_t fullv[AV];
    const int tid = threadIdx.x;
    if (tid == 0) {
#pragma unroll
        for (int s = 0; s < S; ++s) mbar_init(&fullp[s], 1);
#pragma unroll
        for (int s = 0; s < AQ; ++s) mbar_init(&fullq[s], 1);
#pragma unroll
        for (int s = 0; s < AV; ++s) mbar_init(&fullv[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    float* sp = reinterpret_cast<float*>(smem_align<128>(dsmem));  // S p planes
    float* sq = sp + S * P::PST;                                   // AQ p_prev tiles
    float* sv = sq + AQ * P::EST;                                  // AV vel2 tiles
    float* s1 = sv + AV * P::EST;                                  // QS planes of q

    int b = blockIdx.x;
    const int tile_x = b % a.tiles_x;
    b /= a.tiles_x;
    const int tile_y = b % a.tiles_y;
    const int zc = b / a.tiles_y;
    const int x0 = R + tile_x * TX;
    const int y0 = R + tile_y * TY;
    const int zb = R + zc * a.zlen;
    const int ze = min(zb + a.zlen, a.nz - R);
    const int nint = ze - zb;       // output planes (>= 1)
    const int nit = nint + 2 * R;   // iterations: stage A at z = zb-4 .. ze+3
    const int np = nint + 4 * R;    // p planes read: z = zb-8 .. ze+7

    int hp = -1, hq = -1, hv = -1;  // thread 0: highest index issued per ring
    auto issue_p = [&](int j) {
        const int s = j % S;
        mbar_arrive_expect_tx(&fullp[s], P::P_BYTES);
        tma_load_3d(sp + s * P::PST, &pmap, &fullp[s], x0 - 2 * R, y0 - 2 * R, zb - 2 * R + j);
        hp = j;
    };
    auto issue_q = [&](int i) {
        const int s = i % AQ;
        mbar_arrive_expect_tx(&fullq[s], P::E_BYTES);
        tma_load_3d(sq + s * P::EST, &qmap, &fullq[s], x0 - R, y0 - R, zb - R + i);
        hq = i;
    };
    auto issue_v = [&](int i) {
        const int s = i % AV;
        mbar_arrive_expect_tx(&fullv[s], P::E_BYTES);
        tma_load_3d(sv + s * P::EST, &vmap, &fullv[s], x0 - R, y0 - R, zb - R + i);
        hv = i;
    };
    auto wait_p = [&](int j) { return mbar_wait(&fullp[j % S], (j / S) & 1); };
    auto wait_q = [&](int i) { return mbar_wait(&fullq[i % AQ], (i / AQ) & 1); };
    auto wait_v = [&](int i) { return mbar_wait(&fullv[i % AV], (i / AV) & 1); };

    if (tid == 0) {
        prefetch_tmap(&pmap);
        prefetch_tmap(&qmap);
        prefetch_tmap(&vmap);
        for (int j = 0; j < S && j < np; ++j) issue_p(j);
        for (int i = 0; i < AQ && i < nit; ++i) issue_q(i);
        for (int i = 0; i < AV && i < nit; ++i) issue_v(i);
    }

    int ex, ey;
    task_of<TX, TY, RPT>(tid, ex, ey);
    const bool inner = tid < P::NB;  // the task lies in the tile: stage B too
    const int gx = x0 - R + 4 * ex;  // first x of the task (a multiple of 4)
    const int gy = y0 - R + ey;      // first row of the task
    const bool xin = gx >= R && gx < a.nx - R;  // the float4 is interior or halo as a whole
    bool rin[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) rin[r] = xin && gy + r >= R && gy + r < a.ny - R;
    const int poff = (ey + R) * P::SX0 + 4 * ex + R;  // task in a p plane
    const int eoff = ey * P::EX + 4 * ex;             // task in a widened-region tile

    // Source ownership (row, element) within the task.
    int src_r = -1, src_e = 0;
    if (a.src_z >= 0 && a.src_x >= gx && a.src_x < gx + 4 && a.src_y >= gy && a.src_y < gy + RPT &&
        xin) {
        src_r = a.src_y - gy;
        src_e = a.src_x - gx;
    }

    const Leap2Math m(a.w);

    float4 qp[9][RPT];  // p: planes z-4 .. z+4 of stage A (slot = plane index % 9)
    float4 q1[9][RPT];  // q: planes z-8 .. z of stage B's z neighbours (slot = iteration % 9)
    bool bad = false;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (!wait_p(j)) bad = true;
        const float* pl = sp + (j % S) * P::PST + poff;
#pragma unroll
        for (int r = 0; r < RPT; ++r) qp[j][r] = lds128(pl + r * P::SX0);
    }
    bool abort_run = __syncthreads_or(bad) != 0;
    if (!abort_run && tid == 0)
#pragma unroll
        for (int j = 0; j < R; ++j)  // planes 0..3 are queue feed only
            if (j + S < np) issue_p(j + S);

    int64_t goff = static_cast<int64_t>(zb - R) * a.sz + static_cast<int64_t>(gy) * a.sy + gx;
    for (int i0 = 0; i0 < nit && !abort_run; i0 += 9) {
#pragma unroll
        for (int u = 0; u < 9; ++u) {
            const int i = i0 + u;  // stage A at z = zb - 4 + i, stage B at z - 4
            if (i < nit && !abort_run) {
                const int za = zb - R + i;
                // feed: p plane i + 8 (z + 4) into the slot of plane i - 1
                {
                    if (!wait_p(i + 8)) bad = true;
                    const float* pf = sp + ((i + 8) % S) * P::PST + poff;
#pragma unroll
                    for (int r = 0; r < RPT; ++r) qp[(u + 8) % 9][r] = lds128(pf + r * P::SX0);
                }
                // ── stage A: q at za over the widened region ──
                if (!wait_q(i)) bad = true;
                if (!wait_v(i)) bad = true;
                const float* qt = sq + (i % AQ) * P::EST + eoff;
                const float* vt = sv + (i % AV) * P::EST + eoff;
                float4 pv[RPT], qn[RPT];
#pragma unroll
                for (int r = 0; r < RPT; ++r) qn[r] = pv[r] = lds128(qt + r * P::EX);
                if (za >= R && za < a.nz - R) {  // CTA-uniform
                    float4 vv[RPT], c[RPT];
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        vv[r] = lds128(vt + r * P::EX);
                        c[r] = qp[(u + 4) % 9][r];
                    }
                    float2 lap[RPT][2];
                    m.laplacian(sp + ((i + 4) % S) * P::PST + poff, P::SX0, c,
                              [&](int r, int j) -> const float4& { return qp[(u + 4 + r) % 9][j]; },
                              [&](int r, int j) -> const float4& { return qp[(u + 4 - r + 9) % 9][j]; },
                              lap);
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        float4 o = m.update(c[r], pv[r], vv[r], lap[r]);
                        if (src_r == r && za == a.src_z) {
                            Leap2Math::add_source(o, vv[r], a.dt2, source_sample(a, 0), src_e);
                            if (inner && za >= zb && za < ze) record_trace(a, 0, f4get(o, src_e));
                        }
                        if (rin[r]) qn[r] = o;  // halo points keep p_prev
                    }
                }
#pragma unroll
                for (int r = 0; r < RPT; ++r) sts128(s1 + (i % P::QS) * P::EST + eoff + r * P::EX, qn[r]);
                if (inner) {
#pragma unroll
                    for (int r = 0; r < RPT; ++r) q1[u][r] = qn[r];
                    if (za >= zb && za < ze) {
#pragma unroll
                        for (int r = 0; r < RPT; ++r)
                            if (rin[r]) stg_stream(a.out1 + goff + r * a.sy, qn[r]);
                    }
                }
                // ── stage B: p(t+2dt) at za - 4 over the tile ──
                // (no barrier: it reads the q plane written 4 iterations ago and
                // this thread's own q of za from its queue)
                if (inner && i >= 2 * R) {
                    const float* vb = sv + ((i - R) % AV) * P::EST + eoff;
                    float4 c[RPT], pv[RPT], vv[RPT];  // pv: p at za - 4
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        c[r] = q1[(u + 5) % 9][r];
                        pv[r] = qp[u % 9][r];
                        vv[r] = lds128(vb + r * P::EX);
                    }
                    float2 lap[RPT][2];
                    m.laplacian(s1 + ((i - R) % P::QS) * P::EST + eoff, P::EX, c,
                              [&](int r, int j) -> const float4& { return q1[(u + 5 + r) % 9][j]; },
                              [&](int r, int j) -> const float4& { return q1[(u + 5 - r + 9) % 9][j]; },
                              lap);
                    const int zbb = za - R;
#pragma unroll
                    for (int r = 0; r < RPT; ++r) {
                        float4 o = m.update(c[r], pv[r], vv[r], lap[r]);
                        if (src_r == r && zbb == a.src_z) {
                            Leap2Math::add_source(o, vv[r], a.dt2, source_sample(a, 1), src_e);
                            record_trace(a, 1, f4get(o, src_e));
                        }
                        if (rin[r]) stg_stream(a.out2 + goff - R * a.sz + r * a.sy, o);
                    }
                }
                goff += a.sz;
                // p plane i + 4 (stage A's centre), p_prev of iteration i and vel2
                // of iteration i - 4 (stage B) are free: refill them.
                abort_run = __syncthreads_or(bad) != 0;
                if (!abort_run && tid == 0) {
                    if (i + 4 + S < np) issue_p(i + 4 + S);
                    if (i + AQ < nit) issue_q(i + AQ);
                    if (i >= R && i - R + AV < nit) issue_v(i - R + AV);
                }
            }
        }
    }

    if (abort_run && tid == 0) {
        record_error(a.err, kDevWaitTimeout);
        // every copy still in flight lands before the CTA exits
        for (int j = max(0, hp - S + 1); j <= hp; ++j) (void)wait_p(j);
        for (int k = max(0, hq - AQ + 1); k <= hq; ++k) (void)wait_q(k);
        for (int k = max(0, hv - AV + 1); k <= hv; ++k) (void)wait_v(k);
    }
}

template <int TX, int TY, int RPT, int S, int AQ, int AV>
int resident_leap2() {
    using P = Shape2<TX, TY, RPT, S, AQ, AV>;
    static int cached[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (cached[dev & 63] > 0) return cached[dev & 63];
    auto kern = leap2_kernel<TX, TY, RPT, S, AQ, AV>;
    int n = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(P::SMEM)) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, P::NT, P::SMEM) == cudaSuccess &&
        n > 0) {
        cached[dev & 63] = n;
        return n;
    }
    cudaGetLastError();
    return 1;
}

template <int TX, int TY, int RPT, int S, int AQ, int AV>
cudaError_t launch_leap2(const PencilMaps& m, const Leap2Args& a, unsigned ctas,
                         cudaStream_t stream) {
    using P = Shape2<TX, TY, RPT, S, AQ, AV>;
    resident_leap2<TX, TY, RPT, S, AQ, AV>();  // sets the shared-memory attribute once per device
    leap2_kernel<TX, TY, RPT, S, AQ, AV><<<ctas, P::NT, P::SMEM, stream>>>(m.p, m.prev, m.vel2, a);
    return cudaGetLastError();
}

struct Leap2Variant {
    int tx, ty;
    const char* name;
    cudaError_t (*launch)(const PencilMaps&, const Leap2Args&, unsigned, cudaStream_t);
    int (*resident)();
};

#define SB200_LEAP2(TX, TY, RPT, S, AQ, AV, NAME)                                      \
    Leap2Variant {                                                                     \
        TX, TY, NAME, &launch_leap2<TX, TY, RPT, S, AQ, AV>,                           \
            &resident_leap2<TX, TY, RPT, S, AQ, AV>                                    \
    }

// Measured at 1024^3 (ms per step, one-step kernel 2.72-2.73): l64x16 3.94-3.96,
// l32x32 one row per thread (400 threads, 126 registers, 13 warps per SM; the
// default) 3.90-3.96.  Not kept: l32x32 two rows 3.97-4.07, l64x16 one row
// 3.95-4.01 (z split 2-4); a warp-specialised form (A warps holding the p queue,
// B warps the q queue, q planes handed over through an mbarrier ring; 158-161
// registers, 11 warps per SM) at 7.26-7.48 -- its two 9x-unrolled loops run side
// by side and stall on instruction fetch (6.1 stalls per issue against 1.3).
const Leap2Variant kLeap2[] = {
    SB200_LEAP2(64, 16, 2, 8, 3, 8, "l64x16_s8"),
    SB200_LEAP2(32, 32, 1, 8, 3, 8, "l32x32_r1_s8"),
};
constexpr int kNumLeap2 = sizeof(kLeap2) / sizeof(kLeap2[0]);

Leap2Args leap2_args(int v, const GridDesc& g, int zchunks, int* err) {
    Leap2Args a{};
    a.nx = static_cast<int>(g.nx);
    a.ny = static_cast<int>(g.ny);
    a.nz = static_cast<int>(g.nz);
    a.sy = g.nx;
    a.sz = g.nx * g.ny;
    a.tiles_x = static_cast<int>((g.nx - 2 * R + kLeap2[v].tx - 1) / kLeap2[v].tx);
    a.tiles_y = static_cast<int>((g.ny - 2 * R + kLeap2[v].ty - 1) / kLeap2[v].ty);
    const int inz = static_cast<int>(g.nz - 2 * R);
    const int zc = std::max(1, std::min(zchunks, inz));
    a.zlen = (inz + zc - 1) / zc;
    a.src_x = a.src_y = a.src_z = -1;
    a.err = err;
    return a;
}

unsigned leap2_ctas_of(const Leap2Args& a, const GridDesc& g) {
    const int inz = static_cast<int>(g.nz - 2 * R);
    return static_cast<unsigned>(int64_t(a.tiles_x) * a.tiles_y * ((inz + a.zlen - 1) / a.zlen));
}

}  // namespace

int leap2_variant_count() { return kNumLeap2; }
const char* leap2_variant_name(int v) { return (v >= 0 && v < kNumLeap2) ? kLeap2[v].name : nullptr; }
PencilBoxes leap2_boxes(int v) {
    PencilBoxes b;
    b.halo_x = kLeap2[v].tx + 4 * R;
    b.halo_y = kLeap2[v].ty + 4 * R;
    b.tile_x = kLeap2[v].tx + 2 * R;
    b.tile_y = kLeap2[v].ty + 2 * R;
    b.aux_tma = true;
    return b;
}
int leap2_resident(int v) { return kLeap2[v].resident(); }
void leap2_prepare() {
    for (int v = 0; v < kNumLeap2; ++v) kLeap2[v].resident();
}
int64_t leap2_ctas(int v, const GridDesc& g, int zchunks) {
    return leap2_ctas_of(leap2_args(v, g, zchunks, nullptr), g);
}

cudaError_t launch_leap2_f32(const PencilMaps& maps, float* out1, float* out2, const GridDesc& g,
                             const SourceDesc& src, float w1, const PencilConfig& cfg, int* err,
                             cudaStream_t stream) {
    if (!g.has_interior()) return cudaSuccess;
    Leap2Args a = leap2_args(cfg.variant, g, cfg.zchunks, err);
    a.out1 = out1;
    a.out2 = out2;
    a.dt2 = g.dt * g.dt;
    a.w = fold_weights(g, a.dt2);
    if (src.idx >= 0) {
        a.src_x = static_cast<int>(src.idx % g.nx);
        a.src_y = static_cast<int>((src.idx / g.nx) % g.ny);
        a.src_z = static_cast<int>(src.idx / (g.nx * g.ny));
        a.src_w0 = src.w;
        a.src_w1 = w1;
        a.src_wavelet = src.wavelet;
        a.src_step = src.step;
        a.src_off = src.step_offset;
        a.trace = src.trace;
    }
    return kLeap2[cfg.variant].launch(maps, a, leap2_ctas_of(a, g), stream);
}

}  // namespace sb200
