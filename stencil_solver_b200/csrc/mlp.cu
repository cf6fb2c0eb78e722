// Learned coarse correction: a per-point MLP 26 -> 32 -> 32 -> 1 (ReLU) on BF16
// tensor-core mma with FP32 accumulation, and the kernels that train it.
//
// No reference counterpart.  A coarse grid (2x the spacing, 2x the time step)
// advanced by the plain acoustic step is corrected after every step by
//   p_next[i] += s_i * c * MLP(f_i),   c a fixed output scale (the training
// targets' RMS, so the network itself works on O(1) values),
// where f_i is the 25-point star of p around i (in a difference basis, see
// feature_row in mlp_device.cuh) divided by s_i, the smallest power of two
// above its largest magnitude, plus the local Courant number sqrt(vel2) dt / dx,
// padded to 32 features.  The correction is positively homogeneous in p under
// power-of-two scalings of the field.
//
// Parameters: FP32 masters [W1 (32x32, out x in; input columns 26..31 stay 0),
// b1, W2 (32x32), b2, w3 (32), b3] and BF16 copies of W1, W2 and W2^T that the
// mma kernels read.  Forward: x (BF16) -> h1 = relu(W1 x + b1) (FP32, rounded
// to BF16 as the next A operand) -> h2 = relu(W2 h1 + b2) (FP32) ->
// y = w3 . h2 + b3 (FP32).  Backward of mean((y - t)^2) with the same BF16
// operands: dW2 = dh2^T h1, dh1 = dh2 W2, dW1 = dh1^T x as mma over the batch;
// dW3, biases and the loss in FP32.  Adam keeps FP32 moments.
//
// Tensor-core fragments (mma.sync.m16n8k16, row.col, bf16 -> f32): a warp owns
// 16 rows (samples).  The accumulator fragment of one layer (rows g, g+8; cols
// 8t + 2q, +1 for n-tile t, g = lane / 4, q = lane % 4) is exactly the A
// fragment of the next layer's k-step t / 2, so activations never leave the
// registers in the forward pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "dispatch.h"
#include "kernels.h"
#include "mlp_device.cuh"
#include "sb200_common.cuh"
#include "stencil_b200.h"

namespace sb200 {
namespace {

using namespace mlp;

static_assert(NPARAM == SB200_MLP_NPARAM, "parameter count");

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4],
                                         const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Per-warp copy of the network: B fragments of W1 and W2 for every (n-tile,
// k-step), and this lane's bias / w3 columns.
struct NetFrag {
    uint32_t w1[4][2][2];
    uint32_t w2[4][2][2];
    float b1[4][2], b2[4][2], w3[4][2];
    float b3;
};

__device__ __forceinline__ void load_net(NetFrag& n, const float* __restrict__ prm,
                                         const uint32_t* __restrict__ w1b,
                                         const uint32_t* __restrict__ w2b) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            // B(k, n) = W(n, k): row n = 8t + g of W, k = 16 ks + 2q (+8)
            const int w = (8 * t + g) * (F / 2) + 8 * ks + q;
            n.w1[t][ks][0] = w1b[w];
            n.w1[t][ks][1] = w1b[w + 4];
            n.w2[t][ks][0] = w2b[w];
            n.w2[t][ks][1] = w2b[w + 4];
        }
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int c = 8 * t + 2 * q + e;
            n.b1[t][e] = prm[OFF_B1 + c];
            n.b2[t][e] = prm[OFF_B2 + c];
            n.w3[t][e] = prm[OFF_W3 + c];
        }
    }
    n.b3 = prm[OFF_B3];
}

// Activations of one 16-row tile, kept for the backward pass.
struct Acts {
    float h1[4][4];     // relu(W1 x + b1), accumulator layout
    uint32_t a2[2][4];  // h1 as BF16 A fragments of layer 2
    float h2[4][4];     // relu(W2 h1 + b2)
    float y[2];         // outputs of rows g and g + 8
};

// x: A fragments of the tile's features (2 k-steps).
__device__ __forceinline__ void forward_tile(const NetFrag& n, const uint32_t (&x)[2][4], Acts& s) {
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        float d[4] = {n.b1[t][0], n.b1[t][1], n.b1[t][0], n.b1[t][1]};
        mma16816(d, x[0], n.w1[t][0]);
        mma16816(d, x[1], n.w1[t][1]);
#pragma unroll
        for (int e = 0; e < 4; ++e) s.h1[t][e] = fmaxf(d[e], 0.f);
    }
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
        s.a2[kk][0] = pack_bf2(s.h1[2 * kk][0], s.h1[2 * kk][1]);
        s.a2[kk][1] = pack_bf2(s.h1[2 * kk][2], s.h1[2 * kk][3]);
        s.a2[kk][2] = pack_bf2(s.h1[2 * kk + 1][0], s.h1[2 * kk + 1][1]);
        s.a2[kk][3] = pack_bf2(s.h1[2 * kk + 1][2], s.h1[2 * kk + 1][3]);
    }
    float y0 = 0.f, y1 = 0.f;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        float d[4] = {n.b2[t][0], n.b2[t][1], n.b2[t][0], n.b2[t][1]};
        mma16816(d, s.a2[0], n.w2[t][0]);
        mma16816(d, s.a2[1], n.w2[t][1]);
#pragma unroll
        for (int e = 0; e < 4; ++e) s.h2[t][e] = fmaxf(d[e], 0.f);
        y0 = fmaf(n.w3[t][0], s.h2[t][0], fmaf(n.w3[t][1], s.h2[t][1], y0));
        y1 = fmaf(n.w3[t][0], s.h2[t][2], fmaf(n.w3[t][1], s.h2[t][3], y1));
    }
    y0 += __shfl_xor_sync(0xffffffffu, y0, 1);
    y0 += __shfl_xor_sync(0xffffffffu, y0, 2);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 1);
    y1 += __shfl_xor_sync(0xffffffffu, y1, 2);
    s.y[0] = y0 + n.b3;
    s.y[1] = y1 + n.b3;
}

// A fragments of rows [r0, r0+16) of a row-major BF16 feature matrix (32 per
// row); rows at or beyond n read as zero.
__device__ __forceinline__ void load_x(uint32_t (&x)[2][4], const uint32_t* __restrict__ X,
                                       int64_t r0, int64_t n) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const int64_t ra = r0 + g, rb = r0 + g + 8;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
        x[ks][0] = ra < n ? X[ra * 16 + 8 * ks + q] : 0u;
        x[ks][1] = rb < n ? X[rb * 16 + 8 * ks + q] : 0u;
        x[ks][2] = ra < n ? X[ra * 16 + 8 * ks + 4 + q] : 0u;
        x[ks][3] = rb < n ? X[rb * 16 + 8 * ks + 4 + q] : 0u;
    }
}

constexpr int kWarps = 4;  // warps per block of the training kernels

__global__ void __launch_bounds__(32 * kWarps)
    mlp_forward_kernel(const float* __restrict__ prm, const uint32_t* __restrict__ w1b,
                       const uint32_t* __restrict__ w2b, const uint32_t* __restrict__ X,
                       float* __restrict__ y, int64_t n) {
    NetFrag net;
    load_net(net, prm, w1b, w2b);
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r0 = warp * 16; r0 < n; r0 += nw * 16) {
        uint32_t x[2][4];
        load_x(x, X, r0, n);
        Acts s;
        forward_tile(net, x, s);
        if (q == 0) {
            if (r0 + g < n) y[r0 + g] = s.y[0];
            if (r0 + g + 8 < n) y[r0 + g + 8] = s.y[1];
        }
    }
}

// Per-warp scratch for the transposes the weight-gradient mma need: rows of
// 16 samples, padded to 24 halves (48 bytes) so fragment loads hit distinct banks.
constexpr int TP = 24;
struct WarpT {
    uint16_t dh2[H][TP];  // dh2^T: [output unit][sample]
    uint16_t h1[H][TP];   // h1^T
    uint16_t dh1[H][TP];  // dh1^T
    uint16_t x[F][TP];    // x^T
};

__device__ __forceinline__ uint32_t ld_pair(const uint16_t* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}

// Gradient of sum over rows of (y - t)^2 * inv_n (the caller passes 1 / n_total),
// accumulated into grad[NPARAM] (and the loss into grad[NPARAM]).
__global__ void __launch_bounds__(32 * kWarps)
    mlp_grad_kernel(const float* __restrict__ prm, const uint32_t* __restrict__ w1b,
                    const uint32_t* __restrict__ w2b, const uint32_t* __restrict__ w2tb,
                    const uint32_t* __restrict__ X, const float* __restrict__ tgt, int64_t n,
                    float inv_n, float* __restrict__ grad) {
    __shared__ WarpT wt[kWarps];
    __shared__ float red[NSLOT];
    for (int i = threadIdx.x; i < NSLOT; i += blockDim.x) red[i] = 0.f;

    NetFrag net;
    load_net(net, prm, w1b, w2b);
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3, wi = threadIdx.x >> 5;
    WarpT& T = wt[wi];
    // W2^T as B fragments of dh1 = dh2 W2 (k = output unit o, n = input unit i).
    uint32_t w2t[4][2][2];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
            const int w = (8 * t + g) * (H / 2) + 8 * ks + q;
            w2t[t][ks][0] = w2tb[w];
            w2t[t][ks][1] = w2tb[w + 4];
        }

    float gw1[2][4][4], gw2[2][4][4];  // [m-tile of out units][n-tile][frag]
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int e = 0; e < 4; ++e) gw1[m][t][e] = gw2[m][t][e] = 0.f;
    float gb1[4][2] = {}, gb2[4][2] = {}, gw3[4][2] = {};
    float gb3 = 0.f, loss = 0.f;

    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t r0 = warp * 16; r0 < n; r0 += nw * 16) {
        uint32_t x[2][4];
        load_x(x, X, r0, n);
        Acts s;
        forward_tile(net, x, s);
        float dy[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t r = r0 + g + 8 * h;
            const float e = r < n ? s.y[h] - tgt[r] : 0.f;
            dy[h] = 2.f * e * inv_n;
            if (q == 0) {
                loss = fmaf(e * inv_n, e, loss);
                gb3 += dy[h];
            }
        }
        // dh2 = dy w3 [h2 > 0]; dW3, db2 rows partial sums.
        float dh2[4][4];
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int h = e >> 1, c = e & 1;
                gw3[t][c] = fmaf(dy[h], s.h2[t][e], gw3[t][c]);
                dh2[t][e] = s.h2[t][e] > 0.f ? dy[h] * net.w3[t][c] : 0.f;
                gb2[t][c] += dh2[t][e];
            }
        // Transposes for the weight-gradient mma: dh2^T, h1^T (BF16 as used), x^T.
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int row = g + 8 * (e >> 1), col = 8 * t + 2 * q + (e & 1);
                T.dh2[col][row] = bf16_bits(dh2[t][e]);
            }
#pragma unroll
        for (int kk = 0; kk < 2; ++kk)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                // a2[kk][r]: rows g (+8 for r odd), cols 16 kk + 2q (+8 for r >= 2)
                const int row = g + 8 * (r & 1), col = 16 * kk + 2 * q + 8 * (r >> 1);
                T.h1[col][row] = static_cast<uint16_t>(s.a2[kk][r] & 0xffffu);
                T.h1[col + 1][row] = static_cast<uint16_t>(s.a2[kk][r] >> 16);
                T.x[col][row] = static_cast<uint16_t>(x[kk][r] & 0xffffu);
                T.x[col + 1][row] = static_cast<uint16_t>(x[kk][r] >> 16);
            }
        __syncwarp();
        // dW2[o][i] += sum_r dh2[r][o] h1[r][i]: A = dh2^T (o x r), B = h1 (r x i).
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            uint32_t a[4];
            a[0] = ld_pair(&T.dh2[16 * m + g][2 * q]);
            a[1] = ld_pair(&T.dh2[16 * m + g + 8][2 * q]);
            a[2] = ld_pair(&T.dh2[16 * m + g][2 * q + 8]);
            a[3] = ld_pair(&T.dh2[16 * m + g + 8][2 * q + 8]);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const uint32_t b[2] = {ld_pair(&T.h1[8 * t + g][2 * q]),
                                       ld_pair(&T.h1[8 * t + g][2 * q + 8])};
                mma16816(gw2[m][t], a, b);
            }
        }
        // dh1 = (dh2 W2) [h1 > 0]: A = dh2 (accumulator layout -> A), B = W2^T frags.
        uint32_t ad[2][4];
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            ad[kk][0] = pack_bf2(dh2[2 * kk][0], dh2[2 * kk][1]);
            ad[kk][1] = pack_bf2(dh2[2 * kk][2], dh2[2 * kk][3]);
            ad[kk][2] = pack_bf2(dh2[2 * kk + 1][0], dh2[2 * kk + 1][1]);
            ad[kk][3] = pack_bf2(dh2[2 * kk + 1][2], dh2[2 * kk + 1][3]);
        }
        float dh1[4][4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            mma16816(d, ad[0], w2t[t][0]);
            mma16816(d, ad[1], w2t[t][1]);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                dh1[t][e] = s.h1[t][e] > 0.f ? d[e] : 0.f;
                gb1[t][e & 1] += dh1[t][e];
                const int row = g + 8 * (e >> 1), col = 8 * t + 2 * q + (e & 1);
                T.dh1[col][row] = bf16_bits(dh1[t][e]);
            }
        }
        __syncwarp();
        // dW1[o][f] += sum_r dh1[r][o] x[r][f].
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            uint32_t a[4];
            a[0] = ld_pair(&T.dh1[16 * m + g][2 * q]);
            a[1] = ld_pair(&T.dh1[16 * m + g + 8][2 * q]);
            a[2] = ld_pair(&T.dh1[16 * m + g][2 * q + 8]);
            a[3] = ld_pair(&T.dh1[16 * m + g + 8][2 * q + 8]);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const uint32_t b[2] = {ld_pair(&T.x[8 * t + g][2 * q]),
                                       ld_pair(&T.x[8 * t + g][2 * q + 8])};
                mma16816(gw1[m][t], a, b);
            }
        }
        __syncwarp();  // the transposes are rewritten by the next tile
    }

    // Block reduction in shared memory, then one global add per parameter.
    __syncthreads();
#pragma unroll
    for (int m = 0; m < 2; ++m)
#pragma unroll
        for (int t = 0; t < 4; ++t)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int o = 16 * m + g + 8 * (e >> 1), i = 8 * t + 2 * q + (e & 1);
                atomicAdd(&red[OFF_W1 + o * F + i], gw1[m][t][e]);
                atomicAdd(&red[OFF_W2 + o * H + i], gw2[m][t][e]);
            }
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int col = 8 * t + 2 * q + c;
            atomicAdd(&red[OFF_B1 + col], gb1[t][c]);
            atomicAdd(&red[OFF_B2 + col], gb2[t][c]);
            atomicAdd(&red[OFF_W3 + col], gw3[t][c]);
        }
    if (q == 0) {
        atomicAdd(&red[OFF_B3], gb3);
        atomicAdd(&red[NPARAM], loss);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < NSLOT; i += blockDim.x)
        if (red[i] != 0.f) atomicAdd(&grad[i], red[i]);
}

// Adam on the FP32 masters (one thread per parameter; input columns 26..31 of
// W1 never move).
__global__ void mlp_adam_kernel(float* __restrict__ prm, float* __restrict__ m1,
                                float* __restrict__ m2, const float* __restrict__ grad, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    if (i < OFF_B1 && (i % F) >= NIN) return;
    const float gr = grad[i];
    const float a = b1 * m1[i] + (1.f - b1) * gr;
    const float v = b2 * m2[i] + (1.f - b2) * gr * gr;
    m1[i] = a;
    m2[i] = v;
    prm[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// BF16 copies of W1, W2 and W2^T read by the mma kernels.
__global__ void mlp_bf16_kernel(const float* __restrict__ prm, uint16_t* __restrict__ w1b,
                                uint16_t* __restrict__ w2b, uint16_t* __restrict__ w2tb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= H * F) return;
    w1b[i] = bf16_bits(prm[OFF_W1 + i]);
    const uint16_t v = bf16_bits(prm[OFF_W2 + i]);
    w2b[i] = v;
    w2tb[(i % H) * H + i / H] = v;
}

// ── features ──────────────────────────────────────────────────────────────────

__global__ void mlp_samples_kernel(const float* __restrict__ p, const float* __restrict__ vel2,
                                   const float* __restrict__ p_true,
                                   const float* __restrict__ p_plain, int64_t nx, int64_t ny,
                                   float dt_over_dx, const int64_t* __restrict__ cells, int64_t n,
                                   uint32_t* __restrict__ X, float* __restrict__ t) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t c = cells[i];
    Star st;
    gather_star(st, p, c, nx, nx * ny);
    feature_row(X + i * 16, st, sqrtf(vel2[c]) * dt_over_dx);
    t[i] = st.s > 0.f ? (p_true[c] - p_plain[c]) / st.s : 0.f;
}

__global__ void restrict2_kernel(const float* __restrict__ fine, int64_t fnx, int64_t fny,
                                 int64_t fnz, float* __restrict__ coarse, int64_t nx, int64_t ny,
                                 int64_t nz, int off) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nx * ny * nz) return;
    const int64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
    float v = 0.f;
    if (x >= 4 && y >= 4 && z >= 4 && x < nx - 4 && y < ny - 4 && z < nz - 4) {
        const int64_t fx = 2 * x + off, fy = 2 * y + off, fz = 2 * z + off;
        if (fx >= 0 && fy >= 0 && fz >= 0 && fx < fnx && fy < fny && fz < fnz)
            v = fine[(fz * fny + fy) * fnx + fx];
    }
    coarse[i] = v;
}

// field[box] += scale * pattern over a bx x by x bz box at (x0, y0, z0) (a
// spatially extended source); cells outside the grid's interior are skipped.
__global__ void add_box_kernel(float* __restrict__ f, int64_t nx, int64_t ny, int64_t nz, int x0,
                               int y0, int z0, int bx, int by, int bz,
                               const float* __restrict__ pattern, float scale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bx * by * bz) return;
    const int64_t x = x0 + i % bx, y = y0 + (i / bx) % by, z = z0 + i / (bx * by);
    if (x < 4 || y < 4 || z < 4 || x >= nx - 4 || y >= ny - 4 || z >= nz - 4) return;
    f[(z * ny + y) * nx + x] += scale * pattern[i];
}

// Fused correction: each warp takes 32 consecutive interior points of a row,
// lanes build their feature rows in shared memory, two 16-row mma tiles run
// the network, and p_next += s * c * y.
constexpr int CP = 40;  // feature row stride in shared memory (halves): conflict-free A loads
constexpr int kCorrWarps = 8;

__global__ void __launch_bounds__(32 * kCorrWarps)
    mlp_correct_kernel(const float* __restrict__ prm, const uint32_t* __restrict__ w1b,
                       const uint32_t* __restrict__ w2b, const float* __restrict__ p,
                       const float* __restrict__ vel2, float* __restrict__ p_next, int64_t nx,
                       int64_t ny, int64_t nz, float dt_over_dx, float out_scale, float floor) {
    __shared__ __align__(16) uint16_t feat[kCorrWarps][32][CP];
    __shared__ float scale[kCorrWarps][32];
    NetFrag net;
    load_net(net, prm, w1b, w2b);
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3, wi = threadIdx.x >> 5;
    const int64_t ix = nx - 8, segs = (ix + 31) / 32;
    const int64_t items = segs * (ny - 8) * (nz - 8);
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int64_t sy = nx, sz = nx * ny;
    for (int64_t it = warp; it < items; it += nw) {
        const int64_t seg = it % segs, row = it / segs;
        const int64_t y = 4 + row % (ny - 8), z = 4 + row / (ny - 8);
        const int64_t x = 4 + seg * 32 + lane;
        const bool live = x < nx - 4;
        const int64_t c = (z * ny + y) * nx + x;
        uint32_t* fr = reinterpret_cast<uint32_t*>(&feat[wi][lane][0]);
        float s = 0.f;
        if (live) {
            Star st;
            gather_star(st, p, c, sy, sz, floor);
            feature_row(fr, st, sqrtf(vel2[c]) * dt_over_dx);
            s = st.s;
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) fr[j] = 0u;
        }
        scale[wi][lane] = s * out_scale;
        __syncwarp();
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            uint32_t xa[2][4];
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                xa[ks][0] = ld_pair(&feat[wi][16 * m + g][16 * ks + 2 * q]);
                xa[ks][1] = ld_pair(&feat[wi][16 * m + g + 8][16 * ks + 2 * q]);
                xa[ks][2] = ld_pair(&feat[wi][16 * m + g][16 * ks + 8 + 2 * q]);
                xa[ks][3] = ld_pair(&feat[wi][16 * m + g + 8][16 * ks + 8 + 2 * q]);
            }
            Acts a;
            forward_tile(net, xa, a);
            if (q < 2) {  // lane q = 0 writes row g, q = 1 row g + 8
                const int r = 16 * m + g + 8 * q;
                const int64_t xr = 4 + seg * 32 + r;
                const float sr = scale[wi][r];
                if (xr < nx - 4 && sr > 0.f) {
                    const int64_t cr = (z * ny + y) * nx + xr;
                    p_next[cr] = fmaf(sr, q == 0 ? a.y[0] : a.y[1], p_next[cr]);
                }
            }
        }
        __syncwarp();
    }
}

// ── tcgen05 correction ───────────────────────────────────────────────────────
// The same correction on the 5th-generation tensor cores: a CTA of 128 threads
// takes tiles of 128 points (4 row segments of 32), writes their feature rows
// to shared memory, and one thread issues tcgen05.mma (M = 128, N = 32,
// K = 16, BF16 operands from shared memory, FP32 accumulator in TMEM): two per
// layer.  Each thread then owns one point (one TMEM lane): tcgen05.ld of its 32
// accumulator columns, bias + ReLU + BF16 for layer 2's A operand, and the
// final 32-term dot product with w3 in FP32.
constexpr int kTcThreads = 128;
constexpr uint32_t kTcCols = 64;  // TMEM columns: layer 1 in 0..31, layer 2 in 32..63
// Dynamic shared memory requested per CTA (20.5 KB of tiles + alignment): at
// most 8 CTAs then fit on one SM, 8 x 64 = 512 TMEM columns, so tcgen05.alloc
// never waits for another CTA.
constexpr int kTcSmem = 26 * 1024;
__global__ void __launch_bounds__(kTcThreads)
    mlp_correct_tc_kernel(const float* __restrict__ prm, const uint16_t* __restrict__ w1b,
                          const uint16_t* __restrict__ w2b, const float* __restrict__ p,
                          const float* __restrict__ vel2, float* __restrict__ p_next, int nx,
                          int ny, int nz, float dt_over_dx, float out_scale, float floor,
                          int* err) {
    extern __shared__ unsigned char dyn[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t s_tmem;
    __shared__ int s_flag;  // 1: the last MMA wait gave up
    __shared__ __align__(16) float sb1[H], sb2[H], sw3[H];
    unsigned char* base = smem_align<1024>(dyn);
    unsigned char* sA = base;            // 128 x 32 BF16 features
    unsigned char* sA2 = base + 8192;    // 128 x 32 BF16 h1
    unsigned char* sW1 = base + 16384;   // 32 x 32 BF16
    unsigned char* sW2 = base + 18432;   // 32 x 32 BF16
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < H * F; i += kTcThreads) {
        *reinterpret_cast<uint16_t*>(sW1 + core_off(i / F, i % F)) = w1b[i];
        *reinterpret_cast<uint16_t*>(sW2 + core_off(i / H, i % H)) = w2b[i];
    }
    if (tid < H) {
        sb1[tid] = prm[OFF_B1 + tid];
        sb2[tid] = prm[OFF_B2 + tid];
        sw3[tid] = prm[OFF_W3 + tid];
    }
    const float b3 = prm[OFF_B3];
    if (tid == 0) {
        mbar_init(&mbar, 1);
        fence_barrier_init();
        s_flag = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&s_tmem)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t lane_base = tmem + (uint32_t(32 * warp) << 16);
    const uint32_t aA = smem_u32(sA), aA2 = smem_u32(sA2), aW1 = smem_u32(sW1),
                   aW2 = smem_u32(sW2);

    // Work: 32-point segments of interior rows, 4 per tile (one per warp).
    const unsigned segs = unsigned(nx - 8 + 31) / 32u, rows_y = unsigned(ny - 8);
    const unsigned items = segs * rows_y * unsigned(nz - 8);
    const unsigned tiles = (items + 3u) / 4u;
    const int64_t sy = nx, sz = int64_t(nx) * ny;
    int issued = 0, completed = 0;  // thread 0: commits issued / seen complete
    bool abort_run = false;
    // One thread waits for the MMAs; the others meet it at the barrier that
    // follows (no spinning warps).
    auto wait_mma = [&](uint32_t parity) {
        if (tid == 0) {
            if (mbar_wait(&mbar, parity))
                completed = issued;
            else
                s_flag = 1;
        }
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        return s_flag == 0;
    };
    for (unsigned tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const unsigned item = tile * 4u + unsigned(warp);
        int64_t c = 0;
        float sc = 0.f;
        uint32_t fr[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) fr[j] = 0u;
        if (item < items) {
            const unsigned seg = item % segs, row = item / segs;
            const int y = 4 + int(row % rows_y), z = 4 + int(row / rows_y);
            const int x = 4 + int(seg) * 32 + lane;
            if (x < nx - 4) {
                c = (int64_t(z) * ny + y) * nx + x;
                Star st;
                gather_star(st, p, c, sy, sz, floor);
                feature_row(fr, st, sqrtf(vel2[c]) * dt_over_dx);
                sc = st.s * out_scale;
            }
        }
        store_row(sA, tid, fr);
        fence_async_smem();
        // A tile whose points are all exactly zero has a zero correction: skip it.
        if (__syncthreads_or(sc > 0.f) == 0) continue;
        if (tid == 0) {
            tc_fence_after();
            tc_mma(tmem, umma_desc(aA), umma_desc(aW1), 0u);
            tc_mma(tmem, umma_desc(aA + 256), umma_desc(aW1 + 256), 1u);
            tc_commit(&mbar);
            ++issued;
        }
        if (!wait_mma(0)) {
            abort_run = true;
            break;
        }
        float d[32];
        tc_ld32(lane_base, d);
        uint32_t h[16];
#pragma unroll
        for (int q4 = 0; q4 < 8; ++q4) {
            const float4 bb = *reinterpret_cast<const float4*>(&sb1[4 * q4]);
            const float2 u = add2(make_float2(d[4 * q4], d[4 * q4 + 1]), make_float2(bb.x, bb.y));
            const float2 v = add2(make_float2(d[4 * q4 + 2], d[4 * q4 + 3]), make_float2(bb.z, bb.w));
            h[2 * q4] = relu_bf2(u.x, u.y);
            h[2 * q4 + 1] = relu_bf2(v.x, v.y);
        }
        store_row(sA2, tid, h);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            tc_mma(tmem + 32, umma_desc(aA2), umma_desc(aW2), 0u);
            tc_mma(tmem + 32, umma_desc(aA2 + 256), umma_desc(aW2 + 256), 1u);
            tc_commit(&mbar);
            ++issued;
        }
        if (!wait_mma(1)) {
            abort_run = true;
            break;
        }
        tc_ld32(lane_base + 32, d);
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int q4 = 0; q4 < 8; ++q4) {
            const float4 bb = *reinterpret_cast<const float4*>(&sb2[4 * q4]);
            const float4 ww = *reinterpret_cast<const float4*>(&sw3[4 * q4]);
            const float2 u = add2(make_float2(d[4 * q4], d[4 * q4 + 1]), make_float2(bb.x, bb.y));
            const float2 v = add2(make_float2(d[4 * q4 + 2], d[4 * q4 + 3]), make_float2(bb.z, bb.w));
            acc = fma2(make_float2(ww.x, ww.y), make_float2(fmaxf(u.x, 0.f), fmaxf(u.y, 0.f)), acc);
            acc = fma2(make_float2(ww.z, ww.w), make_float2(fmaxf(v.x, 0.f), fmaxf(v.y, 0.f)), acc);
        }
        const float yv = (acc.x + acc.y) + b3;
        if (sc > 0.f) p_next[c] = fmaf(sc, yv, p_next[c]);
        tc_fence_before();
    }
    if (abort_run && tid == 0) {
        record_error(err, kDevWaitTimeout);
        // Let the MMAs still in flight finish (bounded) before TMEM is released.
        for (int k = completed; k < issued; ++k) (void)mbar_wait(&mbar, k & 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTcCols)
                     : "memory");
}

// One axis of a separable Gaussian blur (clamp-to-edge): out = sum_k w[k] in[i + k - r]
// along `axis` (0 = x, 1 = y, 2 = z).
constexpr int kBlurMaxR = 48;
struct BlurWeights {
    float w[2 * kBlurMaxR + 1];
};

__global__ void blur_axis_kernel(const float* __restrict__ in, float* __restrict__ out, int64_t nx,
                                 int64_t ny, int64_t nz, int axis, const BlurWeights bw, int r) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nx * ny * nz) return;
    const int64_t x = i % nx, y = (i / nx) % ny, z = i / (nx * ny);
    const int64_t n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const int64_t pos = axis == 0 ? x : (axis == 1 ? y : z);
    const int64_t stride = axis == 0 ? 1 : (axis == 1 ? nx : nx * ny);
    float acc = 0.f;
    for (int k = -r; k <= r; ++k) {
        const int64_t j = min(max(pos + k, int64_t(0)), n - 1);
        acc = fmaf(bw.w[k + r], in[i + (j - pos) * stride], acc);
    }
    out[i] = acc;
}

// ── host side ────────────────────────────────────────────────────────────────

struct Mlp {
    float* prm = nullptr;  // NPARAM FP32 masters
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* grad = nullptr;  // NSLOT (gradients + loss)
    uint16_t* w1b = nullptr;
    uint16_t* w2b = nullptr;
    uint16_t* w2tb = nullptr;
    int64_t adam_t = 0;
    int sms = 148;
    float out_scale = 1.f;  // the correction is s * out_scale * y
    float min_scale = 0.f;  // correction floor: stars below it get no correction
    int kernel = 0;         // correction kernel: 0 = tcgen05, 1 = mma.sync
    // Host copy of the FP32 parameters for the fused step, which takes biases
    // and w3 by value; stale after a device-side update (train_step).
    std::vector<float> host;
    bool host_valid = false;
};

int cuda_err(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return SB200_OK;
    return set_error(SB200_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

void init_params(std::vector<float>& w, uint64_t seed) {
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    w.assign(NPARAM, 0.f);
    for (int o = 0; o < H; ++o)
        for (int i = 0; i < NIN; ++i)
            w[OFF_W1 + o * F + i] = static_cast<float>(nd(rng) * std::sqrt(2.0 / NIN));
    for (int o = 0; o < H; ++o)
        for (int i = 0; i < H; ++i)
            w[OFF_W2 + o * H + i] = static_cast<float>(nd(rng) * std::sqrt(2.0 / H));
    for (int i = 0; i < H; ++i) w[OFF_W3 + i] = static_cast<float>(nd(rng) * 0.1 / std::sqrt(H));
}

int grid_blocks(const Mlp& m, int64_t work_units_per_block, int64_t units) {
    const int64_t want = (units + work_units_per_block - 1) / work_units_per_block;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(m.sms) * 8)));
}

}  // namespace
}  // namespace sb200

using namespace sb200;

extern "C" {

int sb200_mlp_create(uint64_t seed, void** handle) {
    if (!handle) return set_error(SB200_ERR_INVALID, "sb200_mlp_create: NULL handle");
    *handle = nullptr;
    Mlp* m = new Mlp();
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    int rc = cuda_err(cudaMalloc(&m->prm, NPARAM * 4), "sb200_mlp_create");
    if (!rc) rc = cuda_err(cudaMalloc(&m->m1, NPARAM * 4), "sb200_mlp_create");
    if (!rc) rc = cuda_err(cudaMalloc(&m->m2, NPARAM * 4), "sb200_mlp_create");
    if (!rc) rc = cuda_err(cudaMalloc(&m->grad, NSLOT * 4), "sb200_mlp_create");
    if (!rc) rc = cuda_err(cudaMalloc(&m->w1b, H * F * 2), "sb200_mlp_create");
    if (!rc) rc = cuda_err(cudaMalloc(&m->w2b, H * H * 2), "sb200_mlp_create");
    if (!rc) rc = cuda_err(cudaMalloc(&m->w2tb, H * H * 2), "sb200_mlp_create");
    if (rc) {
        sb200_mlp_destroy(m);
        return rc;
    }
    *handle = m;
    std::vector<float> w;
    init_params(w, seed);
    return sb200_mlp_set_params(m, w.data());
}

int sb200_mlp_destroy(void* h) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m) return SB200_OK;
    for (void* p : {static_cast<void*>(m->prm), static_cast<void*>(m->m1),
                    static_cast<void*>(m->m2), static_cast<void*>(m->grad),
                    static_cast<void*>(m->w1b), static_cast<void*>(m->w2b),
                    static_cast<void*>(m->w2tb)})
        if (p) cudaFree(p);
    delete m;
    return SB200_OK;
}

int sb200_mlp_set_params(void* h, const float* params) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !params) return set_error(SB200_ERR_INVALID, "sb200_mlp_set_params: NULL argument");
    std::vector<float> w(params, params + NPARAM);
    for (int o = 0; o < H; ++o)
        for (int i = NIN; i < F; ++i) w[OFF_W1 + o * F + i] = 0.f;  // padding inputs
    int rc = cuda_err(cudaMemcpy(m->prm, w.data(), NPARAM * 4, cudaMemcpyHostToDevice),
                      "sb200_mlp_set_params");
    m->host = w;
    m->host_valid = !rc;
    if (!rc) rc = cuda_err(cudaMemset(m->m1, 0, NPARAM * 4), "sb200_mlp_set_params");
    if (!rc) rc = cuda_err(cudaMemset(m->m2, 0, NPARAM * 4), "sb200_mlp_set_params");
    if (rc) return rc;
    m->adam_t = 0;
    mlp_bf16_kernel<<<(H * F + 255) / 256, 256>>>(m->prm, m->w1b, m->w2b, m->w2tb);
    rc = cuda_err(cudaGetLastError(), "sb200_mlp_set_params");
    if (!rc) rc = cuda_err(cudaDeviceSynchronize(), "sb200_mlp_set_params");
    return rc;
}

int sb200_mlp_get_params(void* h, float* params) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !params) return set_error(SB200_ERR_INVALID, "sb200_mlp_get_params: NULL argument");
    return cuda_err(cudaMemcpy(params, m->prm, NPARAM * 4, cudaMemcpyDeviceToHost),
                    "sb200_mlp_get_params");
}

int sb200_mlp_set_output_scale(void* h, float scale) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !(scale > 0.f) || !std::isfinite(scale))
        return set_error(SB200_ERR_INVALID, "sb200_mlp_set_output_scale: bad arguments");
    m->out_scale = scale;
    return SB200_OK;
}

int sb200_mlp_set_min_scale(void* h, float floor) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !(floor >= 0.f) || !std::isfinite(floor))
        return set_error(SB200_ERR_INVALID, "sb200_mlp_set_min_scale: bad arguments");
    m->min_scale = floor;
    return SB200_OK;
}

float sb200_mlp_min_scale(void* h) {
    Mlp* m = static_cast<Mlp*>(h);
    return m ? m->min_scale : 0.f;
}

float sb200_mlp_output_scale(void* h) {
    Mlp* m = static_cast<Mlp*>(h);
    return m ? m->out_scale : 0.f;
}

int sb200_mlp_forward(void* h, const uint16_t* X, float* y, int64_t n, void* stream) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !X || !y || n < 0) return set_error(SB200_ERR_INVALID, "sb200_mlp_forward: bad arguments");
    if (n == 0) return SB200_OK;
    const int blocks = grid_blocks(*m, 16 * kWarps, n);
    mlp_forward_kernel<<<blocks, 32 * kWarps, 0, static_cast<cudaStream_t>(stream)>>>(
        m->prm, reinterpret_cast<const uint32_t*>(m->w1b), reinterpret_cast<const uint32_t*>(m->w2b),
        reinterpret_cast<const uint32_t*>(X), y, n);
    return cuda_err(cudaGetLastError(), "sb200_mlp_forward");
}

int sb200_mlp_gradients(void* h, const uint16_t* X, const float* t, int64_t n, float* grad,
                        void* stream) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !X || !t || !grad || n <= 0)
        return set_error(SB200_ERR_INVALID, "sb200_mlp_gradients: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = cuda_err(cudaMemsetAsync(grad, 0, NSLOT * 4, st), "sb200_mlp_gradients");
    if (rc) return rc;
    const int blocks = grid_blocks(*m, 16 * kWarps * 4, n);
    mlp_grad_kernel<<<blocks, 32 * kWarps, 0, st>>>(
        m->prm, reinterpret_cast<const uint32_t*>(m->w1b), reinterpret_cast<const uint32_t*>(m->w2b),
        reinterpret_cast<const uint32_t*>(m->w2tb), reinterpret_cast<const uint32_t*>(X), t, n,
        1.f / static_cast<float>(n), grad);
    return cuda_err(cudaGetLastError(), "sb200_mlp_gradients");
}

int sb200_mlp_train_step(void* h, const uint16_t* X, const float* t, int64_t n, float lr,
                         float* loss, void* stream) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m) return set_error(SB200_ERR_INVALID, "sb200_mlp_train_step: NULL handle");
    if (!(lr > 0.f)) return set_error(SB200_ERR_INVALID, "sb200_mlp_train_step: lr must be positive");
    if (int rc = sb200_mlp_gradients(h, X, t, n, m->grad, stream)) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    m->host_valid = false;
    m->adam_t += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, float(m->adam_t)), c2 = 1.f - std::pow(b2, float(m->adam_t));
    mlp_adam_kernel<<<(NPARAM + 255) / 256, 256, 0, st>>>(m->prm, m->m1, m->m2, m->grad, lr, b1, b2,
                                                          1e-8f, c1, c2);
    int rc = cuda_err(cudaGetLastError(), "sb200_mlp_train_step");
    if (rc) return rc;
    mlp_bf16_kernel<<<(H * F + 255) / 256, 256, 0, st>>>(m->prm, m->w1b, m->w2b, m->w2tb);
    rc = cuda_err(cudaGetLastError(), "sb200_mlp_train_step");
    if (!rc && loss)
        rc = cuda_err(cudaMemcpyAsync(loss, m->grad + NPARAM, 4, cudaMemcpyDeviceToDevice, st),
                      "sb200_mlp_train_step");
    return rc;
}

int sb200_mlp_correct(void* h, const float* p, const float* vel2, float* p_next,
                      const sb200_grid* grid, void* stream) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !p || !vel2 || !p_next || !grid)
        return set_error(SB200_ERR_INVALID, "sb200_mlp_correct: NULL argument");
    if (p == p_next) return set_error(SB200_ERR_INVALID, "sb200_mlp_correct: p_next must not alias p");
    if (grid->nx <= 8 || grid->ny <= 8 || grid->nz <= 8) return SB200_OK;
    const float dx = std::min(grid->dx, std::min(grid->dy, grid->dz));
    const int64_t items = ((grid->nx - 8 + 31) / 32) * (grid->ny - 8) * (grid->nz - 8);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (m->kernel == 1) {
        const int blocks = grid_blocks(*m, kCorrWarps * 4, items);
        mlp_correct_kernel<<<blocks, 32 * kCorrWarps, 0, st>>>(
            m->prm, reinterpret_cast<const uint32_t*>(m->w1b),
            reinterpret_cast<const uint32_t*>(m->w2b), p, vel2, p_next, grid->nx, grid->ny,
            grid->nz, grid->dt / dx, m->out_scale, m->min_scale);
        return cuda_err(cudaGetLastError(), "sb200_mlp_correct");
    }
    int* err = device_error_word();
    if (!err) return set_error(SB200_ERR_CUDA, "sb200_mlp_correct: device error word unavailable");
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr[dev & 63]) {
        if (int rc = cuda_err(cudaFuncSetAttribute(mlp_correct_tc_kernel,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   kTcSmem),
                              "sb200_mlp_correct"))
            return rc;
        attr[dev & 63] = true;
    }
    if (items >= (int64_t(1) << 31) || grid->nx > (1 << 20) || grid->ny > (1 << 20))
        return set_error(SB200_ERR_UNSUPPORTED, "sb200_mlp_correct: grid too large");
    const int64_t tiles = (items + 3) / 4;
    const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(tiles, int64_t(m->sms) * 8)));
    mlp_correct_tc_kernel<<<blocks, kTcThreads, kTcSmem, st>>>(
        m->prm, m->w1b, m->w2b, p, vel2, p_next, static_cast<int>(grid->nx),
        static_cast<int>(grid->ny), static_cast<int>(grid->nz), grid->dt / dx, m->out_scale,
        m->min_scale, err);
    return cuda_err(cudaGetLastError(), "sb200_mlp_correct");
}

namespace {
GridDesc grid_desc(const sb200_grid& grid) {
    GridDesc g;
    g.nx = grid.nx;
    g.ny = grid.ny;
    g.nz = grid.nz;
    g.dx = grid.dx;
    g.dy = grid.dy;
    g.dz = grid.dz;
    g.dt = grid.dt;
    return g;
}

int learned_step_impl(void* h, const float* p, float* p_prev_next, const float* vel2,
                      const sb200_grid* grid, const uint8_t* flags_in, uint8_t* flags_out,
                      const int64_t* box, void* stream, const char* where) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !p || !p_prev_next || !vel2 || !grid)
        return set_error(SB200_ERR_INVALID, std::string(where) + ": NULL argument");
    if (p == p_prev_next)
        return set_error(SB200_ERR_INVALID, std::string(where) + ": p_next must not alias p");
    if (!(grid->dx > 0.f && grid->dy > 0.f && grid->dz > 0.f && grid->dt > 0.f) ||
        grid->nx < 0 || grid->ny < 0 || grid->nz < 0)
        return set_error(SB200_ERR_INVALID, std::string(where) + ": bad grid");
    const GridDesc g = grid_desc(*grid);
    if (!g.has_interior()) return SB200_OK;
    auto a16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    if (g.nx % 4 != 0 || !a16(p) || !a16(p_prev_next) || !a16(vel2) || g.nx > (1 << 20) ||
        g.ny > (1 << 20) || g.nz > (1 << 20))
        return set_error(SB200_ERR_UNSUPPORTED,
                         std::string(where) + ": needs nx % 4 == 0 and 16-byte aligned fields");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!m->host_valid) {  // parameters changed on the device since the last copy
        m->host.resize(NPARAM);
        int rc = cuda_err(cudaMemcpyAsync(m->host.data(), m->prm, NPARAM * 4,
                                          cudaMemcpyDeviceToHost, st),
                          where);
        if (!rc) rc = cuda_err(cudaStreamSynchronize(st), where);
        if (rc) return rc;
        m->host_valid = true;
    }
    int* err = device_error_word();
    if (!err) return set_error(SB200_ERR_CUDA, std::string(where) + ": device error word unavailable");
    const PencilBoxes b = learned_step_boxes();
    PencilMaps maps;
    int rc = tensor_map_3d(&maps.p, p, g.nx, g.ny, g.nz, 4, b.halo_x, b.halo_y);
    if (!rc) rc = tensor_map_3d(&maps.prev, p_prev_next, g.nx, g.ny, g.nz, 4, b.tile_x, b.tile_y);
    if (!rc) rc = tensor_map_3d(&maps.vel2, vel2, g.nx, g.ny, g.nz, 4, b.tile_x, b.tile_y);
    if (rc)
        return set_error(SB200_ERR_CUDA, std::string(where) + ": tensor map encode failed (" +
                                             std::to_string(rc) + ")");
    LearnedNet net;
    net.w1b = m->w1b;
    net.w2b = m->w2b;
    for (int k = 0; k < H; ++k) {
        net.b1[k] = m->host[OFF_B1 + k];
        net.b2[k] = m->host[OFF_B2 + k];
        net.w3[k] = m->host[OFF_W3 + k];
    }
    net.b3 = m->host[OFF_B3];
    net.out_scale = m->out_scale;
    net.min_scale = m->min_scale;
    return cuda_err(launch_learned_step(maps, p_prev_next, g, net, m->sms, err, st, flags_in,
                                        flags_out, box),
                    where);
}
}  // namespace

int sb200_mlp_learned_step(void* h, const float* p, float* p_prev_next, const float* vel2,
                           const sb200_grid* grid, void* stream) {
    return learned_step_impl(h, p, p_prev_next, vel2, grid, nullptr, nullptr, nullptr, stream,
                             "sb200_mlp_learned_step");
}

int64_t sb200_mlp_flags_bytes(void* h, const sb200_grid* grid) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !grid) return set_error(SB200_ERR_INVALID, "sb200_mlp_flags_bytes: NULL argument");
    const LearnedChunks c = learned_step_chunks(grid_desc(*grid), m->sms, true);
    return int64_t(c.tiles_x) * c.tiles_y * c.zchunks;
}

int sb200_mlp_learned_step_flags(void* h, const float* p, float* p_prev_next, const float* vel2,
                                 const sb200_grid* grid, const uint8_t* flags_in,
                                 uint8_t* flags_out, const int64_t* box, void* stream) {
    if (flags_in && flags_in == flags_out)
        return set_error(SB200_ERR_INVALID,
                         "sb200_mlp_learned_step_flags: flags_in and flags_out must differ");
    return learned_step_impl(h, p, p_prev_next, vel2, grid, flags_in, flags_out, box, stream,
                             "sb200_mlp_learned_step_flags");
}

int sb200_mlp_flags_compose(void* h, const sb200_grid* grid, const uint8_t* flags_p,
                            uint8_t* flags_r, void* stream) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || !grid || !flags_p || !flags_r || flags_p == flags_r)
        return set_error(SB200_ERR_INVALID, "sb200_mlp_flags_compose: bad arguments");
    return cuda_err(launch_flags_compose(flags_p, flags_r, grid_desc(*grid), m->sms,
                                         static_cast<cudaStream_t>(stream)),
                    "sb200_mlp_flags_compose");
}

int sb200_mlp_set_kernel(void* h, int kernel) {
    Mlp* m = static_cast<Mlp*>(h);
    if (!m || kernel < 0 || kernel > 1)
        return set_error(SB200_ERR_INVALID, "sb200_mlp_set_kernel: bad arguments");
    m->kernel = kernel;
    return SB200_OK;
}

int sb200_mlp_samples(const float* p, const float* vel2, const float* p_true, const float* p_plain,
                      const sb200_grid* grid, const int64_t* cells, int64_t n, uint16_t* X,
                      float* t, void* stream) {
    if (!p || !vel2 || !p_true || !p_plain || !grid || !cells || !X || !t || n < 0)
        return set_error(SB200_ERR_INVALID, "sb200_mlp_samples: bad arguments");
    if (n == 0) return SB200_OK;
    const float dx = std::min(grid->dx, std::min(grid->dy, grid->dz));
    mlp_samples_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0,
                         static_cast<cudaStream_t>(stream)>>>(
        p, vel2, p_true, p_plain, grid->nx, grid->ny, grid->dt / dx, cells, n,
        reinterpret_cast<uint32_t*>(X), t);
    return cuda_err(cudaGetLastError(), "sb200_mlp_samples");
}

int sb200_add_box(float* field, const sb200_grid* grid, int x0, int y0, int z0, int bx, int by,
                  int bz, const float* pattern, float scale, void* stream) {
    if (!field || !grid || !pattern || bx < 0 || by < 0 || bz < 0)
        return set_error(SB200_ERR_INVALID, "sb200_add_box: bad arguments");
    const int n = bx * by * bz;
    if (n == 0) return SB200_OK;
    add_box_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        field, grid->nx, grid->ny, grid->nz, x0, y0, z0, bx, by, bz, pattern, scale);
    return cuda_err(cudaGetLastError(), "sb200_add_box");
}

int sb200_smooth3(float* field, float* tmp, const sb200_grid* grid, float sigma_cells,
                  void* stream) {
    if (!field || !tmp || !grid || !(sigma_cells > 0.f) || sigma_cells > 16.f)
        return set_error(SB200_ERR_INVALID, "sb200_smooth3: need 0 < sigma_cells <= 16");
    const int r = std::max(1, std::min(kBlurMaxR, static_cast<int>(std::ceil(3.0f * sigma_cells))));
    BlurWeights bw{};
    double sum = 0.0;
    const double s2 = double(sigma_cells) * sigma_cells;
    for (int k = -r; k <= r; ++k) sum += std::exp(-0.5 * double(k) * k / s2);
    for (int k = -r; k <= r; ++k) bw.w[k + r] = static_cast<float>(std::exp(-0.5 * double(k) * k / s2) / sum);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = grid->nx * grid->ny * grid->nz;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    float* src = field;
    float* dst = tmp;
    int rc = SB200_OK;
    for (int axis = 0; axis < 3 && !rc; ++axis) {
        blur_axis_kernel<<<blocks, 256, 0, st>>>(src, dst, grid->nx, grid->ny, grid->nz, axis, bw, r);
        rc = cuda_err(cudaGetLastError(), "sb200_smooth3");
        std::swap(src, dst);
    }
    // three passes leave the result in tmp: copy it back
    if (!rc)
        rc = cuda_err(cudaMemcpyAsync(field, src, n * 4, cudaMemcpyDeviceToDevice, st), "sb200_smooth3");
    if (!rc) rc = cuda_err(cudaStreamSynchronize(st), "sb200_smooth3");
    return rc;
}

int sb200_restrict2(const float* fine, const sb200_grid* fine_grid, float* coarse,
                    const sb200_grid* coarse_grid, int offset, void* stream) {
    if (!fine || !fine_grid || !coarse || !coarse_grid)
        return set_error(SB200_ERR_INVALID, "sb200_restrict2: NULL argument");
    const int64_t n = coarse_grid->nx * coarse_grid->ny * coarse_grid->nz;
    if (n <= 0) return SB200_OK;
    restrict2_kernel<<<static_cast<unsigned>((n + 255) / 256), 256, 0,
                       static_cast<cudaStream_t>(stream)>>>(
        fine, fine_grid->nx, fine_grid->ny, fine_grid->nz, coarse, coarse_grid->nx,
        coarse_grid->ny, coarse_grid->nz, offset);
    return cuda_err(cudaGetLastError(), "sb200_restrict2");
}

}  // extern "C"
