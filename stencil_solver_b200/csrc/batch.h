// Internal interface of the batched-shots path (many independent acoustic grids
// advanced by one persistent launch per step): the per-shot descriptor the
// kernels read from device memory, the work queue they share, and the launchers.
// Device-side types; included from .cu files only.
#pragma once

#include "kernels.h"
#include "sb200_common.cuh"

namespace sb200 {

// Arguments of one FP32 pencil sweep over one grid (one launch of the single-grid
// kernel, or one shot of a batched launch).
struct PencilArgs {
    const float* prev;  // acoustic, AUX = 0: p at t-dt (may alias next)
    const float* vel2;  // acoustic, AUX = 0: v^2
    float* next;
    int nx, ny, nz;
    int64_t sy, sz;
    int tiles_x, tiles_y, zlen;
    Weights w;  // acoustic: weights * dt^2; heat: weights * alpha*dt
    float dt2;  // acoustic: dt^2 (source term)
    int src_x, src_y, src_z;  // -1 when there is no source
    float src_w;
    const float* src_wavelet;
    const int* src_step;
    int src_off;
    float* trace;
    int* err;
    float* prev_out;  // prepass: p_prev + 2 beta dt^2 v^2 lap p (in place over p_prev)
    float heat_c;     // heat: 1 + alpha*dt * (c0/dx^2 + c0/dy^2 + c0/dz^2), the centre's weight
};

// Work queue of a batched launch.  `next` hands out work items, `done` counts
// CTAs that found the queue empty; the last one resets both and advances `step`
// (the step index every shot's source and trace use).  Starts zeroed.
struct BatchQueue {
    int next;
    int done;
    int step;
    int pad;
};

// One shot of the FP32 batch, in device memory (tensor maps must be 64-byte
// aligned): p with the halo box, p_prev and vel2 with the tile box, and the
// sweep's arguments (next = prev: in-place leapfrog).
struct alignas(64) ShotF32 {
    CUtensorMap p, prev, vel2;
    PencilArgs args;
};

// Arguments of one FP16-storage sweep over one grid (pencil_f16.cu): p and
// p_prev FP16 at the power-of-two scale scale->a, K = vel2 dt^2 / dx^2 in BF16.
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

// One shot of the FP16 batch, in device memory: p with the halo box, p_prev and
// K with the tile box, and the sweep's arguments (next = prev: in place).
struct alignas(64) ShotF16 {
    CUtensorMap p, prev, k;
    F16Args args;
};

// Work item: x = shot, y = tile x, z = tile y, w = z chunk.
int batch_f32_variant_count();
const char* batch_f32_variant_name(int v);
PencilBoxes batch_f32_boxes(int v);
int batch_f32_resident(int v);
void batch_f32_prepare();
// Sweep arguments of one shot (tile counts, z chunk length, weights, source) for
// variant v split into zchunks z chunks.
PencilArgs batch_f32_shot_args(int v, const GridDesc& g, int zchunks, float* next,
                               const SourceDesc& src, int* err);
cudaError_t launch_batch_f32(int v, const ShotF32* shots, const int4* items, int n_items,
                             BatchQueue* queue, unsigned ctas, cudaStream_t stream);

int batch_f16_variant_count();
const char* batch_f16_variant_name(int v);
PencilBoxes batch_f16_boxes(int v);
int batch_f16_resident(int v);
void batch_f16_prepare();
// Sweep arguments of one FP16 shot for variant v split into zchunks z chunks;
// scale: the shot's device scale, next: its p_prev / p_next level.
F16Args batch_f16_shot_args(int v, const GridDesc& g, int zchunks, uint16_t* next,
                            const SourceDesc& src, const F16Scale* scale, int* err);
// phase: 0 plain, 1 renormalisation step, 2 the step after it (every shot);
// exact_y: every shot has dx == dy (the FP16 step's exact-y form, as the single-grid
// kernel takes it on such grids, so a shot gets the same bits in both).
cudaError_t launch_batch_f16(int v, const ShotF16* shots, const int4* items, int n_items,
                             BatchQueue* queue, unsigned ctas, int phase, bool exact_y,
                             cudaStream_t stream);
// Whether the FP16 step takes its exact-y form on grid g (dx == dy).
bool f16_exact_y(const GridDesc& g);

}  // namespace sb200
