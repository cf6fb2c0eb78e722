// Internal launcher interface between the C ABI (capi.cu) and the kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace sb200 {

// Halo-inclusive grid, z slowest: idx = (z*ny + y)*nx + x.  Interior is [4, n-4)
// on every axis (the reference's GridDims convention, include/stencil/types.hpp:115-140).
struct GridDesc {
    int64_t nx = 0, ny = 0, nz = 0;
    float dx = 1.f, dy = 1.f, dz = 1.f, dt = 1.f;
    bool has_interior() const { return nx > 8 && ny > 8 && nz > 8; }
    int64_t size() const { return nx * ny * nz; }
    int64_t interior() const {
        return has_interior() ? (nx - 8) * (ny - 8) * (nz - 8) : 0;
    }
};

// Tile configuration of a pencil launch (chosen by the tuner or a default).
struct PencilConfig {
    int variant = 0;  // index into the compiled tile table of the kernel family
    int zchunks = 1;  // z splits of the interior (1 = march the whole column)
};

// Source injection for one step: p_next[idx] += (dt^2*vel2[idx]) * w.
// When wavelet != nullptr the sample is read on the device as
// wavelet[*step + step_offset], which lets a captured CUDA graph replay a chunk of
// steps against a device-side step counter.  When trace != nullptr the thread
// that injects also records the new value at the source (physical units) in
// trace[(step ? *step : 0) + step_offset].
struct SourceDesc {
    int64_t idx = -1;
    float w = 0.f;
    const float* wavelet = nullptr;
    const int* step = nullptr;
    int step_offset = 0;
    float* trace = nullptr;
};

cudaError_t launch_wave_naive(const float* cur, const float* prev, const float* vel2,
                              float* next, const GridDesc& g, const SourceDesc& src,
                              cudaStream_t stream);
cudaError_t launch_set_int(int* dst, int value, cudaStream_t stream);
cudaError_t launch_heat_naive(const float* u, float* u_next, const GridDesc& g, float alpha_dt,
                              cudaStream_t stream);

// Tensor maps of one pencil launch: p (or u) with the halo box, and -- for the
// acoustic variants that stage them through TMA -- p_prev and vel2 with the
// interior tile box.  Unused maps may hold any valid map.
struct PencilMaps {
    CUtensorMap p, prev, vel2;
};

// TMA boxes a variant needs.
struct PencilBoxes {
    int halo_x = 0, halo_y = 0;  // p / u box: tile + 4-cell halo on each side
    int tile_x = 0, tile_y = 0;  // p_prev / vel2 box
    bool aux_tma = false;        // whether p_prev / vel2 go through TMA
};

// FP32 pencil kernels.  Preconditions (checked by the caller): nx % 4 == 0,
// 16-byte aligned pointers, has_interior().  next may alias prev (in place).
int pencil_f32_variant_count(bool heat);
const char* pencil_f32_variant_name(bool heat, int v);
PencilBoxes pencil_f32_boxes(bool heat, int v);
struct Weights;  // sb200_common.cuh

// Network of the fused learned coarse step (learned_step.cu): BF16 W1, W2 on the
// device, biases and w3 by value, the output scale c.
struct LearnedNet {
    const uint16_t* w1b = nullptr;
    const uint16_t* w2b = nullptr;
    float b1[32] = {}, b2[32] = {}, w3[32] = {};
    float b3 = 0.f;
    float out_scale = 1.f;
    float min_scale = 0.f;  // correction floor (stars below it: no correction)
};
// Boxes of its tensor maps, resident CTAs per SM, and the launch: p_next =
// acoustic step of p + learned correction, in place over p_prev.
PencilBoxes learned_step_boxes();
int learned_step_resident();
// Its work split: 32 x 16 column tiles x zchunks z chunks of zlen planes (one
// activity flag byte per tile and chunk).
struct LearnedChunks {
    int tiles_x = 0, tiles_y = 0, zchunks = 0, zlen = 0;
};
LearnedChunks learned_step_chunks(const GridDesc& g, int sms, bool flagged);
// Activity flags of r = p + c L p from those of p (same chunk layout): every
// chunk a star of p reaches gets all bits, the others none.
cudaError_t launch_flags_compose(const uint8_t* in, uint8_t* out, const GridDesc& g, int sms,
                                 cudaStream_t stream);
// flags_in: per chunk, whether p may hold a value at or above the floor (NULL:
// all may); box (x0, x1, y0, y1, z0, z1 cells, or NULL) counts as flagged;
// flags_out receives the flags of p_next (NULL: none).
cudaError_t launch_learned_step(const PencilMaps& maps, float* next, const GridDesc& g,
                                const LearnedNet& net, int sms, int* err, cudaStream_t stream,
                                const uint8_t* flags_in = nullptr, uint8_t* flags_out = nullptr,
                                const int64_t* box = nullptr);

// Laplacian weights of the pencil kernels (C_r / dx_a^2, times `scale`: dt^2 for
// the acoustic step, alpha dt for heat), rounded once from double.
Weights fold_weights(const GridDesc& g, float scale);

cudaError_t launch_wave_pencil_f32(const PencilMaps& maps, const float* prev, const float* vel2,
                                   float* next, const GridDesc& g, const SourceDesc& src,
                                   const PencilConfig& cfg, int* err, cudaStream_t stream);
cudaError_t launch_heat_pencil_f32(const PencilMaps& maps, float* u_next, const GridDesc& g,
                                   float alpha_dt, const PencilConfig& cfg, int* err,
                                   cudaStream_t stream);
// The acoustic tile `cfg.variant` in prepass mode: r = p + beta dt^2 v^2 lap p,
// prev += 2 beta dt^2 v^2 lap p (maps as for the acoustic step, prev read and
// written in place).
cudaError_t launch_prepass_pencil_f32(const PencilMaps& maps, float* prev, const float* vel2,
                                      float* r, const GridDesc& g, float beta,
                                      const PencilConfig& cfg, int* err, cudaStream_t stream);
// Two acoustic steps per sweep (leap2_f32.cu): out1 = p at t+dt, out2 = p at
// t+2dt, the same bits as two launch_wave_pencil_f32 steps.  maps: p with the
// leap2_boxes(v) halo box, p_prev and vel2 with its tile box.  p, p_prev, vel2,
// out1 and out2 are distinct; out1 and out2 keep their halo cells (they must
// hold the walls).  The source adds src's sample at step s and w1 at step s+1
// (with a wavelet table: wavelet[*step + step_offset] and the next sample).
int leap2_variant_count();
const char* leap2_variant_name(int v);
PencilBoxes leap2_boxes(int v);
int leap2_resident(int v);
void leap2_prepare();
int64_t leap2_ctas(int v, const GridDesc& g, int zchunks);
cudaError_t launch_leap2_f32(const PencilMaps& maps, float* out1, float* out2, const GridDesc& g,
                             const SourceDesc& src, float w1, const PencilConfig& cfg, int* err,
                             cudaStream_t stream);

// Resident CTAs per SM of a variant (occupancy query; analytic if that fails).
// The first call per device also sets the variant's shared-memory attribute.
int pencil_f32_resident(bool heat, int v);
// Sets up every variant on the current device (before a stream capture, whose
// launches must not be the first ones).
void pencil_f32_prepare();
void pencil_f16_prepare();
// Number of CTAs a launch uses (for occupancy/wave reasoning in the tuner).
int64_t pencil_f32_ctas(bool heat, int v, const GridDesc& g, int zchunks);

// z splits of variant v on grid g ranked by how well their CTA count fills whole
// waves (SMs x resident CTAs), discounted by the 8 halo planes each extra split
// re-reads; the first max_n (capi.cu).
std::vector<int> zchunk_ranking(int kind, int v, const GridDesc& g, int max_n);

// Tuned (variant, zchunks) for kind on grid g on the current device, if the
// tuner has one (tuner.cpp).
bool tuned_choice(int kind, const GridDesc& g, PencilConfig* out);

// Storage scale of the FP16 path, in device memory: fields hold a * p; a
// renormalisation sets a to a_new and r = a_new / a_old (powers of two).
struct F16Scale {
    float a;
    float r;
};

// FP16-storage acoustic pencil kernel (pencil_f16.cu).  phase 0: plain step;
// 1: output scaled by r (renormalisation step); 2: p_prev scaled by r.
// Preconditions: nx % 8 == 0, 16-byte aligned pointers.
int pencil_f16_variant_count();
const char* pencil_f16_variant_name(int v);
PencilBoxes pencil_f16_boxes(int v);
int pencil_f16_resident(int v);
int64_t pencil_f16_ctas(int v, const GridDesc& g, int zchunks);
cudaError_t launch_wave_pencil_f16(const PencilMaps& maps, uint16_t* next, const GridDesc& g,
                                   const SourceDesc& src, const F16Scale* scale, int phase,
                                   const PencilConfig& cfg, int* err, cudaStream_t stream);

cudaError_t launch_f16_pack(const float* f, uint16_t* h, int64_t n, float scale, cudaStream_t st);
cudaError_t launch_f16_unpack(const uint16_t* h, float* f, int64_t n, float scale,
                              cudaStream_t st);
cudaError_t launch_k_bf16(const float* vel2, uint16_t* k, int64_t n, float dt2_over_dx2,
                          cudaStream_t st);
cudaError_t launch_f16_renorm(const double* stats3, F16Scale* scale, const float* bound,
                              const int* step, float bound_host, float target, cudaStream_t st);

// FP64 interior statistics (reduce.cu): out3 = {sum of (f/scale)^2, max |f/scale|,
// count of non-finite values}.  scratch holds 3 doubles per pass-1 block
// (stats_blocks(g) blocks, at most kMaxStatsBlocks).
constexpr int kMaxStatsBlocks = 1184;  // 148 SMs x 8
int stats_blocks(const GridDesc& g);
cudaError_t launch_field_stats(const void* field, bool half, const GridDesc& g, float scale,
                               double* out3, double* scratch, cudaStream_t stream);

// Tensor maps (tmap.cpp).  Encodes (and caches) a 3-D tiled map over a
// halo-inclusive field of element size esize bytes with the given box and copies
// it to *out.  Returns 0 or a CUresult / -1 (driver entry point unavailable).
int tensor_map_3d(CUtensorMap* out, const void* base, int64_t nx, int64_t ny, int64_t nz,
                  int esize, int box_x, int box_y);

}  // namespace sb200
