/*
 * stencil_b200.h -- C ABI of the B200-native stencil time-stepper.
 *
 * Plain pointers and sizes only.  Device pointers are CUDA device memory owned by
 * the caller; `stream` is a cudaStream_t (NULL = legacy default stream).  Every
 * call is asynchronous on that stream unless stated otherwise and returns an int
 * status (SB200_OK or a negative SB200_ERR_* code).  The kernel entry points
 * never allocate device memory; the run, batch and MLP handles own theirs, and
 * the tuner allocates only a few bytes.  sb200_last_error() describes the last
 * failure on the calling thread.
 *
 * Field layout (the reference's GridDims, include/stencil/types.hpp:103-140):
 * extents include a 4-cell halo on every face, z is slowest,
 * idx = (z*ny + y)*nx + x, the interior is [4, n-4) on each axis and halo cells
 * are never written (fixed zero walls).
 */
#ifndef STENCIL_B200_H
#define STENCIL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB200_OK 0
#define SB200_ERR_INVALID (-1)     /* bad argument (null pointer, aliasing, bad extents) */
#define SB200_ERR_CUDA (-2)        /* CUDA runtime / driver error */
#define SB200_ERR_DEVICE (-3)      /* a kernel's bounded wait gave up (device error word) */
#define SB200_ERR_UNSUPPORTED (-4) /* shape or alignment this entry point cannot take */
#define SB200_ERR_MONITOR (-5)     /* stability monitor tripped (non-finite or blow-up) */

/* Grid descriptor: the reference's GridDims (types.hpp:115-140) with an explicit dt. */
typedef struct sb200_grid {
    int64_t nx, ny, nz; /* halo-inclusive extents (interior = n - 8) */
    float dx, dy, dz;   /* grid spacing [m] */
    float dt;           /* time step [s] */
} sb200_grid;

/* ── library / errors ─────────────────────────────────────────────────────── */
int sb200_version(void);
/* Text of the last failure on the calling thread ("" if none). */
const char* sb200_last_error(void);
/* Reads the current device's error word (synchronous); clears it when clear != 0.
 * Returns the word (0 = no device-side error) or a negative status. */
int sb200_device_error(int clear);

/* ── reference kernel-launcher API (include/stencil/kernels.cuh:33-83) ───────── */

/* Replaces upload_fd_coefficients() (kernels.cuh:33; stencil_naive.cu:38-46).
 * The radius-4 weights are compile-time constants of every kernel here, so this
 * only validates that a CUDA device is usable.  Synchronous. */
int sb200_upload_fd_coefficients(void);

/* Replaces launch_naive() (kernels.cuh:42-43; stencil_naive.cu:92-114):
 *   p_next = 2 p_cur - p_prev + dt^2 vel2 lap(p_cur)   on the interior,
 * evaluated in the reference's operation order without FMA contraction
 * (bit-identical to its CPU path built with -ffp-contract=off).
 * p_next must not alias p_cur; p_next == p_prev is allowed (in place). */
int sb200_launch_naive(const float* p_cur, const float* p_prev, const float* vel2,
                       float* p_next, const sb200_grid* grid, void* stream);

/* Replaces launch_tiled() (kernels.cuh:54-55; stencil_tiled.cu:147-168): the same
 * update by the TMA z-marching pencil kernel (FP32, FMA-contracted; within 1e-6
 * relative L2 of the reference order per step).  Grids whose row pitch is not a
 * multiple of 16 bytes (nx % 4 != 0) or with pointers not 16-byte aligned run
 * the naive kernel instead.  Aliasing rules as sb200_launch_naive. */
int sb200_launch_tiled(const float* p_cur, const float* p_prev, const float* vel2,
                       float* p_next, const sb200_grid* grid, void* stream);

/* Replaces launch_slab() (kernels.cuh:63-64; stencil_multi_gpu.cu:60-66): on one
 * GPU a slab whose z-face halos the caller has filled is an ordinary grid, so
 * this is sb200_launch_tiled. */
int sb200_launch_slab(const float* p_cur, const float* p_prev, const float* vel2,
                      float* p_next, const sb200_grid* grid, void* stream);

/* ── solver-step entry points (src/solver/wave_prop.cpp:67-75, heat_diffusion.cpp:103-122) */

/* One acoustic step with centre-source injection (WavePropSolver::step_impl plus
 * the source rule p_next[src] += (dt^2 vel2[src]) * src_amp after the update).
 * src_index < 0 disables the source.  p_next may alias p_prev. */
int sb200_wave_step_f32(const float* p, const float* p_prev, const float* vel2, float* p_next,
                        const sb200_grid* grid, int64_t src_index, float src_amp,
                        void* stream);

/* sb200_wave_step_f32 evaluated in the reference's operation order with no FMA
 * contraction (the kernel behind sb200_launch_naive): bit-identical to the
 * reference CPU path built with -ffp-contract=off, at about a third of the
 * pencil kernel's throughput.  For callers that need reproducible bits. */
int sb200_wave_step_exact_f32(const float* p, const float* p_prev, const float* vel2,
                              float* p_next, const sb200_grid* grid, int64_t src_index,
                              float src_amp, void* stream);

/* sb200_wave_step_f32 with the source sample read on the device as
 * wavelet[*step + step_offset] (wavelet and step are device pointers), so a
 * captured CUDA graph of several steps can be replayed at any time offset.
 * exact != 0 selects the reference-order kernel. */
int sb200_wave_step_dev_f32(const float* p, const float* p_prev, const float* vel2,
                            float* p_next, const sb200_grid* grid, int64_t src_index,
                            const float* wavelet, const int* step, int step_offset, int exact,
                            void* stream);

/* No reference counterpart.  Two acoustic steps in one sweep over the grid
 * (temporal blocking): p_next = the step of (p, p_prev) with source sample
 * src_amp0, p_next2 = the step of (p_next, p) with src_amp1 -- the same bits as
 * sb200_wave_step_f32(p, p_prev, vel2, p_prev, ...) followed by
 * sb200_wave_step_f32(p_prev, p, vel2, p, ...), at 20 B of DRAM traffic per
 * interior point for the pair instead of 32.  p, p_prev, vel2, p_next and
 * p_next2 must be five distinct buffers (other tiles still read p and p_prev
 * while a tile writes its results); the halo cells of p_next and p_next2 are not
 * written and must hold the walls, as p_prev's and p's do (zeros for the
 * reference's fixed walls).  nx % 4 == 0 and 16-byte aligned fields
 * (SB200_ERR_UNSUPPORTED otherwise). */
int sb200_wave_step2_f32(const float* p, const float* p_prev, const float* vel2, float* p_next,
                         float* p_next2, const sb200_grid* grid, int64_t src_index,
                         float src_amp0, float src_amp1, void* stream);

/* sb200_wave_step2_f32 with the two source samples read on the device as
 * wavelet[*step + step_offset] and wavelet[*step + step_offset + 1].  trace
 * (optional device array, NULL for none) receives the source cell's value after
 * each of the two steps at trace[*step + step_offset] and at the next index. */
int sb200_wave_step2_dev_f32(const float* p, const float* p_prev, const float* vel2,
                             float* p_next, float* p_next2, const sb200_grid* grid,
                             int64_t src_index, const float* wavelet, const int* step,
                             int step_offset, float* trace, void* stream);

/* Writes value to the device int *dst (one-thread kernel, stream-ordered). */
int sb200_set_device_int(int* dst, int value, void* stream);

/* One explicit heat step u_next = u + alpha*dt*lap(u) with a scalar diffusivity
 * (HeatDiffusionSolver::step_impl without its vel2 field and D2D copy: 8 B/point).
 * u_next must not alias u. */
int sb200_heat_step_f32(const float* u, float* u_next, const sb200_grid* grid, float alpha,
                        void* stream);

/* No reference counterpart.  First half of a coarse acoustic step that carries
 * the composition term of two leapfrog steps of dt/2 (the learned 2x-coarse
 * path).  With L = vel2 * lap (the 8th-order Laplacian of the grid), writes
 *   r      = p + beta dt^2 L p                  (interior; halo untouched)
 *   p_prev = p_prev + 2 beta dt^2 L p           (in place, interior)
 * so that a plain step of (r, p_prev) -- sb200_wave_step_f32 or
 * sb200_mlp_learned_step -- gives 2 p - p_prev + dt^2 L p + beta dt^4 L^2 p.
 * beta = 1/16 is the dt^4 term of two steps of dt/2.  r, p and p_prev must be
 * distinct; r's halo cells must hold zeros (they are never written); nx % 4 == 0
 * and 16-byte aligned fields (the pencil kernel).  20 B per interior point. */
int sb200_wave_prepass_f32(const float* p, float* p_prev, const float* vel2, float* r,
                           const sb200_grid* grid, float beta, void* stream);

/* ── inputs of the benchmark configurations (host memory; no reference counterpart:
 *    the reference has only a constant / two-layer velocity and a Gaussian pulse,
 *    include/stencil/grid.hpp:57-99) ─────────────────────────────────────────── */

/* Seeded layered velocity model written as v^2 into vel2[nz*ny*nx] (host):
 * n_layers horizontal layers whose interfaces are uniform random depths over the
 * interior, velocities rising linearly from v_top to v_bottom with depth, times
 * (1 + perturbation*g) with g a Gaussian-correlated field (correlation function
 * exp(-r^2/corr_cells^2)) scaled to max|g| = 1.  *v_max_out (optional) receives
 * the largest velocity.  Deterministic for a given seed on every host. */
int sb200_model_layered(float* vel2, int64_t nx, int64_t ny, int64_t nz, uint64_t seed,
                        int n_layers, float v_top, float v_bottom, float perturbation,
                        float corr_cells, float* v_max_out);

/* Ricker wavelet w(t_n) = (1 - 2 pi^2 f^2 tau^2) exp(-pi^2 f^2 tau^2),
 * tau = n*dt - t0, n = 0..n_steps-1, evaluated in double and rounded to float. */
int sb200_ricker(double freq, double t0, double dt, int64_t n_steps, float* out);

/* The heat step in the reference's operation order (no FMA contraction):
 * u_next = u + (alpha*dt) * ((lap_x + lap_y) + lap_z). */
int sb200_heat_step_exact_f32(const float* u, float* u_next, const sb200_grid* grid,
                              float alpha, void* stream);

/* ── FP16-storage acoustic path ─────────────────────────────────────────────
 * No reference counterpart: a reduced-storage precision variant of the
 * acoustic step.  p and p_prev are FP16 holding a * p for a power-of-two scale
 * a kept in device memory (sb200_f16_scale); K = vel2 dt^2 / dx^2 is BF16;
 * arithmetic is FP32.  8 B per interior point and step. */
typedef struct sb200_f16_scale {
    float a; /* current storage scale (fields hold a * p) */
    float r; /* a_new / a_old of the last renormalisation */
} sb200_f16_scale;

/* dst[i] = fp16(src[i] * scale) / src[i] = float(dst[i]) / scale over n elements. */
int sb200_f16_pack(const float* src, uint16_t* dst, int64_t n, float scale, void* stream);
int sb200_f16_unpack(const uint16_t* src, float* dst, int64_t n, float scale, void* stream);
/* K[i] = bf16(vel2[i] * dt^2 / dx^2) over the whole grid. */
int sb200_k_field_bf16(const float* vel2, uint16_t* k, const sb200_grid* grid, void* stream);
/* One FP16-storage step, p_next written in place over p_prev.  phase 0 = plain,
 * 1 = the renormalisation step (output scaled by scale->r), 2 = the step after
 * it (p_prev scaled by scale->r).  The source adds a * dt^2 vel2[src] * w with
 * w = wavelet[*step + step_offset] (device) or src_amp when wavelet is NULL.
 * Needs nx % 8 == 0 and 16-byte aligned fields (SB200_ERR_UNSUPPORTED
 * otherwise). */
int sb200_wave_step_f16(const uint16_t* p, uint16_t* p_prev_next, const uint16_t* k,
                        const sb200_grid* grid, int64_t src_index, float src_amp,
                        const float* wavelet, const int* step, int step_offset,
                        const sb200_f16_scale* scale, int phase, void* stream);
/* Renormalisation (one device thread): with m = stats3[1] / a (stats of the
 * stored field) and b = bound[*step] (or bound_host when bound is NULL),
 * a_new = 2^floor(log2(target / (m + b))), r = a_new / a, a = a_new. */
int sb200_f16_renorm(const double* stats3, sb200_f16_scale* scale, const float* bound,
                     const int* step, float bound_host, float target, void* stream);

/* ── FP64 field statistics (stability monitor, FP16 scale renormalisation) ──
 * out3 (device, 3 doubles) receives, over the interior of the field:
 *   out3[0] = sum of (f/scale)^2, out3[1] = max |f/scale|, out3[2] = number of
 *   non-finite values,
 * accumulated in double with a fixed reduction order (bit-reproducible).
 * scratch (device) must hold at least sb200_field_stats_scratch_len(grid)
 * doubles; it is overwritten.  Asynchronous on `stream`. */
int64_t sb200_field_stats_scratch_len(const sb200_grid* grid);
int sb200_field_stats_f32(const float* field, const sb200_grid* grid, double* out3,
                          double* scratch, int64_t scratch_len, void* stream);
/* The same over an FP16 field stored scaled by `scale` (a value v is v/scale). */
int sb200_field_stats_f16(const uint16_t* field, const sb200_grid* grid, float scale,
                          double* out3, double* scratch, int64_t scratch_len, void* stream);
/* No reference counterpart.  sb200_field_stats_f32 without a scratch argument,
 * for callers that cannot allocate device memory (for example a monitor
 * running while another thread captures a CUDA graph in global capture mode,
 * where cudaMalloc is refused).  It allocates nothing: the per-block partials
 * go to a static device array of 3 * 1184 doubles (28,416 bytes) in the
 * library, which no grid outgrows (a larger need would be rejected with
 * SB200_ERR_INVALID).  Same kernels and block count as sb200_field_stats_f32,
 * so the same bits.  Nothing in the array must start at zero.  The array is
 * shared per device: calls that overlap on the device (unordered streams) race.
 * The first call per device looks up the array's address
 * (cudaGetSymbolAddress); make it before any stream capture starts.  The
 * looked-up address is kept for the life of the process and does not survive
 * cudaDeviceReset.  While another stream of the process is being captured, pass
 * an explicit stream created with cudaStreamNonBlocking: stream NULL is the
 * legacy default stream, whose implicit synchronisation with blocking streams
 * would invalidate that capture. */
int sb200_field_stats_f32_noalloc(const float* field, const sb200_grid* grid, double* out3,
                                  void* stream);

/* ── pencil-kernel configuration (used by the tuner and the tests) ──────────── */
#define SB200_KIND_WAVE_F32 0
#define SB200_KIND_HEAT_F32 1
#define SB200_KIND_WAVE_F16 2
#define SB200_KIND_WAVE2_F32 3 /* sb200_wave_step2_f32: two acoustic steps per sweep */
int sb200_pencil_variant_count(int kind);
const char* sb200_pencil_variant_name(int kind, int variant);
/* Forces (variant, zchunks) for every later launch of `kind` on this process;
 * variant < 0 restores automatic selection. */
int sb200_set_pencil_override(int kind, int variant, int zchunks);
/* The (variant, zchunks) the next launch of `kind` on `grid` would use. */
int sb200_pencil_choice(int kind, const sb200_grid* grid, int* variant, int* zchunks);

/* ── run handle: a whole simulation behind one object ─────────────────────────
 * Replaces the reference's ISolver / SolverBase (include/stencil/solver.hpp:13-24,
 * src/solver/solver_base.cpp:28-116) for C callers: the handle owns the device
 * state (it is the one part of this ABI that allocates), takes the initial
 * fields from host memory, steps on its own stream (CUDA-graph chunks), records
 * the source trace, runs the FP64 stability monitor and hands results back to
 * host memory. */
#define SB200_PHYSICS_WAVE 0
#define SB200_PHYSICS_HEAT 1
#define SB200_PRECISION_F32 0
#define SB200_PRECISION_F16 1 /* acoustic only: FP16 p/p_prev, BF16 vel2 dt^2/dx^2 */

typedef struct sb200_run_config {
    sb200_grid grid;
    int physics;          /* SB200_PHYSICS_* */
    int precision;        /* SB200_PRECISION_* */
    int exact;            /* FP32 only: 1 = reference-order kernels (bit-exact path) */
    float diffusivity;    /* heat: alpha (the step is u += alpha*dt*lap u) */
    int64_t src_index;    /* acoustic point source cell; < 0: no source */
    float src_freq;       /* Ricker peak frequency [Hz]; <= 0: set the wavelet explicitly */
    float src_t0;         /* Ricker delay [s]; < 0: 1/src_freq */
    int graph_chunk;      /* steps per captured CUDA graph (rounded down to even); 0: none */
    int renorm_every;     /* FP16: steps between renormalisations (even, >= 2; 0: 50) */
    int monitor_every;    /* FP32: steps between monitor checks (0: only at sync points) */
    float monitor_limit;  /* largest |p| the monitor accepts (<= 0: 1e30) */
    float f16_target;     /* FP16: renormalise so that max|p| * a <= target (<= 0: 4096) */
} sb200_run_config;

/* Fills cfg with defaults for a grid (wave, FP32, no source, graphs of 100). */
void sb200_run_config_init(sb200_run_config* cfg, const sb200_grid* grid);
int sb200_run_create(const sb200_run_config* cfg, void** handle);
int sb200_run_destroy(void* handle);
/* Initial fields from host memory (nx*ny*nz floats each): p, p_prev (NULL: =
 * p), vel2 (acoustic; ignored for heat).  Resets the step count.  Synchronous. */
int sb200_run_set_fields(void* handle, const float* p, const float* p_prev, const float* vel2);
/* Replaces the source wavelet with n host samples (one per step). */
int sb200_run_set_wavelet(void* handle, const float* w, int64_t n);
/* Enqueues n steps on the handle's stream (asynchronous). */
int sb200_run_steps(void* handle, int64_t n);
/* Waits for the enqueued steps; returns SB200_ERR_MONITOR if the monitor saw a
 * non-finite value or |p| above the limit, SB200_ERR_DEVICE on a device error. */
int sb200_run_synchronize(void* handle);
/* Current field in physical units into host memory (synchronous). */
int sb200_run_get_field(void* handle, float* p);
/* XY plane z of the current field (nx*ny floats, x fastest) in physical units
 * into host memory (synchronous).  Only that plane crosses to the host: the
 * per-frame read of the reference's slice writer (src/main_slice.cpp:112-121,
 * which downloads the whole grid and keeps plane nz/2). */
int sb200_run_get_plane(void* handle, int64_t z, float* plane);
/* First n source-trace samples (p at the source after each step) to host memory. */
int sb200_run_get_trace(void* handle, float* trace, int64_t n);
/* FP64 statistics {sum p^2, max |p|, non-finite count} of the current field. */
int sb200_run_stats(void* handle, double* out3);
int64_t sb200_run_steps_done(void* handle);
/* The handle's cudaStream_t. */
void* sb200_run_stream(void* handle);

/* ── autotuner ──────────────────────────────────────────────────────────────
 * Times every compiled tile variant of `kind` at its three best-filling z splits
 * on `grid` (reps launches each after one warm-up, CUDA events, legacy default
 * stream, synchronous) and records the fastest for later launches of that kind
 * on that grid and device.  The stencil reads field (and, for the acoustic kind,
 * prev and vel2) and writes only `scratch`, a caller buffer of the grid's size
 * that aliases none of them.  For SB200_KIND_WAVE_F16, field is p (FP16), vel2
 * is K (BF16), prev is only checked for NULL, and scratch is the in-place
 * p_prev / p_next buffer (FP16; its contents are overwritten).  Outputs are
 * optional. */
int sb200_tune(int kind, const sb200_grid* grid, const void* field, const void* prev,
               const void* vel2, void* scratch, int reps, int* variant, int* zchunks,
               float* best_ms);
/* Saves / loads the tuned table ("kind nx ny nz variant zchunks ms device" per
 * line).  Load returns the number of entries read or a negative status. */
int sb200_tune_save(const char* path);
int sb200_tune_load(const char* path);

/* ── batched shots ─────────────────────────────────────────────────────────
 * No reference counterpart (the reference runs one grid per solver).  Many
 * independent acoustic shots of uneven sizes advance together: each step is one
 * persistent launch whose CTAs pull (shot, tile, z chunk) items from a device
 * work queue; chunks of graph_chunk steps replay from captured CUDA graphs.
 * Every shot uses the same arithmetic as sb200_wave_step_f32 (in-place leapfrog,
 * source rule p[src] += dt^2 vel2[src] w[n] after the update, trace = p[src]
 * after each step).  Shots need nx % 4 == 0 and a source (if any) in the
 * interior.  The handle owns its device memory and a non-blocking stream. */
typedef struct {
    sb200_grid grid;
    int64_t src_index; /* flat source cell, or -1 */
} sb200_shot;

typedef struct {
    int precision;     /* SB200_PRECISION_F32, or SB200_PRECISION_F16: p / p_prev in
                          FP16 at per-shot power-of-two scales renormalised every 50
                          steps (FP64 statistics), K in BF16; every nx % 8 == 0 */
    int graph_chunk;   /* steps per captured graph; 0 = one launch per step (FP16:
                          a multiple of 50 so that each chunk starts on a renorm) */
    int64_t max_steps; /* capacity of the per-shot wavelet and trace tables */
} sb200_batch_config;

void sb200_batch_config_init(sb200_batch_config* cfg);
int sb200_batch_create(const sb200_shot* shots, int n_shots, const sb200_batch_config* cfg,
                       void** handle);
int sb200_batch_destroy(void* handle);
/* Host fields of one shot (halo-inclusive, z-major); p_prev NULL means p. */
int sb200_batch_set_fields(void* handle, int shot, const float* p, const float* p_prev,
                           const float* vel2);
/* Source samples w[0..n) of one shot (n <= max_steps; the rest stay zero). */
int sb200_batch_set_wavelet(void* handle, int shot, const float* w, int64_t n);
/* Enqueues n steps of every shot; the run may not pass max_steps in total. */
int sb200_batch_steps(void* handle, int64_t n);
/* Waits for the enqueued steps.  Returns SB200_ERR_MONITOR when a shot's
 * stability monitor tripped: a non-finite value, or (FP32) max |p| above the
 * limit, in the FP64 statistics taken at every graph-chunk end (FP32), at every
 * renormalisation (FP16) and at synchronisation; SB200_ERR_DEVICE on a device
 * error.  The run handle's monitor per shot (sb200_run_synchronize). */
int sb200_batch_synchronize(void* handle);
/* Largest |p| the FP32 monitor accepts (default 1e30). */
int sb200_batch_set_monitor_limit(void* handle, float limit);
/* Per-shot monitor flags (n_shots ints, 1 = tripped) to host memory after the
 * check of the current level (synchronous; set_fields clears a shot's flag). */
int sb200_batch_monitor_flags(void* handle, int* flags);
int sb200_batch_get_field(void* handle, int shot, float* p);
int sb200_batch_get_trace(void* handle, int shot, float* trace, int64_t n);
/* Times every (tile variant, z-chunk length) on the batch's own buffers and
 * keeps the fastest (cached per process by the shots' extents).  Call it before
 * sb200_batch_set_fields: it leaves fields, traces and the step count zeroed. */
int sb200_batch_tune(void* handle, int reps);
int sb200_batch_set_choice(void* handle, int variant, int zlen);
int sb200_batch_choice(void* handle, int* variant, int* zlen, int* n_items, int* ctas);
int64_t sb200_batch_steps_done(void* handle);
void* sb200_batch_stream(void* handle);
/* Tile variants of FP32 batches (set_choice / choice index these; an FP16
 * batch indexes its own table, named by sb200_batch_variant_name_f16). */
int sb200_batch_variant_count(void);
const char* sb200_batch_variant_name(int variant);
int sb200_batch_variant_count_f16(void);
const char* sb200_batch_variant_name_f16(int variant);

/* ── learned coarse correction ─────────────────────────────────────────────
 * No reference counterpart.  A per-point MLP 26 -> 32 -> 32 -> 1 (ReLU), BF16
 * tensor-core mma with FP32 accumulation, corrects a 2x-coarser grid stepped
 * with 2x dt:  p_next[i] += s_i * c * MLP(f_i).  f_i is the 25-point star of p
 * at i in a difference basis, divided by s_i (the star's largest magnitude):
 * [p_c, (p_+r - p_-r) for axis x, y, z and r = 1..4, (p_+r + p_-r - 2 p_c)
 * likewise], evaluated in FP32; then the Courant number sqrt(vel2) dt / dx;
 * zero-padded to 32 BF16 features per row.  c is the handle's output scale.
 * Parameters (FP32, SB200_MLP_NPARAM): W1[32][32] (out x in; inputs 26..31
 * unused), b1[32], W2[32][32], b2[32], w3[32], b3. */
#define SB200_MLP_NPARAM 2145
#define SB200_MLP_FEATURES 32

/* Handle with the parameters on the current device, He-initialised from seed. */
int sb200_mlp_create(uint64_t seed, void** handle);
int sb200_mlp_destroy(void* handle);
/* Host copies of the FP32 parameters (synchronous); set also resets Adam. */
int sb200_mlp_get_params(void* handle, float* params);
int sb200_mlp_set_params(void* handle, const float* params);
/* Output scale c of the correction (default 1; training divides the targets by
 * it).  Get returns 0 for a NULL handle. */
int sb200_mlp_set_output_scale(void* handle, float scale);
float sb200_mlp_output_scale(void* handle);
/* y[r] = MLP(X[r]) for n rows of 32 BF16 features (device pointers). */
int sb200_mlp_forward(void* handle, const uint16_t* X, float* y, int64_t n, void* stream);
/* Gradient of mean_r (MLP(X[r]) - t[r])^2 into grad[0..NPARAM) (device FP32,
 * overwritten) and the loss into grad[NPARAM]. */
int sb200_mlp_gradients(void* handle, const uint16_t* X, const float* t, int64_t n, float* grad,
                        void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the batch; *loss (device,
 * optional) receives the batch loss before the step. */
int sb200_mlp_train_step(void* handle, const uint16_t* X, const float* t, int64_t n, float lr,
                         float* loss, void* stream);
/* p_next += s * c * MLP(features of p) on the interior (p, vel2, p_next device
 * FP32; p_next must not alias p).  Runs on tcgen05 (TMEM accumulators) unless
 * sb200_mlp_set_kernel selected the mma.sync kernel. */
int sb200_mlp_correct(void* handle, const float* p, const float* vel2, float* p_next,
                      const sb200_grid* grid, void* stream);
/* One learned coarse step in one fused launch: p_prev_next <- acoustic step of
 * (p, p_prev_next, vel2) + s * c * MLP(features of p), in place over p_prev (no
 * source term: inject it afterwards).  Bit for bit sb200_wave_step_f32 followed
 * by sb200_mlp_correct (tcgen05).  Needs nx % 4 == 0 and 16-byte aligned fields
 * (SB200_ERR_UNSUPPORTED otherwise); p_prev_next must not alias p.  After a
 * train_step the first call copies the parameters to the host (synchronising
 * the stream). */
int sb200_mlp_learned_step(void* handle, const float* p, float* p_prev_next, const float* vel2,
                           const sb200_grid* grid, void* stream);
/* Bytes of the activity flags of sb200_mlp_learned_step_flags on `grid` (one
 * byte per 32 x 16 column tile and z chunk of its launch; depends on the grid
 * and the device). */
int64_t sb200_mlp_flags_bytes(void* handle, const sb200_grid* grid);
/* sb200_mlp_learned_step with activity flags (the same bits).  flags_in (device,
 * sb200_mlp_flags_bytes bytes, or NULL: every chunk active) describes p, one
 * byte per chunk: bit 0 = some value at or above half the correction floor, bits 1-6
 * = such a value within 4 cells of the chunk's -x, +x, -y, +y, -z, +z face;
 * 0xFF when unknown.  Cells of `box` (x0, x1, y0, y1, z0, z1, half-open; NULL:
 * none) count as active too -- pass the box of whatever was added to p after
 * the step that wrote its flags (a source).  A chunk whose own bit 0 and whose
 * face neighbours' facing bits are clear takes the plain step with no network
 * work.  flags_out (or NULL) receives the flags of p_next; it must not be
 * flags_in.  Start a run with flags_in all 0xFF (or NULL). */
int sb200_mlp_learned_step_flags(void* handle, const float* p, float* p_prev_next,
                                 const float* vel2, const sb200_grid* grid, const uint8_t* flags_in,
                                 uint8_t* flags_out, const int64_t* box, void* stream);
/* Activity flags for the field r = p + c L p of sb200_wave_prepass_f32, from the
 * flags of p (both in the layout of sb200_mlp_flags_bytes): a chunk gets every
 * bit when a 25-point star of p reaches it (p's chunk or a face neighbour's
 * facing slab is flagged), else none.  The learned step of r then takes these as
 * flags_in; its box argument must be grown by the stencil radius (4 cells),
 * since the pre-pass spreads a box's values that far.  flags_p != flags_r. */
int sb200_mlp_flags_compose(void* handle, const sb200_grid* grid, const uint8_t* flags_p,
                            uint8_t* flags_r, void* stream);
/* Correction floor: a point whose 25-point star has largest magnitude below
 * `floor` gets no correction (default 0: every point with a nonzero star).  Ahead
 * of a wavefront the stencil leaves values that decay and underflow; a correction
 * proportional to them keeps them alive, so a floor far below the field's scale
 * keeps those regions exactly zero (and lets the fused step skip them). */
int sb200_mlp_set_min_scale(void* handle, float floor);
float sb200_mlp_min_scale(void* handle);
/* Correction kernel of the handle: 0 = tcgen05 (default), 1 = mma.sync. */
int sb200_mlp_set_kernel(void* handle, int kernel);
/* Training rows at n cells (device int64 flat indices, interior only):
 * X[r] = features of p at cells[r], t[r] = (p_true - p_plain)[cell] / s. */
int sb200_mlp_samples(const float* p, const float* vel2, const float* p_true, const float* p_plain,
                      const sb200_grid* grid, const int64_t* cells, int64_t n, uint16_t* X,
                      float* t, void* stream);
/* field[x0+i, y0+j, z0+k] += scale * pattern[(k*by + j)*bx + i] for the box's
 * interior cells (pattern device FP32): a spatially extended source term. */
int sb200_add_box(float* field, const sb200_grid* grid, int x0, int y0, int z0, int bx, int by,
                  int bz, const float* pattern, float scale, void* stream);
/* In-place Gaussian smoothing (separable, clamp-to-edge, width sigma_cells <= 16,
 * radius 3 sigma) of a whole halo-inclusive field; tmp is a device buffer of
 * the same size.  Used to give a velocity model the resolution both grids of
 * the learned path share.  Synchronous on `stream`. */
int sb200_smooth3(float* field, float* tmp, const sb200_grid* grid, float sigma_cells,
                  void* stream);
/* coarse[x,y,z] = fine[2x+offset, 2y+offset, 2z+offset] on the coarse interior
 * (zero on its halo and where the fine index falls outside the fine grid). */
int sb200_restrict2(const float* fine, const sb200_grid* fine_grid, float* coarse,
                    const sb200_grid* coarse_grid, int offset, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* STENCIL_B200_H */
