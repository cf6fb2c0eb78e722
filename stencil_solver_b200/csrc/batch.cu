// Batch engine: many independent acoustic shots of uneven grid sizes advanced
// together, one persistent launch per time step (no reference counterpart; the
// reference runs one grid per solver).
//
// Device layout: one arena holds every shot's two time levels and its vel2
// (each rounded up to 256 bytes); per parity, a table of shot descriptors
// (TMA maps + sweep arguments) tells the kernel which level is current.  The
// work list is every shot's (tile x, tile y, z chunk) triple, shots in order of
// decreasing size so the largest pieces are handed out first; CTAs pull items
// from a device counter until the list is empty (batch_f32_kernel).  The
// kernel's last CTA resets the counter and advances the shared step index that
// selects each shot's source sample and trace slot, so chunks of steps replay
// from captured CUDA graphs with no host work between steps.
//
// The tile shape and z-chunk length come from a small autotuner (sb200_batch_tune)
// that times each candidate on the batch itself; choices are cached per process
// by the precision and the set of shot extents.
//
// FP16 storage (batch_f16_kernel): the levels hold p / p_prev in FP16 at a
// per-shot power-of-two scale and the third array K = vel2 dt^2 / dx^2 in BF16.
// Every 50 steps each shot's FP64 statistics and source bound set its new scale
// (sb200_f16_renorm, reading the device step counter), the launch after that
// rescales the output (phase 1) and the next one p_prev (phase 2); a captured
// 100-step chunk holds two such windows.  Fields cross the boundary in FP32
// through a one-shot staging buffer (pack on set_fields, unpack on get_field).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "batch.h"
#include "dispatch.h"
#include "kernels.h"
#include "stencil_b200.h"

namespace sb200 {
namespace {

constexpr size_t kAlign = 256;
size_t round_up(size_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// z-chunk lengths the tuner tries (0: one chunk per column).
constexpr int kZlens[] = {0, 128, 64, 32};

// Stability monitor of one shot: a non-finite value or max |p| above the limit
// (FP64 statistics {sum p^2, max |p|, non-finite count}) sets its flag.
__global__ void batch_monitor_kernel(const double* stats3, int* flag, double limit) {
    if (!(stats3[2] == 0.0) || !(stats3[1] <= limit)) *flag = 1;
}

struct BatchChoice {
    int variant = 0;
    int zlen = 64;
    float ms = 0.f;
};
std::mutex g_choice_mu;
std::map<std::string, BatchChoice>* g_choices = nullptr;

class Batch {
public:
    int init(const sb200_shot* shots, int n, const sb200_batch_config& cfg) {
        if (!shots || n <= 0) return set_error(SB200_ERR_INVALID, "sb200_batch_create: no shots");
        if (cfg.precision != SB200_PRECISION_F32 && cfg.precision != SB200_PRECISION_F16)
            return set_error(SB200_ERR_UNSUPPORTED, "sb200_batch_create: unknown precision");
        f16_ = cfg.precision == SB200_PRECISION_F16;
        esz_ = f16_ ? 2 : 4;
        if (cfg.max_steps <= 0)
            return set_error(SB200_ERR_INVALID, "sb200_batch_create: max_steps must be positive");
        chunk_ = cfg.graph_chunk > 0 ? cfg.graph_chunk : 0;
        if (f16_ && chunk_ % kRenorm != 0)
            return set_error(SB200_ERR_INVALID,
                             "sb200_batch_create: FP16 graph_chunk must be a multiple of 50");
        cap_ = cfg.max_steps;
        size_t off = 0;
        for (int s = 0; s < n; ++s) {
            const sb200_grid& g = shots[s].grid;
            if (g.nx <= 8 || g.ny <= 8 || g.nz <= 8)
                return set_error(SB200_ERR_INVALID, "sb200_batch_create: shot " + std::to_string(s) +
                                                        ": every extent must exceed 8");
            if (g.nx % (f16_ ? 8 : 4) != 0)
                return set_error(SB200_ERR_UNSUPPORTED,
                                 "sb200_batch_create: shot " + std::to_string(s) + ": nx must be a multiple of " +
                                     std::to_string(f16_ ? 8 : 4));
            if (g.nx > 4096 || g.ny > 4096 || g.nz > 4096)
                return set_error(SB200_ERR_INVALID, "sb200_batch_create: shot " + std::to_string(s) +
                                                        ": extent above 4096");
            if (!(g.dx > 0) || !(g.dy > 0) || !(g.dz > 0) || !(g.dt > 0))
                return set_error(SB200_ERR_INVALID, "sb200_batch_create: shot " + std::to_string(s) +
                                                        ": spacing and dt must be positive");
            Shot h;
            h.g.nx = g.nx;
            h.g.ny = g.ny;
            h.g.nz = g.nz;
            h.g.dx = g.dx;
            h.g.dy = g.dy;
            h.g.dz = g.dz;
            h.g.dt = g.dt;
            h.src = shots[s].src_index;
            if (h.src >= 0) {
                const int64_t x = h.src % g.nx, y = (h.src / g.nx) % g.ny, z = h.src / (g.nx * g.ny);
                if (z >= g.nz || x < 4 || y < 4 || z < 4 || x >= g.nx - 4 || y >= g.ny - 4 ||
                    z >= g.nz - 4)
                    return set_error(SB200_ERR_INVALID, "sb200_batch_create: shot " +
                                                            std::to_string(s) +
                                                            ": the source must be an interior cell");
            }
            const size_t bytes = round_up(static_cast<size_t>(h.g.size()) * esz_);
            max_points_ = std::max<int64_t>(max_points_, h.g.size());
            h.off[0] = off;
            h.off[1] = off + bytes;
            h.off[2] = off + 2 * bytes;
            off += 3 * bytes;
            shots_.push_back(h);
        }
        arena_bytes_ = off;
        err_ = device_error_word();
        if (!err_) return set_error(SB200_ERR_CUDA, "sb200_batch_create: device error word unavailable");
        if (int rc = cuda(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking))) return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&arena_), arena_bytes_)) return rc;
        for (int p = 0; p < 2; ++p)
            if (int rc = alloc(&table_[p], shot_bytes() * n)) return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&queue_), sizeof(BatchQueue))) return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&wave_), sizeof(float) * cap_ * n)) return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&trace_), sizeof(float) * cap_ * n)) return rc;
        // FP64 statistics (monitor; FP16: renormalisation too), their scratch,
        // and one monitor flag per shot
        if (int rc = alloc(reinterpret_cast<void**>(&stats_), sizeof(double) * 3 * n)) return rc;
        for (const Shot& h : shots_) {
            sb200_grid gg = to_grid(h.g);
            scratch_len_ = std::max(scratch_len_, sb200_field_stats_scratch_len(&gg));
        }
        if (int rc = alloc(reinterpret_cast<void**>(&scratch_), sizeof(double) * scratch_len_)) return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&mon_), sizeof(int) * n)) return rc;
        if (int rc = cuda(cudaMemsetAsync(mon_, 0, sizeof(int) * n, st_))) return rc;
        if (f16_) {
            // scales, source bounds, FP32 staging
            if (int rc = alloc(reinterpret_cast<void**>(&scale_), sizeof(F16Scale) * n)) return rc;
            if (int rc = alloc(reinterpret_cast<void**>(&bound_), sizeof(float) * cap_ * n)) return rc;
            if (int rc = alloc(reinterpret_cast<void**>(&staging_), sizeof(float) * max_points_)) return rc;
            if (int rc = cuda(cudaMemsetAsync(bound_, 0, sizeof(float) * cap_ * n, st_))) return rc;
            std::vector<F16Scale> ones(n, F16Scale{1.f, 1.f});
            if (int rc = cuda(cudaMemcpyAsync(scale_, ones.data(), sizeof(F16Scale) * n,
                                              cudaMemcpyHostToDevice, st_)))
                return rc;
            if (int rc = cuda(cudaStreamSynchronize(st_))) return rc;
            wave_host_.assign(n, {});
            vel2_src_.assign(n, 0.f);
        }
        if (int rc = cuda(cudaMemsetAsync(arena_, 0, arena_bytes_, st_))) return rc;
        if (int rc = cuda(cudaMemsetAsync(wave_, 0, sizeof(float) * cap_ * n, st_))) return rc;
        if (int rc = reset_clock()) return rc;
        if (f16_)
            batch_f16_prepare();
        else
            batch_f32_prepare();
        BatchChoice c;
        if (cached_choice(&c)) {
            variant_ = c.variant;
            zlen_ = c.zlen;
        }
        if (int rc = build()) return rc;
        return cuda(cudaStreamSynchronize(st_));
    }

    ~Batch() {
        if (st_) cudaStreamSynchronize(st_);
        drop_graphs();
        for (void* p : {static_cast<void*>(arena_), static_cast<void*>(table_[0]),
                        static_cast<void*>(table_[1]), static_cast<void*>(queue_),
                        static_cast<void*>(wave_), static_cast<void*>(trace_),
                        static_cast<void*>(items_), static_cast<void*>(scale_),
                        static_cast<void*>(stats_), static_cast<void*>(scratch_),
                        static_cast<void*>(bound_), static_cast<void*>(staging_),
                        static_cast<void*>(mon_)})
            if (p) cudaFree(p);
        if (st_) cudaStreamDestroy(st_);
    }

    int set_fields(int s, const float* p, const float* p_prev, const float* vel2) {
        if (s < 0 || s >= n_shots()) return set_error(SB200_ERR_INVALID, "sb200_batch_set_fields: bad shot");
        if (!p || !vel2) return set_error(SB200_ERR_INVALID, "sb200_batch_set_fields: NULL field");
        if (!p_prev) p_prev = p;
        const Shot& h = shots_[s];
        const size_t bytes = static_cast<size_t>(h.g.size()) * 4;
        const int cur = static_cast<int>(step_ & 1);  // level that is current now
        // new fields: the shot's monitor starts clear (and is checked again)
        if (int rc = cuda(cudaMemsetAsync(mon_ + s, 0, sizeof(int), st_))) return rc;
        checked_step_ = -1;
        if (f16_) return set_fields_f16(s, p, p_prev, vel2, cur);
        if (int rc = cuda(cudaMemcpyAsync(arena_ + h.off[cur], p, bytes, cudaMemcpyHostToDevice, st_)))
            return rc;
        if (int rc = cuda(cudaMemcpyAsync(arena_ + h.off[cur ^ 1], p_prev, bytes,
                                          cudaMemcpyHostToDevice, st_)))
            return rc;
        if (int rc = cuda(cudaMemcpyAsync(arena_ + h.off[2], vel2, bytes, cudaMemcpyHostToDevice, st_)))
            return rc;
        return cuda(cudaStreamSynchronize(st_));
    }

    int set_wavelet(int s, const float* w, int64_t n) {
        if (s < 0 || s >= n_shots()) return set_error(SB200_ERR_INVALID, "sb200_batch_set_wavelet: bad shot");
        if (!w || n <= 0 || n > cap_)
            return set_error(SB200_ERR_INVALID, "sb200_batch_set_wavelet: need 1..max_steps samples");
        if (int rc = cuda(cudaMemcpyAsync(wave_ + s * cap_, w, sizeof(float) * n,
                                          cudaMemcpyHostToDevice, st_)))
            return rc;
        if (f16_) {
            wave_host_[s].assign(w, w + n);
            if (int rc = upload_bound(s)) return rc;
        }
        return cuda(cudaStreamSynchronize(st_));
    }

    int steps(int64_t n) {
        if (n < 0) return set_error(SB200_ERR_INVALID, "sb200_batch_steps: negative count");
        if (step_ + n > cap_)
            return set_error(SB200_ERR_INVALID, "sb200_batch_steps: the run would pass max_steps (" +
                                                    std::to_string(cap_) + ")");
        int64_t done = 0;
        while (done < n) {
            // FP16: a graph chunk starts on a renormalisation step (its phase
            // pattern is then the same every time).
            if (chunk_ > 0 && n - done >= chunk_ && (!f16_ || step_ % kRenorm == 0)) {
                const int par = static_cast<int>(step_ & 1);
                if (!graph_[par])
                    if (int rc = capture(par, &graph_[par])) return rc;
                if (int rc = cuda(cudaGraphLaunch(graph_[par], st_))) return rc;
                step_ += chunk_;
                done += chunk_;
                continue;
            }
            if (int rc = step_once(step_, static_cast<int>(step_ & 1))) return rc;
            ++step_;
            ++done;
        }
        return SB200_OK;
    }

    int synchronize() {
        if (checked_step_ != step_) {  // the monitor over the current level of every shot
            if (int rc = enqueue_monitor(static_cast<int>(step_ & 1))) return rc;
            checked_step_ = step_;
        }
        if (int rc = cuda(cudaStreamSynchronize(st_))) return rc;
        int e = 0;
        if (int rc = cuda(cudaMemcpy(&e, err_, sizeof(int), cudaMemcpyDeviceToHost))) return rc;
        if (e) return set_error(SB200_ERR_DEVICE, "sb200_batch: a kernel's bounded wait gave up");
        std::vector<int> f(static_cast<size_t>(n_shots()));
        if (int rc = cuda(cudaMemcpy(f.data(), mon_, sizeof(int) * f.size(), cudaMemcpyDeviceToHost)))
            return rc;
        for (int k = 0; k < n_shots(); ++k)
            if (f[k])
                return set_error(SB200_ERR_MONITOR,
                                 "sb200_batch: stability monitor tripped on shot " + std::to_string(k) +
                                     " (non-finite value or |p| above the limit)");
        return SB200_OK;
    }

    // Per-shot FP64 statistics of level `par` and the monitor check: a
    // non-finite value, or (FP32) |p| above the limit, sets the shot's flag.
    // FP16 checks for non-finite values (the stored field is scaled).
    int enqueue_monitor(int par) {
        for (int s = 0; s < n_shots(); ++s) {
            const Shot& h = shots_[s];
            const sb200_grid gg = to_grid(h.g);
            const int rc =
                f16_ ? sb200_field_stats_f16(reinterpret_cast<const uint16_t*>(arena_ + h.off[par]),
                                             &gg, 1.f, stats_ + 3 * s, scratch_, scratch_len_, st_)
                     : sb200_field_stats_f32(reinterpret_cast<const float*>(arena_ + h.off[par]),
                                             &gg, stats_ + 3 * s, scratch_, scratch_len_, st_);
            if (rc) return rc;
            batch_monitor_kernel<<<1, 1, 0, st_>>>(stats_ + 3 * s, mon_ + s,
                                                   f16_ ? 1e300 : monitor_limit_);
        }
        return cuda(cudaGetLastError());
    }

    int set_monitor_limit(float limit) {
        if (!(limit > 0.f)) return set_error(SB200_ERR_INVALID, "sb200_batch_set_monitor_limit: limit <= 0");
        monitor_limit_ = limit;
        return SB200_OK;
    }

    int monitor_flags(int* out) {
        if (!out) return set_error(SB200_ERR_INVALID, "sb200_batch_monitor_flags: NULL output");
        if (checked_step_ != step_) {
            if (int rc = enqueue_monitor(static_cast<int>(step_ & 1))) return rc;
            checked_step_ = step_;
        }
        if (int rc = cuda(cudaMemcpyAsync(out, mon_, sizeof(int) * n_shots(), cudaMemcpyDeviceToHost, st_)))
            return rc;
        return cuda(cudaStreamSynchronize(st_));
    }

    int get_field(int s, float* out) {
        if (s < 0 || s >= n_shots() || !out)
            return set_error(SB200_ERR_INVALID, "sb200_batch_get_field: bad shot or NULL output");
        if (int rc = synchronize()) return rc;
        const Shot& h = shots_[s];
        if (f16_) {  // FP16 level -> FP32 in p's units (divided by the shot's scale)
            F16Scale sc;
            if (int rc = cuda(cudaMemcpy(&sc, scale_ + s, sizeof(sc), cudaMemcpyDeviceToHost)))
                return rc;
            if (int rc = sb200_f16_unpack(reinterpret_cast<const uint16_t*>(arena_ + h.off[step_ & 1]),
                                          staging_, h.g.size(), sc.a, st_))
                return rc;
            // on the batch's (non-blocking) stream, behind the unpack: a plain
            // cudaMemcpy would not wait for it
            if (int rc = cuda(cudaMemcpyAsync(out, staging_, static_cast<size_t>(h.g.size()) * 4,
                                              cudaMemcpyDeviceToHost, st_)))
                return rc;
            return cuda(cudaStreamSynchronize(st_));
        }
        return cuda(cudaMemcpy(out, arena_ + h.off[step_ & 1], static_cast<size_t>(h.g.size()) * 4,
                               cudaMemcpyDeviceToHost));
    }

    int get_trace(int s, float* out, int64_t n) {
        if (s < 0 || s >= n_shots() || !out || n < 0 || n > step_)
            return set_error(SB200_ERR_INVALID, "sb200_batch_get_trace: bad shot, output or count");
        if (int rc = synchronize()) return rc;
        return cuda(cudaMemcpy(out, trace_ + s * cap_, sizeof(float) * n, cudaMemcpyDeviceToHost));
    }

    // Times every (tile variant, z-chunk length) on the batch's own buffers,
    // keeps the fastest, then clears the fields, traces and step count.
    int tune(int reps) {
        reps = std::max(1, reps);
        cudaEvent_t e0, e1;
        if (int rc = cuda(cudaEventCreate(&e0))) return rc;
        if (int rc = cuda(cudaEventCreate(&e1))) {
            cudaEventDestroy(e0);
            return rc;
        }
        // every candidate runs 2 + 2 * reps steps from step index 0: the source
        // tables hold max_steps samples
        reps = static_cast<int>(std::min<int64_t>(reps, std::max<int64_t>(1, (cap_ - 2) / 2)));
        if (cap_ < 4) return set_error(SB200_ERR_INVALID, "sb200_batch_tune: max_steps below 4");
        BatchChoice best;
        best.ms = 1e30f;
        int rc = SB200_OK;
        for (int v = 0; v < variant_count() && !rc; ++v) {
            for (int zl : kZlens) {
                variant_ = v;
                zlen_ = zl;
                if ((rc = build())) break;
                if ((rc = reset_clock())) break;
                if ((rc = launch(0, 0))) break;  // warm-up
                if ((rc = launch(1, 0))) break;
                if ((rc = cuda(cudaEventRecord(e0, st_)))) break;
                for (int k = 0; k < 2 * reps && !rc; ++k) rc = launch(k & 1, 0);
                if (rc || (rc = cuda(cudaEventRecord(e1, st_)))) break;
                if ((rc = cuda(cudaEventSynchronize(e1)))) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                ms /= float(2 * reps);
                if (ms < best.ms) {
                    best.variant = v;
                    best.zlen = zl;
                    best.ms = ms;
                }
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc) return rc;
        if (int r2 = synchronize()) return r2;
        variant_ = best.variant;
        zlen_ = best.zlen;
        {
            std::lock_guard<std::mutex> lock(g_choice_mu);
            if (!g_choices) g_choices = new std::map<std::string, BatchChoice>();
            (*g_choices)[key()] = best;
        }
        if (int r2 = build()) return r2;
        if (int r2 = cuda(cudaMemsetAsync(arena_, 0, arena_bytes_, st_))) return r2;
        step_ = 0;
        if (int r2 = reset_clock()) return r2;
        return cuda(cudaStreamSynchronize(st_));
    }

    int set_choice(int v, int zlen) {
        if (v < 0 || v >= variant_count() || zlen < 0)
            return set_error(SB200_ERR_INVALID, "sb200_batch_set_choice: bad variant or z length");
        if (int rc = synchronize()) return rc;
        variant_ = v;
        zlen_ = zlen;
        return build();
    }

    void choice(int* v, int* zlen, int* items, int* ctas) const {
        if (v) *v = variant_;
        if (zlen) *zlen = zlen_;
        if (items) *items = n_items_;
        if (ctas) *ctas = static_cast<int>(ctas_);
    }

    int n_shots() const { return static_cast<int>(shots_.size()); }
    int64_t steps_done() const { return step_; }
    cudaStream_t stream() const { return st_; }

private:
    struct Shot {
        GridDesc g;
        int64_t src = -1;
        size_t off[3] = {0, 0, 0};  // level 0, level 1, vel2
    };

    int cuda(cudaError_t e) {
        if (e == cudaSuccess) return SB200_OK;
        return set_error(SB200_ERR_CUDA, std::string("sb200_batch: ") + cudaGetErrorString(e));
    }
    int alloc(void** p, size_t bytes) { return cuda(cudaMalloc(p, std::max<size_t>(bytes, 16))); }

    // Zeroes the trace table and the work queue (step index 0).
    int reset_clock() {
        if (int rc = cuda(cudaMemsetAsync(trace_, 0, sizeof(float) * cap_ * n_shots(), st_))) return rc;
        return cuda(cudaMemsetAsync(queue_, 0, sizeof(BatchQueue), st_));
    }

    std::string key() const {
        std::string k = f16_ ? "f16" : "f32";
        for (const Shot& h : shots_)
            k += ":" + std::to_string(h.g.nx) + "x" + std::to_string(h.g.ny) + "x" +
                 std::to_string(h.g.nz);
        int dev = 0;
        cudaGetDevice(&dev);
        return k + "@" + std::to_string(dev);
    }

    bool cached_choice(BatchChoice* c) const {
        std::lock_guard<std::mutex> lock(g_choice_mu);
        if (!g_choices) return false;
        auto it = g_choices->find(key());
        if (it == g_choices->end()) return false;
        *c = it->second;
        return true;
    }

    // Shot tables (both parities) and the work list for the current choice.
    int build() {
        drop_graphs();
        const int n = n_shots();
        const PencilBoxes bx = f16_ ? batch_f16_boxes(variant_) : batch_f32_boxes(variant_);
        std::vector<ShotF32> tab[2];
        std::vector<ShotF16> tab16[2];
        for (int par = 0; par < 2; ++par) {
            if (f16_)
                tab16[par].resize(n);
            else
                tab[par].resize(n);
        }
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
            return shots_[a].g.interior() > shots_[b].g.interior();
        });
        std::vector<int4> items;
        std::vector<int> tiles_x(n), tiles_y(n), zlen(n);
        for (int s = 0; s < n; ++s) {
            const Shot& h = shots_[s];
            const int inz = static_cast<int>(h.g.nz - 8);
            const int zc = zlen_ > 0 ? (inz + zlen_ - 1) / zlen_ : 1;
            for (int par = 0; par < 2; ++par) {
                char* cur = arena_ + h.off[par];
                char* prev = arena_ + h.off[par ^ 1];
                char* vel = arena_ + h.off[2];
                SourceDesc src;
                if (h.src >= 0) {
                    src.idx = h.src;
                    src.wavelet = wave_ + s * cap_;
                    src.step = &queue_->step;
                    src.step_offset = 0;
                    src.trace = trace_ + s * cap_;
                }
                CUtensorMap *mp, *mq, *mv;
                if (f16_) {
                    ShotF16& d = tab16[par][s];
                    std::memset(&d, 0, sizeof(d));
                    mp = &d.p;
                    mq = &d.prev;
                    mv = &d.k;
                    d.args = batch_f16_shot_args(variant_, h.g, zc, reinterpret_cast<uint16_t*>(prev),
                                                 src, scale_ + s, err_);
                    tiles_x[s] = d.args.tiles_x;
                    tiles_y[s] = d.args.tiles_y;
                    zlen[s] = d.args.zlen;
                } else {
                    ShotF32& d = tab[par][s];
                    std::memset(&d, 0, sizeof(d));
                    mp = &d.p;
                    mq = &d.prev;
                    mv = &d.vel2;
                    d.args = batch_f32_shot_args(variant_, h.g, zc, reinterpret_cast<float*>(prev), src,
                                                 err_);
                    d.args.vel2 = reinterpret_cast<const float*>(vel);
                    tiles_x[s] = d.args.tiles_x;
                    tiles_y[s] = d.args.tiles_y;
                    zlen[s] = d.args.zlen;
                }
                int rc = tensor_map_3d(mp, cur, h.g.nx, h.g.ny, h.g.nz, esz_, bx.halo_x, bx.halo_y);
                if (!rc) rc = tensor_map_3d(mq, prev, h.g.nx, h.g.ny, h.g.nz, esz_, bx.tile_x, bx.tile_y);
                if (!rc) rc = tensor_map_3d(mv, vel, h.g.nx, h.g.ny, h.g.nz, esz_, bx.tile_x, bx.tile_y);
                if (rc)
                    return set_error(SB200_ERR_CUDA, "sb200_batch: tensor map encoding failed (" +
                                                         std::to_string(rc) + ")");
            }
        }
        for (int s : order) {
            const int inz = static_cast<int>(shots_[s].g.nz - 8);
            const int zc = (inz + zlen[s] - 1) / zlen[s];
            for (int z = 0; z < zc; ++z)
                for (int y = 0; y < tiles_y[s]; ++y)
                    for (int x = 0; x < tiles_x[s]; ++x) items.push_back(make_int4(s, x, y, z));
        }
        for (int par = 0; par < 2; ++par) {
            const void* src = f16_ ? static_cast<const void*>(tab16[par].data())
                                   : static_cast<const void*>(tab[par].data());
            if (int rc = cuda(cudaMemcpyAsync(table_[par], src, shot_bytes() * n,
                                              cudaMemcpyHostToDevice, st_)))
                return rc;
        }
        if (static_cast<int>(items.size()) > items_cap_) {
            if (items_) cudaFree(items_);
            items_ = nullptr;
            if (int rc = alloc(reinterpret_cast<void**>(&items_), sizeof(int4) * items.size())) return rc;
            items_cap_ = static_cast<int>(items.size());
        }
        if (int rc = cuda(cudaMemcpyAsync(items_, items.data(), sizeof(int4) * items.size(),
                                          cudaMemcpyHostToDevice, st_)))
            return rc;
        n_items_ = static_cast<int>(items.size());
        int sms = 148;
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaGetLastError();
        const int resident = f16_ ? batch_f16_resident(variant_) : batch_f32_resident(variant_);
        ctas_ = static_cast<unsigned>(std::min<int64_t>(int64_t(sms) * resident, std::max(1, n_items_)));
        // the host copies above read std::vectors that go out of scope here
        return cuda(cudaStreamSynchronize(st_));
    }

    // FP16: the exact-y form when every shot has dx == dy (per-shot bits then
    // equal the single-grid FP16 step's on that shot's grid).
    bool exact_y() const {
        for (const Shot& h : shots_)
            if (!f16_exact_y(h.g)) return false;
        return true;
    }

    int launch(int par, int phase) {
        const cudaError_t e =
            f16_ ? launch_batch_f16(variant_, static_cast<const ShotF16*>(table_[par]), items_,
                                    n_items_, queue_, ctas_, phase, exact_y(), st_)
                 : launch_batch_f32(variant_, static_cast<const ShotF32*>(table_[par]), items_,
                                    n_items_, queue_, ctas_, st_);
        return cuda(e);
    }

    // Step number k of the run (level parity par).  FP16: step k % kRenorm == 0
    // renormalises every shot's scale from its FP64 statistics first and runs
    // as phase 1, the next step as phase 2.
    int step_once(int64_t k, int par) {
        int phase = 0;
        if (f16_) {
            const int64_t r = k % kRenorm;
            if (r == 0) {
                if (int rc = renorm_all(par)) return rc;
                phase = 1;
            } else if (r == 1) {
                phase = 2;
            }
        }
        return launch(par, phase);
    }

    int renorm_all(int par) {
        for (int s = 0; s < n_shots(); ++s) {
            const Shot& h = shots_[s];
            const sb200_grid gg = to_grid(h.g);
            if (int rc = sb200_field_stats_f16(reinterpret_cast<const uint16_t*>(arena_ + h.off[par]),
                                               &gg, 1.f, stats_ + 3 * s, scratch_, scratch_len_, st_))
                return rc;
            batch_monitor_kernel<<<1, 1, 0, st_>>>(stats_ + 3 * s, mon_ + s, 1e300);
            if (int rc = sb200_f16_renorm(stats_ + 3 * s, reinterpret_cast<sb200_f16_scale*>(scale_ + s),
                                          bound_ + s * cap_, &queue_->step, 0.f, kTarget, st_))
                return rc;
        }
        return SB200_OK;
    }

    int capture(int par, cudaGraphExec_t* out) {
        cudaGraph_t g = nullptr;
        if (int rc = cuda(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal))) return rc;
        int rc = SB200_OK;
        for (int k = 0; k < chunk_ && !rc; ++k) rc = step_once(k, (par + k) & 1);
        if (!rc && !f16_) rc = enqueue_monitor((par + chunk_) & 1);  // FP32: at every chunk end
        const cudaError_t e = cudaStreamEndCapture(st_, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (int r2 = cuda(e)) return r2;
        rc = cuda(cudaGraphInstantiate(out, g, 0));
        cudaGraphDestroy(g);
        return rc;
    }

    int variant_count() const { return f16_ ? batch_f16_variant_count() : batch_f32_variant_count(); }
    size_t shot_bytes() const { return f16_ ? sizeof(ShotF16) : sizeof(ShotF32); }

    static sb200_grid to_grid(const GridDesc& g) {
        sb200_grid gg{};
        gg.nx = g.nx;
        gg.ny = g.ny;
        gg.nz = g.nz;
        gg.dx = g.dx;
        gg.dy = g.dy;
        gg.dz = g.dz;
        gg.dt = g.dt;
        return gg;
    }

    // FP16: the shot's fields go through the FP32 staging buffer: p and p_prev
    // packed at the initial power-of-two scale (target / (max |p| + the source
    // bound of the first window)), vel2 to K in BF16.
    int set_fields_f16(int s, const float* p, const float* p_prev, const float* vel2, int cur) {
        const Shot& h = shots_[s];
        const int64_t n = h.g.size();
        double m = 0.0;
        for (int64_t i = 0; i < n; ++i)
            m = std::max(m, std::max(std::fabs(double(p[i])), std::fabs(double(p_prev[i]))));
        vel2_src_[s] = h.src >= 0 ? vel2[h.src] : 0.f;
        const std::vector<float> b = host_bound(s);
        const double bnd = b.empty() ? 0.0 : b[0];
        double a0 = 1.0;
        if (m + bnd > 0.0)
            a0 = std::ldexp(1.0, std::max(-120, std::min(120, int(std::floor(std::log2(
                                                                  double(kTarget) / (m + bnd)))))));
        const F16Scale s0{static_cast<float>(a0), 1.f};
        if (int rc = cuda(cudaMemcpyAsync(scale_ + s, &s0, sizeof(s0), cudaMemcpyHostToDevice, st_)))
            return rc;
        const size_t bytes = static_cast<size_t>(n) * 4;
        const sb200_grid gg = to_grid(h.g);
        struct Part {
            const float* host;
            int level;  // index into the shot's offsets: current, previous, K (2)
        };
        const Part parts[3] = {{p, cur}, {p_prev, cur ^ 1}, {vel2, 2}};
        for (const Part& part : parts) {
            if (int rc = cuda(cudaMemcpyAsync(staging_, part.host, bytes, cudaMemcpyHostToDevice, st_)))
                return rc;
            uint16_t* dst = reinterpret_cast<uint16_t*>(arena_ + h.off[part.level]);
            const int rc = part.level == 2 ? sb200_k_field_bf16(staging_, dst, &gg, st_)
                                           : sb200_f16_pack(staging_, dst, n, float(a0), st_);
            if (rc) return rc;
            // the staging buffer is reused by the next part
            if (int r2 = cuda(cudaStreamSynchronize(st_))) return r2;
        }
        return upload_bound(s);
    }

    // bound[k] = 2 x sum over the renormalisation window from step k of
    // |dt^2 vel2[src] w|: the most the source can add to |p| before the next
    // renormalisation (2x: the wave can focus).
    std::vector<float> host_bound(int s) const {
        const std::vector<float>& w = wave_host_[s];
        const int64_t n = static_cast<int64_t>(w.size());
        std::vector<float> b(std::max<int64_t>(n, 1), 0.f);
        if (shots_[s].src < 0 || n == 0) return b;
        const double k = double(shots_[s].g.dt) * shots_[s].g.dt * vel2_src_[s];
        double acc = 0.0;
        for (int64_t j = n - 1; j >= 0; --j) {
            acc += std::fabs(k * w[j]);
            if (j + kRenorm < n) acc -= std::fabs(k * w[j + kRenorm]);
            b[j] = static_cast<float>(2.0 * acc);
        }
        return b;
    }

    int upload_bound(int s) {
        std::vector<float> b = host_bound(s);
        b.resize(static_cast<size_t>(cap_), 0.f);
        if (int rc = cuda(cudaMemcpyAsync(bound_ + s * cap_, b.data(), sizeof(float) * cap_,
                                          cudaMemcpyHostToDevice, st_)))
            return rc;
        return cuda(cudaStreamSynchronize(st_));
    }

    void drop_graphs() {
        for (auto& g : graph_)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }

    static constexpr int kRenorm = 50;        // FP16: steps between renormalisations
    static constexpr float kTarget = 4096.f;  // FP16: scaled max |p| aimed for

    std::vector<Shot> shots_;
    char* arena_ = nullptr;
    size_t arena_bytes_ = 0;
    void* table_[2] = {nullptr, nullptr};  // ShotF32 or ShotF16 tables
    bool f16_ = false;
    int esz_ = 4;
    int64_t max_points_ = 0;
    F16Scale* scale_ = nullptr;  // FP16: per-shot scale
    double* stats_ = nullptr;    // per-shot FP64 statistics (3 each)
    int* mon_ = nullptr;         // per-shot monitor flags (1: tripped)
    double monitor_limit_ = 1e30;
    int64_t checked_step_ = -1;  // step count at the last monitor check
    double* scratch_ = nullptr;
    int64_t scratch_len_ = 0;
    float* bound_ = nullptr;    // FP16: per-shot source bound per step (max_steps each)
    float* staging_ = nullptr;  // FP16: one shot's FP32 field
    std::vector<std::vector<float>> wave_host_;
    std::vector<float> vel2_src_;

    BatchQueue* queue_ = nullptr;
    int4* items_ = nullptr;
    int items_cap_ = 0;
    int n_items_ = 0;
    unsigned ctas_ = 1;
    float* wave_ = nullptr;
    float* trace_ = nullptr;
    int64_t cap_ = 0;
    int chunk_ = 0;
    int variant_ = 0;
    int zlen_ = 64;
    int* err_ = nullptr;
    cudaStream_t st_ = nullptr;
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};
    int64_t step_ = 0;
};

Batch* as_batch(void* h) { return static_cast<Batch*>(h); }

}  // namespace
}  // namespace sb200

using namespace sb200;

extern "C" {

void sb200_batch_config_init(sb200_batch_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->precision = SB200_PRECISION_F32;
    cfg->graph_chunk = 100;
    cfg->max_steps = 1000;
}

int sb200_batch_create(const sb200_shot* shots, int n_shots, const sb200_batch_config* cfg,
                       void** handle) {
    if (!cfg || !handle) return set_error(SB200_ERR_INVALID, "sb200_batch_create: NULL argument");
    *handle = nullptr;
    Batch* b = new Batch();
    const int rc = b->init(shots, n_shots, *cfg);
    if (rc) {
        delete b;
        return rc;
    }
    *handle = b;
    return SB200_OK;
}

int sb200_batch_destroy(void* h) {
    delete as_batch(h);
    return SB200_OK;
}

#define SB200_BATCH_OR_FAIL(h) \
    if (!(h)) return set_error(SB200_ERR_INVALID, "NULL batch handle")

int sb200_batch_set_fields(void* h, int shot, const float* p, const float* p_prev,
                           const float* vel2) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->set_fields(shot, p, p_prev, vel2);
}

int sb200_batch_set_wavelet(void* h, int shot, const float* w, int64_t n) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->set_wavelet(shot, w, n);
}

int sb200_batch_steps(void* h, int64_t n) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->steps(n);
}

int sb200_batch_synchronize(void* h) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->synchronize();
}

int sb200_batch_get_field(void* h, int shot, float* out) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->get_field(shot, out);
}

int sb200_batch_get_trace(void* h, int shot, float* out, int64_t n) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->get_trace(shot, out, n);
}

int sb200_batch_tune(void* h, int reps) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->tune(reps);
}

int sb200_batch_set_monitor_limit(void* h, float limit) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL batch handle");
    return as_batch(h)->set_monitor_limit(limit);
}

int sb200_batch_monitor_flags(void* h, int* flags) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL batch handle");
    return as_batch(h)->monitor_flags(flags);
}

int sb200_batch_set_choice(void* h, int variant, int zlen) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->set_choice(variant, zlen);
}

int sb200_batch_choice(void* h, int* variant, int* zlen, int* n_items, int* ctas) {
    SB200_BATCH_OR_FAIL(h);
    as_batch(h)->choice(variant, zlen, n_items, ctas);
    return SB200_OK;
}

int64_t sb200_batch_steps_done(void* h) {
    SB200_BATCH_OR_FAIL(h);
    return as_batch(h)->steps_done();
}

void* sb200_batch_stream(void* h) { return h ? static_cast<void*>(as_batch(h)->stream()) : nullptr; }

int sb200_batch_variant_count(void) { return batch_f32_variant_count(); }

const char* sb200_batch_variant_name(int v) { return batch_f32_variant_name(v); }

int sb200_batch_variant_count_f16(void) { return batch_f16_variant_count(); }

const char* sb200_batch_variant_name_f16(int v) { return batch_f16_variant_name(v); }

}  // extern "C"
