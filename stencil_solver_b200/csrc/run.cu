// Run engine: the device state of one simulation and its time loop, behind the
// C ABI handle API (sb200_run_*) and the C++ solvers of stencil::make_solver.
//
// Replaces the reference's SolverBase / WavePropSolver / HeatDiffusionSolver
// (src/solver/solver_base.cpp:28-133, wave_prop.cpp:67-75,
// heat_diffusion.cpp:73-122) with a B200 layout: two time levels (in-place
// leapfrog) instead of a three-level ring, a dedicated scalar-diffusivity heat
// kernel instead of the wave kernel on an alpha field plus a copy per step, and
// CUDA-graph replay of step chunks.
//
// Chunk schedule (C = graph chunk, even so that the two time levels return to
// their buffers):
//   FP32 acoustic / heat : C steps, then FP64 statistics + monitor check;
//   FP16 acoustic        : statistics(p) -> monitor check -> renormalise ->
//                          step (phase 1) -> step (phase 2) -> C-2 plain steps,
//                          with C = the renormalisation interval.
// Source samples are read on the device at wavelet[*step + k] (the host sets
// *step before each replay), so one captured graph serves every chunk; the
// injecting thread writes the trace at the same index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dispatch.h"
#include "kernels.h"
#include "stencil_b200.h"

namespace sb200 {

namespace {

__global__ void monitor_kernel(const double* stats3, int* flag, double limit) {
    if (!(stats3[2] == 0.0) || !(stats3[1] <= limit)) atomicExch(flag, 1);
}

constexpr int64_t kStageFloats = int64_t(1) << 24;  // host <-> device staging: 64 MB

class Run {
public:
    int init(const sb200_run_config& c) {
        c_ = c;
        if (c_.renorm_every <= 0) c_.renorm_every = 50;
        if (c_.monitor_limit <= 0.f) c_.monitor_limit = 1e30f;
        if (c_.f16_target <= 0.f) c_.f16_target = 4096.f;
        c_.graph_chunk = c_.graph_chunk > 0 ? std::max(2, c_.graph_chunk & ~1) : 0;
        const sb200_grid& gr = c_.grid;
        if (gr.nx <= 8 || gr.ny <= 8 || gr.nz <= 8)
            return set_error(SB200_ERR_INVALID, "sb200_run_create: every extent must exceed 8");
        if (!(gr.dx > 0) || !(gr.dy > 0) || !(gr.dz > 0) || !(gr.dt > 0))
            return set_error(SB200_ERR_INVALID, "sb200_run_create: spacing and dt must be positive");
        heat_ = c_.physics == SB200_PHYSICS_HEAT;
        fp16_ = c_.precision == SB200_PRECISION_F16;
        if (c_.physics != SB200_PHYSICS_WAVE && !heat_)
            return set_error(SB200_ERR_INVALID, "sb200_run_create: unknown physics");
        if (c_.precision != SB200_PRECISION_F32 && !fp16_)
            return set_error(SB200_ERR_INVALID, "sb200_run_create: unknown precision");
        if (fp16_ && heat_)
            return set_error(SB200_ERR_UNSUPPORTED, "sb200_run_create: FP16 storage is acoustic only");
        if (fp16_ && (gr.nx % 8 != 0))
            return set_error(SB200_ERR_UNSUPPORTED, "sb200_run_create: FP16 storage needs nx % 8 == 0");
        if (fp16_ && (c_.renorm_every < 2 || c_.renorm_every % 2))
            return set_error(SB200_ERR_INVALID, "sb200_run_create: renorm_every must be even >= 2");
        if (fp16_ && c_.exact)
            return set_error(SB200_ERR_INVALID, "sb200_run_create: exact is FP32 only");
        if (heat_ && c_.src_index >= 0)
            return set_error(SB200_ERR_INVALID, "sb200_run_create: the heat run takes no source");
        n_ = gr.nx * gr.ny * gr.nz;
        if (c_.src_index >= n_) return set_error(SB200_ERR_INVALID, "sb200_run_create: bad source");
        if (fp16_) c_.graph_chunk = c_.graph_chunk ? c_.renorm_every : 0;

        if (int rc = cuda(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking))) return rc;
        const size_t es = fp16_ ? 2 : 4;
        if (int rc = alloc(&a_, n_ * es)) return rc;
        if (int rc = alloc(&b_, n_ * es)) return rc;
        if (!heat_) {
            if (fp16_) {
                if (int rc = alloc(reinterpret_cast<void**>(&k_), n_ * 2)) return rc;
            } else if (int rc = alloc(reinterpret_cast<void**>(&vel2_), n_ * 4)) {
                return rc;
            }
        }
        if (int rc = alloc(reinterpret_cast<void**>(&step_dev_), sizeof(int))) return rc;
        scratch_len_ = sb200_field_stats_scratch_len(&c_.grid);
        if (int rc = alloc(reinterpret_cast<void**>(&stats_dev_), 3 * sizeof(double))) return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&scratch_dev_), scratch_len_ * sizeof(double)))
            return rc;
        if (int rc = alloc(reinterpret_cast<void**>(&monitor_dev_), sizeof(int))) return rc;
        if (fp16_) {
            if (int rc = alloc(reinterpret_cast<void**>(&scale_dev_), sizeof(F16Scale))) return rc;
        }
        home_ = a_;
        if (int rc = cuda(cudaMemsetAsync(a_, 0, n_ * es, st_))) return rc;
        if (int rc = cuda(cudaMemsetAsync(b_, 0, n_ * es, st_))) return rc;
        if (int rc = cuda(cudaMemsetAsync(monitor_dev_, 0, sizeof(int), st_))) return rc;
        if (!heat_ && c_.src_index >= 0 && c_.src_freq > 0.f) {
            const double t0 = c_.src_t0 >= 0.f ? c_.src_t0 : 1.0 / c_.src_freq;
            std::vector<float> w(4096);
            sb200_ricker(c_.src_freq, t0, c_.grid.dt, static_cast<int64_t>(w.size()), w.data());
            if (int rc = set_wavelet(w.data(), static_cast<int64_t>(w.size()), true)) return rc;
        }
        return cuda(cudaStreamSynchronize(st_));
    }

    ~Run() {
        if (st_) cudaStreamSynchronize(st_);
        drop_graphs();
        for (void* p : {a_, b_, static_cast<void*>(vel2_), static_cast<void*>(k_),
                        static_cast<void*>(wavelet_dev_), static_cast<void*>(trace_dev_),
                        static_cast<void*>(bound_dev_), static_cast<void*>(step_dev_),
                        static_cast<void*>(stats_dev_), static_cast<void*>(scratch_dev_),
                        static_cast<void*>(monitor_dev_), static_cast<void*>(scale_dev_),
                        static_cast<void*>(stage_)})
            if (p) cudaFree(p);
        if (st_) cudaStreamDestroy(st_);
    }

    int set_fields(const float* p, const float* p_prev, const float* vel2) {
        if (!p) return set_error(SB200_ERR_INVALID, "sb200_run_set_fields: p is NULL");
        if (!heat_ && !vel2) return set_error(SB200_ERR_INVALID, "sb200_run_set_fields: vel2 is NULL");
        if (!p_prev) p_prev = p;
        step_ = 0;
        if (int rc = cuda(cudaMemsetAsync(monitor_dev_, 0, sizeof(int), st_))) return rc;
        if (!fp16_) {
            if (int rc = cuda(cudaMemcpyAsync(a_, p, n_ * 4, cudaMemcpyHostToDevice, st_))) return rc;
            if (heat_) {  // both levels carry the caller's halo (never written)
                if (int rc = cuda(cudaMemcpyAsync(b_, p, n_ * 4, cudaMemcpyHostToDevice, st_)))
                    return rc;
            } else {
                if (int rc = cuda(cudaMemcpyAsync(b_, p_prev, n_ * 4, cudaMemcpyHostToDevice, st_)))
                    return rc;
                if (int rc = cuda(cudaMemcpyAsync(vel2_, vel2, n_ * 4, cudaMemcpyHostToDevice, st_)))
                    return rc;
                vel2_host_src_ = c_.src_index >= 0 ? vel2[c_.src_index] : 0.f;
            }
            return cuda(cudaStreamSynchronize(st_));
        }
        // FP16: initial scale from the host fields and the first window's source.
        double m = 0.0;
        for (int64_t i = 0; i < n_; ++i)
            m = std::max(m, std::max(std::fabs(double(p[i])), std::fabs(double(p_prev[i]))));
        vel2_host_src_ = c_.src_index >= 0 ? vel2[c_.src_index] : 0.f;
        rebuild_bound();
        const double bnd = bound_host_.empty() ? 0.0 : bound_host_[0];
        double a0 = 1.0;
        if (m + bnd > 0.0)
            a0 = std::ldexp(1.0, std::max(-120, std::min(120, int(std::floor(std::log2(
                                                                  double(c_.f16_target) / (m + bnd)))))));
        const F16Scale s0{static_cast<float>(a0), 1.f};
        // on the run's stream: steps still queued there read the scale
        if (int rc = cuda(cudaMemcpyAsync(scale_dev_, &s0, sizeof(s0), cudaMemcpyHostToDevice, st_)))
            return rc;
        if (int rc = stage_in(p, a_, float(a0), false)) return rc;
        if (int rc = stage_in(p_prev, b_, float(a0), false)) return rc;
        if (int rc = stage_in(vel2, k_, 1.f, true)) return rc;
        return cuda(cudaStreamSynchronize(st_));
    }

    // generated: the samples are the run's own Ricker, which steps() extends on
    // demand; caller samples are used as given and bound the run's length.
    int set_wavelet(const float* w, int64_t n, bool generated = false) {
        if (!w || n <= 0) return set_error(SB200_ERR_INVALID, "sb200_run_set_wavelet: bad samples");
        if (heat_ || c_.src_index < 0)
            return set_error(SB200_ERR_INVALID, "sb200_run_set_wavelet: the run has no source");
        ricker_ = generated;
        wavelet_host_.assign(w, w + n);
        if (int rc = upload_tables(std::max<int64_t>(n, cap_))) return rc;
        rebuild_bound();
        return SB200_OK;
    }

    int steps(int64_t n) {
        if (n < 0) return set_error(SB200_ERR_INVALID, "sb200_run_steps: negative count");
        if (!heat_ && c_.src_index >= 0) {
            if (ricker_ && step_ + n + 2 > static_cast<int64_t>(wavelet_host_.size())) {
                if (int rc = grow_ricker(step_ + n + 2)) return rc;
            } else if (step_ + n > static_cast<int64_t>(wavelet_host_.size())) {
                return set_error(SB200_ERR_INVALID, "sb200_run_steps: wavelet shorter than the run");
            }
        }
        const int C = c_.graph_chunk;
        int64_t done = 0;
        while (done < n) {
            const bool aligned = !fp16_ || step_ % c_.renorm_every == 0;
            if (C > 0 && aligned && n - done >= C) {
                // a graph bakes in which buffer is current: one per parity
                const int par = a_ == home_ ? 0 : 1;
                if (!graph_[par]) {
                    if (int rc = capture(&graph_[par])) return rc;
                }
                if (int rc = sb200_set_device_int(step_dev_, static_cast<int>(step_), st_)) return rc;
                if (int rc = cuda(cudaGraphLaunch(graph_[par], st_))) return rc;
                step_ += C;
                done += C;
                continue;
            }
            if (int rc = eager_step()) return rc;
            ++done;
        }
        return SB200_OK;
    }

    int synchronize() {
        if (int rc = cuda(cudaStreamSynchronize(st_))) return rc;
        int flag = 0;
        if (int rc = cuda(cudaMemcpy(&flag, monitor_dev_, sizeof(int), cudaMemcpyDeviceToHost)))
            return rc;
        const int dev_err = sb200_device_error(1);
        if (dev_err > 0)
            return set_error(SB200_ERR_DEVICE, "a kernel's bounded wait gave up (device error " +
                                                   std::to_string(dev_err) + ")");
        if (flag)
            return set_error(SB200_ERR_MONITOR,
                             "stability monitor: non-finite value or |p| above the limit");
        return SB200_OK;
    }

    int get_field(float* host) {
        if (!host) return set_error(SB200_ERR_INVALID, "sb200_run_get_field: NULL destination");
        if (int rc = synchronize()) return rc;
        if (!fp16_) return cuda(cudaMemcpy(host, a_, n_ * 4, cudaMemcpyDeviceToHost));
        F16Scale s;
        if (int rc = cuda(cudaMemcpy(&s, scale_dev_, sizeof(s), cudaMemcpyDeviceToHost))) return rc;
        if (int rc = ensure_stage()) return rc;
        for (int64_t off = 0; off < n_; off += kStageFloats) {
            const int64_t m = std::min(kStageFloats, n_ - off);
            if (int rc = sb200_f16_unpack(static_cast<const uint16_t*>(a_) + off, stage_, m, s.a, st_))
                return rc;
            if (int rc = cuda(cudaMemcpyAsync(host + off, stage_, m * 4, cudaMemcpyDeviceToHost, st_)))
                return rc;
        }
        return cuda(cudaStreamSynchronize(st_));
    }

    // XY plane z (nx * ny floats, x fastest) of the current field in physical
    // units: one contiguous range of the z-major field, so only that range
    // crosses to the host (FP16: unpacked on the device first).
    int get_plane(int64_t z, float* host) {
        if (!host) return set_error(SB200_ERR_INVALID, "sb200_run_get_plane: NULL destination");
        const int64_t plane = c_.grid.nx * c_.grid.ny;
        if (z < 0 || z >= c_.grid.nz)
            return set_error(SB200_ERR_INVALID, "sb200_run_get_plane: z outside [0, nz)");
        if (int rc = synchronize()) return rc;
        if (!fp16_)
            return cuda(cudaMemcpy(host, static_cast<const float*>(a_) + z * plane, plane * 4,
                                   cudaMemcpyDeviceToHost));
        F16Scale s;
        if (int rc = cuda(cudaMemcpy(&s, scale_dev_, sizeof(s), cudaMemcpyDeviceToHost))) return rc;
        if (int rc = ensure_stage()) return rc;
        for (int64_t off = 0; off < plane; off += kStageFloats) {
            const int64_t m = std::min(kStageFloats, plane - off);
            if (int rc = sb200_f16_unpack(static_cast<const uint16_t*>(a_) + z * plane + off, stage_,
                                          m, s.a, st_))
                return rc;
            if (int rc = cuda(cudaMemcpyAsync(host + off, stage_, m * 4, cudaMemcpyDeviceToHost, st_)))
                return rc;
        }
        return cuda(cudaStreamSynchronize(st_));
    }

    int get_trace(float* host, int64_t n) {
        if (!host || n < 0) return set_error(SB200_ERR_INVALID, "sb200_run_get_trace: bad arguments");
        if (!trace_dev_ || n > cap_ || n > step_)
            return set_error(SB200_ERR_INVALID, "sb200_run_get_trace: no trace of that length");
        if (int rc = synchronize()) return rc;
        return cuda(cudaMemcpy(host, trace_dev_, n * 4, cudaMemcpyDeviceToHost));
    }

    int stats(double* out3) {
        if (!out3) return set_error(SB200_ERR_INVALID, "sb200_run_stats: NULL destination");
        if (int rc = enqueue_stats()) return rc;
        if (int rc = cuda(cudaStreamSynchronize(st_))) return rc;
        if (int rc = cuda(cudaMemcpy(out3, stats_dev_, 3 * sizeof(double), cudaMemcpyDeviceToHost)))
            return rc;
        if (fp16_) {  // stats of the stored field: bring them to physical units
            F16Scale s;
            if (int rc = cuda(cudaMemcpy(&s, scale_dev_, sizeof(s), cudaMemcpyDeviceToHost))) return rc;
            out3[0] /= double(s.a) * s.a;
            out3[1] /= s.a;
        }
        return SB200_OK;
    }

    int64_t steps_done() const { return step_; }
    cudaStream_t stream() const { return st_; }

private:
    int cuda(cudaError_t e) {
        if (e == cudaSuccess) return SB200_OK;
        return set_error(SB200_ERR_CUDA, std::string("run: ") + cudaGetErrorString(e));
    }
    int alloc(void** p, size_t bytes) { return cuda(cudaMalloc(p, bytes)); }

    int ensure_stage() {
        if (stage_) return SB200_OK;
        return alloc(reinterpret_cast<void**>(&stage_), size_t(kStageFloats) * 4);
    }

    // Host FP32 -> device FP16 (scaled) or BF16 K (vel2 -> vel2 dt^2/dx^2) by chunks.
    int stage_in(const float* host, void* dst, float scale, bool k_field) {
        if (int rc = ensure_stage()) return rc;
        const sb200_grid one = {1, 1, 1, c_.grid.dx, c_.grid.dy, c_.grid.dz, c_.grid.dt};
        for (int64_t off = 0; off < n_; off += kStageFloats) {
            const int64_t m = std::min(kStageFloats, n_ - off);
            if (int rc = cuda(cudaMemcpyAsync(stage_, host + off, m * 4, cudaMemcpyHostToDevice, st_)))
                return rc;
            uint16_t* d = static_cast<uint16_t*>(dst) + off;
            int rc;
            if (k_field) {
                sb200_grid chunk = one;
                chunk.nx = m;
                rc = sb200_k_field_bf16(stage_, d, &chunk, st_);
            } else {
                rc = sb200_f16_pack(stage_, d, m, scale, st_);
            }
            if (rc) return rc;
            // the staging buffer is reused by the next chunk: wait for this one
            if (int rc2 = cuda(cudaStreamSynchronize(st_))) return rc2;
        }
        return SB200_OK;
    }

    // Device wavelet / trace tables of capacity cap (steps); a reallocation
    // invalidates the captured graph.
    int upload_tables(int64_t cap) {
        if (cap > cap_) {
            if (wavelet_dev_) cudaFree(wavelet_dev_);
            if (bound_dev_) cudaFree(bound_dev_);
            float* old_trace = trace_dev_;
            trace_dev_ = nullptr;
            if (int rc = alloc(reinterpret_cast<void**>(&wavelet_dev_), cap * 4)) return rc;
            if (int rc = alloc(reinterpret_cast<void**>(&bound_dev_), cap * 4)) return rc;
            if (int rc = alloc(reinterpret_cast<void**>(&trace_dev_), cap * 4)) return rc;
            if (int rc = cuda(cudaMemsetAsync(trace_dev_, 0, cap * 4, st_))) return rc;
            if (old_trace) {
                if (int rc = cuda(cudaMemcpyAsync(trace_dev_, old_trace, cap_ * 4,
                                                  cudaMemcpyDeviceToDevice, st_)))
                    return rc;
                cudaStreamSynchronize(st_);
                cudaFree(old_trace);
            }
            cap_ = cap;
            drop_graphs();
        }
        std::vector<float> w(cap_, 0.f);
        std::copy(wavelet_host_.begin(),
                  wavelet_host_.begin() + std::min<int64_t>(cap_, wavelet_host_.size()), w.begin());
        if (int rc = cuda(cudaMemcpyAsync(wavelet_dev_, w.data(), cap_ * 4, cudaMemcpyHostToDevice, st_)))
            return rc;
        return cuda(cudaStreamSynchronize(st_));
    }

    int grow_ricker(int64_t need) {
        int64_t n = std::max<int64_t>(need, 2 * static_cast<int64_t>(wavelet_host_.size()));
        std::vector<float> w(n);
        const double t0 = c_.src_t0 >= 0.f ? c_.src_t0 : 1.0 / c_.src_freq;
        sb200_ricker(c_.src_freq, t0, c_.grid.dt, n, w.data());
        wavelet_host_ = w;
        if (int rc = upload_tables(std::max(n, cap_))) return rc;
        rebuild_bound();
        return SB200_OK;
    }

    // FP16: bound[s] = sum over the next renorm window of |dt^2 vel2[src] w|,
    // the most the source can add to |p| before the next renormalisation.
    void rebuild_bound() {
        if (!fp16_) return;
        const int64_t n = static_cast<int64_t>(wavelet_host_.size());
        bound_host_.assign(std::max<int64_t>(n, 1), 0.f);
        if (c_.src_index < 0 || n == 0) return;
        const double k = double(c_.grid.dt) * c_.grid.dt * vel2_host_src_;
        const int W = c_.renorm_every;
        double acc = 0.0;
        for (int64_t s = n - 1; s >= 0; --s) {
            acc += std::fabs(k * wavelet_host_[s]);
            if (s + W < n) acc -= std::fabs(k * wavelet_host_[s + W]);
            bound_host_[s] = static_cast<float>(2.0 * acc);  // 2x: the wave can focus
        }
        if (bound_dev_ && cap_ > 0) {
            std::vector<float> b(cap_, 0.f);
            std::copy(bound_host_.begin(), bound_host_.begin() + std::min<int64_t>(cap_, n), b.begin());
            cudaMemcpyAsync(bound_dev_, b.data(), cap_ * 4, cudaMemcpyHostToDevice, st_);
            cudaStreamSynchronize(st_);
        }
    }

    int enqueue_stats() {
        if (fp16_)
            return sb200_field_stats_f16(static_cast<const uint16_t*>(a_), &c_.grid, 1.f, stats_dev_,
                                         scratch_dev_, scratch_len_, st_);
        return sb200_field_stats_f32(static_cast<const float*>(a_), &c_.grid, stats_dev_,
                                     scratch_dev_, scratch_len_, st_);
    }

    int monitor(double limit) {
        monitor_kernel<<<1, 1, 0, st_>>>(stats_dev_, monitor_dev_, limit);
        return cuda(cudaGetLastError());
    }

    // One step.  device_src: read the source sample / write the trace through
    // the device step counter at offset k (graph capture); otherwise use the host
    // sample of step_ + k and the trace index step_ + k.
    int enqueue_step(bool device_src, int k, int phase) {
        SourceDesc src;
        if (!heat_ && c_.src_index >= 0) {
            src.idx = c_.src_index;
            src.trace = trace_dev_;
            src.step_offset = device_src ? k : static_cast<int>(step_ + k);
            if (device_src) {
                src.wavelet = wavelet_dev_;
                src.step = step_dev_;
            } else {
                src.w = wavelet_host_[static_cast<size_t>(step_ + k)];
            }
        }
        int rc;
        if (heat_) {
            rc = c_.exact ? sb200_heat_step_exact_f32(static_cast<const float*>(a_),
                                                      static_cast<float*>(b_), &c_.grid,
                                                      c_.diffusivity, st_)
                          : sb200_heat_step_f32(static_cast<const float*>(a_),
                                                static_cast<float*>(b_), &c_.grid, c_.diffusivity,
                                                st_);
        } else if (fp16_) {
            rc = dispatch_wave_f16(static_cast<const uint16_t*>(a_), static_cast<uint16_t*>(b_), k_,
                                   &c_.grid, src, reinterpret_cast<const sb200_f16_scale*>(scale_dev_),
                                   phase, st_);
        } else {
            rc = dispatch_wave_f32(static_cast<const float*>(a_), static_cast<const float*>(b_),
                                   vel2_, static_cast<float*>(b_), &c_.grid, src, st_, c_.exact != 0);
        }
        std::swap(a_, b_);
        return rc;
    }

    // Statistics of the current FP16 field -> monitor -> renormalisation.
    int renorm(bool device_bound) {
        if (int rc = enqueue_stats()) return rc;
        if (int rc = monitor(1e300)) return rc;  // non-finite check (stored units)
        const float bh = device_bound || bound_host_.empty()
                             ? 0.f
                             : bound_host_[std::min<size_t>(static_cast<size_t>(step_),
                                                            bound_host_.size() - 1)];
        return sb200_f16_renorm(stats_dev_, reinterpret_cast<sb200_f16_scale*>(scale_dev_),
                                device_bound && bound_dev_ ? bound_dev_ : nullptr, step_dev_, bh,
                                c_.f16_target, st_);
    }

    int eager_step() {
        int phase = 0;
        if (fp16_) {
            const int64_t r = step_ % c_.renorm_every;
            if (r == 0) {
                if (int rc = renorm(false)) return rc;
                phase = 1;
            } else if (r == 1) {
                phase = 2;
            }
        }
        if (int rc = enqueue_step(false, 0, phase)) return rc;
        ++step_;
        if (!fp16_ && c_.monitor_every > 0 && step_ % c_.monitor_every == 0) {
            if (int rc = enqueue_stats()) return rc;
            if (int rc = monitor(c_.monitor_limit)) return rc;
        }
        return SB200_OK;
    }

    void drop_graphs() {
        for (auto& g : graph_)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }

    int capture(cudaGraphExec_t* out) {
        const int C = c_.graph_chunk;
        // Everything a launch sets up on first use (kernel attributes, occupancy
        // queries, the kernel choice, tensor maps) happens before the capture.
        pencil_f32_prepare();
        pencil_f16_prepare();
        int v = 0, z = 0;
        sb200_pencil_choice(heat_ ? SB200_KIND_HEAT_F32
                                  : (fp16_ ? SB200_KIND_WAVE_F16 : SB200_KIND_WAVE_F32),
                            &c_.grid, &v, &z);
        cudaGraph_t g = nullptr;
        if (int rc = cuda(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal))) return rc;
        int rc = SB200_OK;
        if (fp16_ && !rc) rc = renorm(true);
        for (int k = 0; k < C && !rc; ++k)
            rc = enqueue_step(true, k, fp16_ ? (k == 0 ? 1 : (k == 1 ? 2 : 0)) : 0);
        if (!fp16_ && !rc) {
            rc = enqueue_stats();
            if (!rc) rc = monitor(c_.monitor_limit);
        }
        const cudaError_t e = cudaStreamEndCapture(st_, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (int rc2 = cuda(e)) return rc2;
        rc = cuda(cudaGraphInstantiate(out, g, 0));
        cudaGraphDestroy(g);
        return rc;
    }

    sb200_run_config c_{};
    bool heat_ = false, fp16_ = false, ricker_ = false;
    int64_t n_ = 0;
    cudaStream_t st_ = nullptr;
    void* a_ = nullptr;  // current level
    void* b_ = nullptr;  // previous level (acoustic) / next level (heat)
    float* vel2_ = nullptr;
    uint16_t* k_ = nullptr;
    float* wavelet_dev_ = nullptr;
    float* trace_dev_ = nullptr;
    float* bound_dev_ = nullptr;
    int64_t cap_ = 0;
    std::vector<float> wavelet_host_, bound_host_;
    float vel2_host_src_ = 0.f;
    int* step_dev_ = nullptr;
    double* stats_dev_ = nullptr;
    double* scratch_dev_ = nullptr;
    int64_t scratch_len_ = 0;
    int* monitor_dev_ = nullptr;
    F16Scale* scale_dev_ = nullptr;
    float* stage_ = nullptr;
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};
    void* home_ = nullptr;  // buffer that is current at even parity
    int64_t step_ = 0;
};

Run* as_run(void* h) { return static_cast<Run*>(h); }

}  // namespace
}  // namespace sb200

using namespace sb200;

extern "C" {

void sb200_run_config_init(sb200_run_config* cfg, const sb200_grid* grid) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    if (grid) cfg->grid = *grid;
    cfg->physics = SB200_PHYSICS_WAVE;
    cfg->precision = SB200_PRECISION_F32;
    cfg->src_index = -1;
    cfg->src_freq = 15.f;
    cfg->src_t0 = -1.f;
    cfg->graph_chunk = 100;
    cfg->renorm_every = 50;
    cfg->monitor_every = 0;
    cfg->monitor_limit = 1e30f;
    cfg->f16_target = 4096.f;
}

int sb200_run_create(const sb200_run_config* cfg, void** handle) {
    if (!cfg || !handle) return set_error(SB200_ERR_INVALID, "sb200_run_create: NULL argument");
    *handle = nullptr;
    Run* r = new Run();
    const int rc = r->init(*cfg);
    if (rc) {
        delete r;
        return rc;
    }
    *handle = r;
    return SB200_OK;
}

int sb200_run_destroy(void* handle) {
    delete as_run(handle);
    return SB200_OK;
}

int sb200_run_set_fields(void* h, const float* p, const float* p_prev, const float* vel2) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->set_fields(p, p_prev, vel2);
}

int sb200_run_set_wavelet(void* h, const float* w, int64_t n) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->set_wavelet(w, n);
}

int sb200_run_steps(void* h, int64_t n) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->steps(n);
}

int sb200_run_synchronize(void* h) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->synchronize();
}

int sb200_run_get_field(void* h, float* p) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->get_field(p);
}

int sb200_run_get_plane(void* h, int64_t z, float* p) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->get_plane(z, p);
}

int sb200_run_get_trace(void* h, float* trace, int64_t n) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->get_trace(trace, n);
}

int sb200_run_stats(void* h, double* out3) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->stats(out3);
}

int64_t sb200_run_steps_done(void* h) {
    if (!h) return set_error(SB200_ERR_INVALID, "NULL run handle");
    return as_run(h)->steps_done();
}

void* sb200_run_stream(void* h) { return h ? static_cast<void*>(as_run(h)->stream()) : nullptr; }

}  // extern "C"
