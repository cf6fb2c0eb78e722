// Wave and heat solvers behind stencil::make_solver (include/stencil/solver.hpp).
//
// Replace the reference's SolverBase / WavePropSolver / HeatDiffusionSolver
// (src/solver/solver_base.cpp:28-133, wave_prop.cpp:67-75, heat_diffusion.cpp:73-122)
// with a B200 layout:
//   * acoustic: two time levels, p_next written in place over p_prev (the
//     reference keeps three levels and rotates a ring), plus vel2;
//   * heat: two levels ping-ponged by the dedicated scalar-diffusivity kernel
//     (the reference runs the wave kernel on a vel2 field filled with alpha and
//     copies cur -> prev after every step);
//   * run() replays CUDA graphs of graph_chunk steps; the source sample of
//     every captured step is read on the device from the wavelet table at
//     (*step + offset), with *step set before each replay.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "stencil/config.hpp"
#include "stencil/grid.hpp"
#include "stencil/solver.hpp"
#include "stencil/timer.hpp"
#include "stencil_b200.h"

namespace stencil {

namespace {

void cuda_ok(cudaError_t e, const char* where) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[CUDA ERROR] %s: %s\n", where, cudaGetErrorString(e));
        std::exit(EXIT_FAILURE);
    }
}

void abi_ok(int status, const char* where) {
    if (status == SB200_OK) return;
    if (status == SB200_ERR_INVALID || status == SB200_ERR_UNSUPPORTED)
        throw std::invalid_argument(std::string(where) + ": " + sb200_last_error());
    std::fprintf(stderr, "[CUDA ERROR] %s: %s\n", where, sb200_last_error());
    std::exit(EXIT_FAILURE);
}

sb200_grid to_c(const GridDims& g) {
    sb200_grid c;
    c.nx = static_cast<int64_t>(g.nx);
    c.ny = static_cast<int64_t>(g.ny);
    c.nz = static_cast<int64_t>(g.nz);
    c.dx = g.dx;
    c.dy = g.dy;
    c.dz = g.dz;
    c.dt = g.dt;
    return c;
}

class B200Solver : public ISolver {
public:
    ~B200Solver() override { release(); }

    void init(const Config& cfg) override {
        release();
        cfg_ = cfg;
        dims_ = cfg.make_grid();
        if (dims_.nx <= 2 * STENCIL_RADIUS || dims_.ny <= 2 * STENCIL_RADIUS ||
            dims_.nz <= 2 * STENCIL_RADIUS)
            throw std::invalid_argument("make_solver: every extent must exceed 2*STENCIL_RADIUS");
        if (!(dims_.dt > 0)) throw std::invalid_argument("make_solver: dt must be positive");
        cuda_ok(cudaSetDevice(cfg.device), "cudaSetDevice");
        cuda_ok(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        abi_ok(sb200_upload_fd_coefficients(), "upload_fd_coefficients");
        const std::size_t bytes = dims_.size() * sizeof(real_t);
        cuda_ok(cudaMalloc(&a_, bytes), "cudaMalloc");
        cuda_ok(cudaMalloc(&b_, bytes), "cudaMalloc");
        cuda_ok(cudaMalloc(&step_dev_, sizeof(int)), "cudaMalloc");
        setup_fields();
        cuda_ok(cudaStreamSynchronize(stream_), "init");
        if (cfg.verbose) print_grid_info(dims_, name().c_str());
    }

    void step() override {
        one_step_eager();
    }

    PerfResult run(int n_steps, int warmup) override {
        NVTX_PUSH(name().c_str());
        for (int i = 0; i < warmup; ++i) one_step_eager();
        cuda_ok(cudaStreamSynchronize(stream_), "run");
        GpuTimer timer;
        timer.start(stream_);
        advance(n_steps);
        timer.stop(stream_);
        const double ms = double(timer.elapsed_ms()) / std::max(n_steps, 1);
        NVTX_POP();
        PerfResult r;
        r.label = name();
        r.time_ms = ms;
        const double s = ms * 1e-3;
        r.bandwidth_gbs = bytes_per_step() / s / 1e9;
        r.model_bandwidth_gbs = bandwidth_bytes_per_step(dims_) / s / 1e9;
        r.gflops = flops_per_step(dims_) / s / 1e9;
        r.gpts = double(dims_.interior_size()) / s / 1e9;
        r.grid_size = dims_.nx;
        r.dtype = "fp32";
        return r;
    }

    void download(HostGrid& out) const override {
        if (out.data.size() != dims_.size())
            throw std::invalid_argument("download: HostGrid size does not match the solver grid");
        cuda_ok(cudaMemcpyAsync(out.ptr(), a_, out.bytes(), cudaMemcpyDeviceToHost, stream_),
                "download");
        cuda_ok(cudaStreamSynchronize(stream_), "download");
    }

    const GridDims& dims() const override { return dims_; }
    long long steps_taken() const override { return step_; }

protected:
    virtual void setup_fields() = 0;
    virtual void enqueue_step(bool device_source, int step_offset) = 0;
    virtual double bytes_per_step() const = 0;

    std::string variant_name() const {
        switch (cfg_.variant) {
            case KernelVariant::Naive:
                return "naive";
            case KernelVariant::Tiled:
                return "tiled";
            default:
                return "multigpu";
        }
    }
    bool exact() const { return cfg_.variant == KernelVariant::Naive; }

    void one_step_eager() {
        enqueue_step(false, 0);
        swap_levels();
        ++step_;
    }

    // n steps: whole chunks by graph replay, the rest eagerly.
    void advance(int n) {
        const int chunk = std::max(2, cfg_.graph_chunk & ~1);  // even: buffers return home
        int done = 0;
        if (cfg_.use_graphs && n >= chunk) {
            if (!graph_ready_) capture(chunk);
            while (n - done >= chunk) {
                abi_ok(sb200_set_device_int(step_dev_, static_cast<int>(step_), stream_),
                       "set step");
                cuda_ok(cudaGraphLaunch(graph_exec_, stream_), "cudaGraphLaunch");
                step_ += chunk;
                done += chunk;
            }
        }
        for (; done < n; ++done) one_step_eager();
    }

    void capture(int chunk) {
        ensure_wavelet(step_ + chunk);
        cudaGraph_t graph = nullptr;
        cuda_ok(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
        for (int k = 0; k < chunk; ++k) {
            enqueue_step(true, k);
            swap_levels();
        }
        cuda_ok(cudaStreamEndCapture(stream_, &graph), "capture");
        cuda_ok(cudaGraphInstantiate(&graph_exec_, graph, 0), "cudaGraphInstantiate");
        cudaGraphDestroy(graph);
        graph_ready_ = true;
        graph_chunk_ = chunk;
    }

    // Host-side wavelet samples for steps [0, n) and their device copy (the
    // table only grows; a growth invalidates captured graphs).
    void ensure_wavelet(long long n) {
        if (!cfg_.source_enabled) return;
        const long long cap = std::max<long long>(n, 1024);
        if (static_cast<long long>(wavelet_.size()) >= n && wavelet_dev_) return;
        const long long size = std::max<long long>(cap, 2 * static_cast<long long>(wavelet_.size()));
        wavelet_.resize(static_cast<std::size_t>(size));
        const double t0 = cfg_.source_t0 >= 0 ? cfg_.source_t0 : 1.0 / cfg_.source_freq;
        abi_ok(sb200_ricker(cfg_.source_freq, t0, dims_.dt, size, wavelet_.data()), "ricker");
        if (wavelet_dev_) cudaFree(wavelet_dev_);
        cuda_ok(cudaMalloc(&wavelet_dev_, wavelet_.size() * sizeof(float)), "cudaMalloc");
        cuda_ok(cudaMemcpyAsync(wavelet_dev_, wavelet_.data(), wavelet_.size() * sizeof(float),
                                cudaMemcpyHostToDevice, stream_),
                "wavelet upload");
        if (graph_ready_) {
            cudaGraphExecDestroy(graph_exec_);
            graph_ready_ = false;
        }
    }

    void swap_levels() { std::swap(a_, b_); }

    int64_t source_index() const {
        if (!cfg_.source_enabled) return -1;
        if (cfg_.source_x >= dims_.nx || cfg_.source_y >= dims_.ny || cfg_.source_z >= dims_.nz)
            throw std::invalid_argument("source cell outside the grid");
        return static_cast<int64_t>(dims_.idx(cfg_.source_x, cfg_.source_y, cfg_.source_z));
    }

    void release() {
        if (graph_ready_) cudaGraphExecDestroy(graph_exec_);
        graph_ready_ = false;
        for (float** p : {&a_, &b_, &vel2_, &wavelet_dev_})
            if (*p) {
                cudaFree(*p);
                *p = nullptr;
            }
        if (step_dev_) cudaFree(step_dev_);
        step_dev_ = nullptr;
        if (stream_) cudaStreamDestroy(stream_);
        stream_ = nullptr;
        wavelet_.clear();
        step_ = 0;
    }

    Config cfg_;
    GridDims dims_;
    cudaStream_t stream_ = nullptr;
    float* a_ = nullptr;  // current level (p or u)
    float* b_ = nullptr;  // previous level (acoustic) / scratch level (heat)
    float* vel2_ = nullptr;
    float* wavelet_dev_ = nullptr;
    int* step_dev_ = nullptr;
    std::vector<float> wavelet_;
    long long step_ = 0;
    bool graph_ready_ = false;
    int graph_chunk_ = 0;
    cudaGraphExec_t graph_exec_ = nullptr;
};

class WaveSolver final : public B200Solver {
public:
    std::string name() const override { return "wave/" + variant_name(); }
    std::vector<float> source_trace() const override { return trace_; }

protected:
    void setup_fields() override {
        const std::size_t bytes = dims_.size() * sizeof(real_t);
        cuda_ok(cudaMalloc(&vel2_, bytes), "cudaMalloc");
        HostGrid h(dims_);
        if (cfg_.model == VelocityModel::Layered)
            init_seeded_layered_velocity(h, cfg_.seed, cfg_.layers, cfg_.v_top, cfg_.v_bottom,
                                         cfg_.perturbation, cfg_.corr_cells);
        else
            init_constant_velocity(h, cfg_.velocity);
        cuda_ok(cudaMemcpyAsync(vel2_, h.ptr(), bytes, cudaMemcpyHostToDevice, stream_), "upload");
        cuda_ok(cudaStreamSynchronize(stream_), "upload");
        HostGrid p(dims_);
        if (cfg_.initial == InitialCondition::Gaussian)
            init_gaussian(p, cfg_.pulse_cx, cfg_.pulse_cy, cfg_.pulse_cz, cfg_.pulse_sigma);
        else if (cfg_.initial == InitialCondition::UniformRandom)
            init_uniform_random(p, cfg_.seed);
        // p = p_prev: a field at rest (zero initial velocity), as the reference starts.
        cuda_ok(cudaMemcpyAsync(a_, p.ptr(), bytes, cudaMemcpyHostToDevice, stream_), "upload");
        cuda_ok(cudaMemcpyAsync(b_, p.ptr(), bytes, cudaMemcpyHostToDevice, stream_), "upload");
        src_ = source_index();
        ensure_wavelet(1024);
    }

    void enqueue_step(bool device_source, int step_offset) override {
        const sb200_grid g = to_c(dims_);
        if (device_source && src_ >= 0) {
            abi_ok(sb200_wave_step_dev_f32(a_, b_, vel2_, b_, &g, src_, wavelet_dev_, step_dev_,
                                           step_offset, exact() ? 1 : 0, stream_),
                   "wave step");
            return;
        }
        float amp = 0.f;
        if (src_ >= 0) {
            ensure_wavelet(step_ + 1);
            amp = wavelet_[static_cast<std::size_t>(step_)];
        }
        if (exact())
            abi_ok(sb200_wave_step_exact_f32(a_, b_, vel2_, b_, &g, src_, amp, stream_),
                   "wave step");
        else
            abi_ok(sb200_wave_step_f32(a_, b_, vel2_, b_, &g, src_, amp, stream_), "wave step");
    }

    double bytes_per_step() const override { return compulsory_bytes_per_step(dims_); }

    int64_t src_ = -1;
    std::vector<float> trace_;
};

class HeatSolver final : public B200Solver {
public:
    std::string name() const override { return "heat/" + variant_name(); }

protected:
    void setup_fields() override {
        const std::size_t bytes = dims_.size() * sizeof(real_t);
        HostGrid u(dims_);
        if (cfg_.initial == InitialCondition::UniformRandom)
            init_uniform_random(u, cfg_.seed);
        else if (cfg_.initial == InitialCondition::Gaussian)
            init_gaussian(u, cfg_.pulse_cx, cfg_.pulse_cy, cfg_.pulse_cz, cfg_.pulse_sigma);
        cuda_ok(cudaMemcpyAsync(a_, u.ptr(), bytes, cudaMemcpyHostToDevice, stream_), "upload");
        cuda_ok(cudaMemsetAsync(b_, 0, bytes, stream_), "memset");  // halo of the other level
        if (cfg_.source_enabled)
            throw std::invalid_argument("make_solver: the heat solver takes no point source");
    }

    void enqueue_step(bool, int) override {
        const sb200_grid g = to_c(dims_);
        if (exact())
            abi_ok(sb200_heat_step_exact_f32(a_, b_, &g, cfg_.diffusivity, stream_), "heat step");
        else
            abi_ok(sb200_heat_step_f32(a_, b_, &g, cfg_.diffusivity, stream_), "heat step");
    }

    double bytes_per_step() const override { return heat_compulsory_bytes_per_step(dims_); }
};

}  // namespace

std::unique_ptr<ISolver> make_solver(const Config& cfg) {
    std::unique_ptr<ISolver> s;
    switch (cfg.physics) {
        case Physics::WavePropagation:
            s = std::make_unique<WaveSolver>();
            break;
        case Physics::HeatDiffusion:
            s = std::make_unique<HeatSolver>();
            break;
        default:
            throw std::invalid_argument("make_solver: unknown Physics value");
    }
    s->init(cfg);
    return s;
}

}  // namespace stencil
