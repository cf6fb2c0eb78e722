// Wave and heat solvers behind stencil::make_solver (include/stencil/solver.hpp).
//
// Replace the reference's SolverBase / WavePropSolver / HeatDiffusionSolver
// (src/solver/solver_base.cpp:28-133, wave_prop.cpp:67-75,
// heat_diffusion.cpp:73-122).  A solver builds the configured initial field and
// velocity model on the host and hands them to a run engine (run.cu, C ABI
// sb200_run_*), which owns the device state: two time levels with an in-place
// leapfrog, the dedicated heat kernel, FP16 storage when asked for, CUDA-graph
// replay of step chunks, the source trace and the FP64 stability monitor.
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

// The reference's error behaviour: CUDA failures print and exit; bad
// arguments throw std::invalid_argument.  The stability monitor (no reference
// counterpart) throws std::runtime_error.
void abi_ok(int status, const char* where) {
    if (status == SB200_OK) return;
    if (status == SB200_ERR_INVALID || status == SB200_ERR_UNSUPPORTED)
        throw std::invalid_argument(std::string(where) + ": " + sb200_last_error());
    if (status == SB200_ERR_MONITOR)
        throw std::runtime_error(std::string(where) + ": " + sb200_last_error());
    std::fprintf(stderr, "[CUDA ERROR] %s: %s\n", where, sb200_last_error());
    std::exit(EXIT_FAILURE);
}

class B200Solver final : public ISolver {
public:
    ~B200Solver() override {
        if (run_) sb200_run_destroy(run_);
    }

    void init(const Config& cfg) override {
        if (run_) sb200_run_destroy(run_);
        run_ = nullptr;
        cfg_ = cfg;
        dims_ = cfg.make_grid();
        if (dims_.nx <= 2 * STENCIL_RADIUS || dims_.ny <= 2 * STENCIL_RADIUS ||
            dims_.nz <= 2 * STENCIL_RADIUS)
            throw std::invalid_argument("make_solver: every extent must exceed 2*STENCIL_RADIUS");
        if (cudaSetDevice(cfg.device) != cudaSuccess) {
            std::fprintf(stderr, "[CUDA ERROR] cudaSetDevice(%d) failed\n", cfg.device);
            std::exit(EXIT_FAILURE);
        }
        heat_ = cfg.physics == Physics::HeatDiffusion;
        sb200_grid g{static_cast<int64_t>(dims_.nx), static_cast<int64_t>(dims_.ny),
                     static_cast<int64_t>(dims_.nz), dims_.dx, dims_.dy, dims_.dz, dims_.dt};
        sb200_run_config rc;
        sb200_run_config_init(&rc, &g);
        rc.physics = heat_ ? SB200_PHYSICS_HEAT : SB200_PHYSICS_WAVE;
        rc.precision = cfg.precision == Precision::FP16 ? SB200_PRECISION_F16 : SB200_PRECISION_F32;
        rc.exact = cfg.variant == KernelVariant::Naive ? 1 : 0;
        rc.diffusivity = cfg.diffusivity;
        rc.graph_chunk = cfg.use_graphs ? cfg.graph_chunk : 0;
        rc.renorm_every = cfg.renorm_every;
        rc.monitor_every = cfg.monitor_every;
        if (cfg.source_enabled) {
            if (cfg.source_x >= dims_.nx || cfg.source_y >= dims_.ny || cfg.source_z >= dims_.nz)
                throw std::invalid_argument("make_solver: source cell outside the grid");
            rc.src_index =
                static_cast<int64_t>(dims_.idx(cfg.source_x, cfg.source_y, cfg.source_z));
            rc.src_freq = cfg.source_freq;
            rc.src_t0 = cfg.source_t0;
        }
        abi_ok(sb200_run_create(&rc, &run_), "make_solver");

        HostGrid p(dims_);
        if (cfg.initial == InitialCondition::Gaussian)
            init_gaussian(p, cfg.pulse_cx, cfg.pulse_cy, cfg.pulse_cz, cfg.pulse_sigma);
        else if (cfg.initial == InitialCondition::UniformRandom)
            init_uniform_random(p, cfg.seed);
        if (heat_) {
            abi_ok(sb200_run_set_fields(run_, p.ptr(), nullptr, nullptr), "make_solver");
        } else {
            HostGrid v(dims_);
            if (cfg.model == VelocityModel::Layered)
                init_seeded_layered_velocity(v, cfg.seed, cfg.layers, cfg.v_top, cfg.v_bottom,
                                             cfg.perturbation, cfg.corr_cells);
            else
                init_constant_velocity(v, cfg.velocity);
            // p_prev = p: the field starts at rest, as the reference's does.
            abi_ok(sb200_run_set_fields(run_, p.ptr(), p.ptr(), v.ptr()), "make_solver");
        }
        if (cfg.verbose) print_grid_info(dims_, name().c_str());
    }

    void step() override { abi_ok(sb200_run_steps(run_, 1), "step"); }

    PerfResult run(int n_steps, int warmup) override {
        NVTX_PUSH(name().c_str());
        abi_ok(sb200_run_steps(run_, warmup), "run");
        abi_ok(sb200_run_synchronize(run_), "run");
        auto st = static_cast<cudaStream_t>(sb200_run_stream(run_));
        GpuTimer timer;
        timer.start(st);
        abi_ok(sb200_run_steps(run_, n_steps), "run");
        timer.stop(st);
        const double ms = double(timer.elapsed_ms()) / std::max(n_steps, 1);
        abi_ok(sb200_run_synchronize(run_), "run");
        NVTX_POP();
        PerfResult r;
        r.label = name();
        r.time_ms = ms;
        const double s = ms * 1e-3;
        const double bytes = heat_ ? heat_compulsory_bytes_per_step(dims_)
                                   : (cfg_.precision == Precision::FP16
                                          ? compulsory_bytes_per_step(dims_) / 2.0
                                          : compulsory_bytes_per_step(dims_));
        r.bandwidth_gbs = bytes / s / 1e9;
        r.model_bandwidth_gbs = bandwidth_bytes_per_step(dims_) / s / 1e9;
        r.gflops = flops_per_step(dims_) / s / 1e9;
        r.gpts = double(dims_.interior_size()) / s / 1e9;
        r.grid_size = dims_.nx;
        r.dtype = cfg_.precision == Precision::FP16 ? "fp16-storage" : "fp32";
        return r;
    }

    void download(HostGrid& out) const override {
        if (out.data.size() != dims_.size())
            throw std::invalid_argument("download: HostGrid size does not match the solver grid");
        abi_ok(sb200_run_get_field(run_, out.ptr()), "download");
    }

    const GridDims& dims() const override { return dims_; }

    std::string name() const override {
        std::string v;
        switch (cfg_.variant) {
            case KernelVariant::Naive:
                v = "naive";
                break;
            case KernelVariant::Tiled:
                v = "tiled";
                break;
            default:
                v = "multigpu";
        }
        return std::string(heat_ ? "heat/" : "wave/") + v;
    }

    long long steps_taken() const override { return sb200_run_steps_done(run_); }

    std::vector<float> source_trace() const override {
        const long long n = steps_taken();
        if (!cfg_.source_enabled || n <= 0) return {};
        std::vector<float> t(static_cast<std::size_t>(n));
        abi_ok(sb200_run_get_trace(run_, t.data(), n), "source_trace");
        return t;
    }

private:
    Config cfg_;
    GridDims dims_;
    bool heat_ = false;
    void* run_ = nullptr;
};

}  // namespace

std::unique_ptr<ISolver> make_solver(const Config& cfg) {
    if (cfg.physics != Physics::WavePropagation && cfg.physics != Physics::HeatDiffusion)
        throw std::invalid_argument("make_solver: unknown Physics value");
    auto s = std::make_unique<B200Solver>();
    s->init(cfg);
    return s;
}

}  // namespace stencil
