#pragma once
/**
 * stencil/timer.hpp -- timers and per-run performance record, B200 build.
 *
 * Source-compatible with the reference's include/stencil/timer.hpp (CpuTimer,
 * GpuTimer, PerfResult, print_perf, print_speedup, format_perf_table).
 * PerfResult gains the B200 reporting fields (Gpts/s, dtype, HBM fraction).
 */
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "stencil/types.hpp"

namespace stencil {

class CpuTimer {
public:
    void start() noexcept { t0_ = clock::now(); }
    void stop() noexcept { t1_ = clock::now(); }
    double elapsed_ms() const noexcept {
        return std::chrono::duration<double, std::milli>(t1_ - t0_).count();
    }

private:
    using clock = std::chrono::steady_clock;
    clock::time_point t0_, t1_;
};

/// CUDA-event timer on a stream; elapsed_ms() waits for the stop event.
class GpuTimer {
public:
    GpuTimer() {
        CUDA_CHECK(cudaEventCreate(&start_));
        CUDA_CHECK(cudaEventCreate(&stop_));
    }
    ~GpuTimer() {
        cudaEventDestroy(start_);
        cudaEventDestroy(stop_);
    }
    GpuTimer(const GpuTimer&) = delete;
    GpuTimer& operator=(const GpuTimer&) = delete;
    void start(cudaStream_t s = nullptr) { CUDA_CHECK(cudaEventRecord(start_, s)); }
    void stop(cudaStream_t s = nullptr) { CUDA_CHECK(cudaEventRecord(stop_, s)); }
    float elapsed_ms() {
        float ms = 0.f;
        CUDA_CHECK(cudaEventSynchronize(stop_));
        CUDA_CHECK(cudaEventElapsedTime(&ms, start_, stop_));
        return ms;
    }

private:
    cudaEvent_t start_{};
    cudaEvent_t stop_{};
};

struct PerfResult {
    std::string label;
    double time_ms = 0.0;              ///< mean time per step [ms]
    double bandwidth_gbs = 0.0;        ///< compulsory bytes / time [GB/s]
    double gflops = 0.0;               ///< flop model / time [GFLOP/s]
    double model_bandwidth_gbs = 0.0;  ///< no-reuse model bytes / time [GB/s]
    std::size_t grid_size = 0;         ///< nx (grids of the reference are cubic)
    // ── B200 additions ──
    double gpts = 0.0;          ///< interior point updates per second [G/s]
    std::string dtype = "fp32";
    double hbm_fraction = 0.0;  ///< bandwidth_gbs / measured HBM peak (0 if unknown)
};

inline void print_perf(const PerfResult& r) {
    std::printf("  %-24s  %8.3f ms/step  %7.1f GB/s  %7.1f GFLOP/s  %7.1f Gpts/s\n",
                r.label.c_str(), r.time_ms, r.bandwidth_gbs, r.gflops, r.gpts);
}

inline void print_speedup(const PerfResult& base, const PerfResult& opt) {
    if (base.time_ms <= 0.0 || opt.time_ms <= 0.0) return;
    std::printf("\n  Speedup  (%s -> %s) : %.2fx\n", base.label.c_str(), opt.label.c_str(),
                base.time_ms / opt.time_ms);
    if (base.bandwidth_gbs > 0.0)
        std::printf("  Bandwidth gain          : %+.1f%%\n",
                    (opt.bandwidth_gbs / base.bandwidth_gbs - 1.0) * 100.0);
}

/// One row per result (a grid-size sweep of one kernel); no speedup column.
void format_perf_table(const std::vector<PerfResult>& results);

}  // namespace stencil
