#pragma once
/**
 * stencil/solver.hpp -- solver interface, B200 build.
 *
 * Source-compatible with the reference's include/stencil/solver.hpp.
 * make_solver(cfg) builds and initialises a wave or heat solver on cfg.device:
 * it allocates the fields, uploads the configured initial condition and
 * velocity model, and returns a solver whose step() enqueues one time step
 * and whose run() times n steps with CUDA events (replayed from captured CUDA
 * graphs of cfg.graph_chunk steps when cfg.use_graphs is set).
 */
#include <memory>
#include <string>
#include <vector>

#include "stencil/config.hpp"
#include "stencil/grid.hpp"
#include "stencil/timer.hpp"
#include "stencil/types.hpp"

namespace stencil {

class ISolver {
public:
    virtual ~ISolver() = default;
    virtual void init(const Config& cfg) = 0;
    virtual void step() = 0;
    virtual PerfResult run(int n_steps, int warmup = 0) = 0;
    virtual void download(HostGrid& out) const = 0;
    virtual const GridDims& dims() const = 0;
    virtual std::string name() const = 0;

    // ── B200 additions (not in the reference interface) ──
    /// Steps taken since init().
    virtual long long steps_taken() const { return 0; }
    /// p (or u) at the source cell after every step, when a source is configured.
    virtual std::vector<float> source_trace() const { return {}; }
};

std::unique_ptr<ISolver> make_solver(const Config& cfg);

}  // namespace stencil
