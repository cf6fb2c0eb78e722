#pragma once
/**
 * stencil/config.hpp -- run configuration and CLI parsing, B200 build.
 *
 * Source-compatible with the reference's include/stencil/config.hpp (same
 * enums, Config fields and defaults, make_grid() and parse_args() flags and
 * errors).  Added for the benchmark configurations, all defaulting to the
 * reference's behaviour:
 *   dt_override  > 0 sets dt directly (the reference always derives
 *                dt = CFL_LIMIT * min(dx) / velocity);
 *   source_*     Ricker point source injected after every step;
 *   model        constant velocity (reference) or the seeded layered model;
 *   initial      Gaussian pulse (reference), rest, or seeded uniform [0,1).
 */
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "stencil/types.hpp"

namespace stencil {

enum class Physics {
    WavePropagation,  ///< acoustic leapfrog (default)
    HeatDiffusion,    ///< explicit forward-Euler heat equation
};

enum class KernelVariant {
    Naive,     ///< reference-order kernel (bit-identical to the reference CPU path)
    Tiled,     ///< TMA z-marching pencil kernel
    MultiGPU,  ///< single-GPU slab path (the domain-decomposed driver is not provided)
};

enum class VelocityModel {
    Constant,  ///< v = velocity everywhere (reference)
    Layered,   ///< seeded layered model, see sb200_model_layered()
};

enum class Precision {
    FP32,  ///< FP32 fields (reference)
    FP16,  ///< acoustic only: FP16 p / p_prev with a power-of-two scale, BF16 vel2 dt^2/dx^2
};

enum class InitialCondition {
    Gaussian,       ///< interior Gaussian pulse for p and p_prev (reference)
    Rest,           ///< p = p_prev = 0 (source-driven runs)
    UniformRandom,  ///< seeded U[0,1) interior (heat benchmark)
};

struct Config {
    // grid (halo-inclusive extents)
    std::size_t nx = 256;
    std::size_t ny = 256;
    std::size_t nz = 256;
    real_t dx = static_cast<real_t>(10.0);
    real_t dy = static_cast<real_t>(10.0);
    real_t dz = static_cast<real_t>(10.0);
    bool ny_explicit = false;
    bool nz_explicit = false;

    // time stepping
    int steps = 100;
    int warmup_steps = 10;
    real_t velocity = static_cast<real_t>(1500.0);
    real_t diffusivity = static_cast<real_t>(1.0e-4);

    // Gaussian pulse (InitialCondition::Gaussian)
    real_t pulse_cx = static_cast<real_t>(0.5);
    real_t pulse_cy = static_cast<real_t>(0.5);
    real_t pulse_cz = static_cast<real_t>(0.5);
    real_t pulse_sigma = static_cast<real_t>(5.0);

    // execution
    Physics physics = Physics::WavePropagation;
    KernelVariant variant = KernelVariant::Naive;
    int device = 0;
    bool verbose = false;
    std::string output_path;

    // ── B200 additions ──
    real_t dt_override = 0;  ///< > 0: use this dt instead of the CFL-derived one
    bool source_enabled = false;
    std::size_t source_x = 0, source_y = 0, source_z = 0;  ///< cell of the point source
    real_t source_freq = static_cast<real_t>(15.0);       ///< Ricker peak frequency [Hz]
    real_t source_t0 = -1;                                 ///< delay [s]; < 0 means 1/freq
    VelocityModel model = VelocityModel::Constant;
    std::uint64_t seed = 1234;
    int layers = 8;
    real_t v_top = static_cast<real_t>(1500.0);
    real_t v_bottom = static_cast<real_t>(4500.0);
    real_t perturbation = static_cast<real_t>(0.05);
    real_t corr_cells = static_cast<real_t>(20.0);
    InitialCondition initial = InitialCondition::Gaussian;
    bool use_graphs = true;  ///< run() replays captured CUDA graphs of graph_chunk steps
    int graph_chunk = 100;
    Precision precision = Precision::FP32;
    int renorm_every = 50;   ///< FP16: steps between scale renormalisations
    int monitor_every = 0;   ///< FP32: steps between stability-monitor checks (0: chunk ends)

    /// Grid descriptor: extents and spacing from the config; dt = dt_override
    /// when set, else CFL_LIMIT * min(dx, dy, dz) / velocity.
    GridDims make_grid() const {
        GridDims g;
        g.nx = nx;
        g.ny = ny;
        g.nz = nz;
        g.dx = dx;
        g.dy = dy;
        g.dz = dz;
        if (dt_override > 0) {
            g.dt = dt_override;
        } else {
            const real_t h = std::min(dx, std::min(dy, dz));
            g.dt = GridDims::CFL_LIMIT * h / velocity;
        }
        return g;
    }
};

/**
 * parse_args -- Config from argv.  Reference flags:
 *   --nx --ny --nz --dx --dy --dz --steps --warmup --velocity --diffusivity
 *   --physics wave|heat --kernel naive|tiled|multigpu --device --output --verbose
 * (--ny/--nz must equal --nx when given: the reference CLI is cubic-only).
 * Added: --dt F, --source X,Y,Z, --freq F, --model constant|layered, --seed N,
 *        --ic gaussian|rest|uniform, --precision fp32|fp16.
 * Throws std::runtime_error on unknown flags, values or missing arguments.
 */
inline Config parse_args(int argc, char** argv) {
    Config cfg;
    for (int i = 1; i < argc; ++i) {
        const std::string flag = argv[i];
        auto value = [&]() -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("missing value for flag " + flag);
            return argv[++i];
        };
        auto as_size = [&]() { return static_cast<std::size_t>(std::stoul(value())); };
        auto as_real = [&]() { return static_cast<real_t>(std::stod(value())); };
        if (flag == "--nx") {
            cfg.nx = as_size();
        } else if (flag == "--ny") {
            cfg.ny = as_size();
            cfg.ny_explicit = true;
        } else if (flag == "--nz") {
            cfg.nz = as_size();
            cfg.nz_explicit = true;
        } else if (flag == "--dx") {
            cfg.dx = as_real();
        } else if (flag == "--dy") {
            cfg.dy = as_real();
        } else if (flag == "--dz") {
            cfg.dz = as_real();
        } else if (flag == "--steps") {
            cfg.steps = static_cast<int>(as_size());
        } else if (flag == "--warmup") {
            cfg.warmup_steps = static_cast<int>(as_size());
        } else if (flag == "--velocity") {
            cfg.velocity = as_real();
        } else if (flag == "--diffusivity") {
            cfg.diffusivity = as_real();
        } else if (flag == "--device") {
            cfg.device = static_cast<int>(as_size());
        } else if (flag == "--output") {
            cfg.output_path = value();
        } else if (flag == "--verbose") {
            cfg.verbose = true;
        } else if (flag == "--physics") {
            const std::string v = value();
            if (v == "wave")
                cfg.physics = Physics::WavePropagation;
            else if (v == "heat")
                cfg.physics = Physics::HeatDiffusion;
            else
                throw std::runtime_error("unknown physics: " + v);
        } else if (flag == "--kernel") {
            const std::string v = value();
            if (v == "naive")
                cfg.variant = KernelVariant::Naive;
            else if (v == "tiled")
                cfg.variant = KernelVariant::Tiled;
            else if (v == "multigpu")
                cfg.variant = KernelVariant::MultiGPU;
            else
                throw std::runtime_error("unknown kernel: " + v);
        } else if (flag == "--dt") {
            cfg.dt_override = as_real();
        } else if (flag == "--source") {
            const std::string v = value();
            std::size_t a = 0, b = 0, c = 0;
            if (std::sscanf(v.c_str(), "%zu,%zu,%zu", &a, &b, &c) != 3)
                throw std::runtime_error("--source expects X,Y,Z");
            cfg.source_enabled = true;
            cfg.source_x = a;
            cfg.source_y = b;
            cfg.source_z = c;
        } else if (flag == "--freq") {
            cfg.source_freq = as_real();
        } else if (flag == "--model") {
            const std::string v = value();
            if (v == "constant")
                cfg.model = VelocityModel::Constant;
            else if (v == "layered")
                cfg.model = VelocityModel::Layered;
            else
                throw std::runtime_error("unknown model: " + v);
        } else if (flag == "--seed") {
            cfg.seed = static_cast<std::uint64_t>(std::stoull(value()));
        } else if (flag == "--precision") {
            const std::string v = value();
            if (v == "fp32")
                cfg.precision = Precision::FP32;
            else if (v == "fp16")
                cfg.precision = Precision::FP16;
            else
                throw std::runtime_error("unknown precision: " + v);
        } else if (flag == "--ic") {
            const std::string v = value();
            if (v == "gaussian")
                cfg.initial = InitialCondition::Gaussian;
            else if (v == "rest")
                cfg.initial = InitialCondition::Rest;
            else if (v == "uniform")
                cfg.initial = InitialCondition::UniformRandom;
            else
                throw std::runtime_error("unknown initial condition: " + v);
        } else {
            throw std::runtime_error("unknown flag: " + flag);
        }
    }
    if ((cfg.ny_explicit || cfg.nz_explicit) && (cfg.nx != cfg.ny || cfg.ny != cfg.nz))
        throw std::runtime_error("the CLI takes cubic grids only (got --nx " +
                                 std::to_string(cfg.nx) + " --ny " + std::to_string(cfg.ny) +
                                 " --nz " + std::to_string(cfg.nz) +
                                 "); set Config fields directly for other shapes");
    return cfg;
}

}  // namespace stencil
