// oracle/ref_shim.cpp -- C entry points over the reference's own CPU path.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/build.py together with the
// reference's unmodified sources (read in place from the reference checkout,
// never copied) into oracle/_ref/libstencil_ref_*.so.  Used to pin the oracle
// restatement and as the timed CPU baseline; never linked by the product.
//
// Wrapped reference entry points:
//   stencil::upload_fd_coefficients   src/kernels/stencil_naive.cu:129-134 (CPU branch)
//   stencil::launch_naive             src/kernels/stencil_naive.cu:136-170 (CPU branch)
//   stencil::make_solver / ISolver    src/solver/solver_base.cpp:119-133
#include <omp.h>

#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "stencil/config.hpp"
#include "stencil/grid.hpp"
#include "stencil/kernels.cuh"
#include "stencil/solver.hpp"
#include "stencil/types.hpp"

using stencil::GridDims;

extern "C" {

int ref_real_size() { return static_cast<int>(sizeof(real_t)); }

void ref_upload_fd_coefficients() { stencil::upload_fd_coefficients(); }

// One call of the reference launcher on host arrays.
void ref_launch_naive(const real_t* cur, const real_t* prev, const real_t* vel2, real_t* next,
                      int64_t nx, int64_t ny, int64_t nz, double dx, double dy, double dz,
                      double dt) {
    GridDims g;
    g.nx = static_cast<std::size_t>(nx);
    g.ny = static_cast<std::size_t>(ny);
    g.nz = static_cast<std::size_t>(nz);
    g.dx = static_cast<real_t>(dx);
    g.dy = static_cast<real_t>(dy);
    g.dz = static_cast<real_t>(dz);
    g.dt = static_cast<real_t>(dt);
    stencil::launch_naive(cur, prev, vel2, next, g, nullptr);
}

// n_steps of the reference launcher with a three-level ring (the solver's
// rotation, grid.hpp:144-153) and the project-defined source rule applied after
// each step: next[src] += (dt*dt*vel2[src]) * wavelet[n].  src < 0 = no source.
// Returns the final field in cur and the previous one in prev.
void ref_wave_run(real_t* cur, real_t* prev, real_t* scratch, const real_t* vel2, int64_t nx,
                  int64_t ny, int64_t nz, double dx, double dy, double dz, double dt,
                  int64_t n_steps, int64_t src, const double* wavelet) {
    real_t* b[3] = {prev, cur, scratch};
    int ip = 0, ic = 1, in = 2;
    const real_t dtr = static_cast<real_t>(dt);
    for (int64_t n = 0; n < n_steps; ++n) {
        ref_launch_naive(b[ic], b[ip], vel2, b[in], nx, ny, nz, dx, dy, dz, dt);
        if (src >= 0 && wavelet) {
            const real_t k = (dtr * dtr) * vel2[src];
            b[in][src] = b[in][src] + k * static_cast<real_t>(wavelet[n]);
        }
        const int t = ip;
        ip = ic;
        ic = in;
        in = t;
    }
    // (cur, prev) <- (b[ic], b[ip]); the three names are a permutation of the
    // caller's buffers, so copy through temporaries.
    const std::size_t N = static_cast<std::size_t>(nx * ny * nz);
    std::vector<real_t> fc(b[ic], b[ic] + N), fp(b[ip], b[ip] + N);
    std::memcpy(cur, fc.data(), N * sizeof(real_t));
    std::memcpy(prev, fp.data(), N * sizeof(real_t));
}

// Reference solver run through make_solver (Gaussian IC, constant velocity,
// dt from Config::make_grid).  physics: 0 wave, 1 heat.  Writes the final
// current field into out (nx*ny*nz reals).  Returns 0 on success.
int ref_solver_run(int physics, int64_t n, double dx, double velocity, double diffusivity,
                   double sigma, int steps, real_t* out) {
    try {
        stencil::Config cfg;
        cfg.nx = cfg.ny = cfg.nz = static_cast<std::size_t>(n);
        cfg.dx = cfg.dy = cfg.dz = static_cast<real_t>(dx);
        cfg.velocity = static_cast<real_t>(velocity);
        cfg.diffusivity = static_cast<real_t>(diffusivity);
        cfg.pulse_sigma = static_cast<real_t>(sigma);
        cfg.physics = physics == 1 ? stencil::Physics::HeatDiffusion
                                   : stencil::Physics::WavePropagation;
        cfg.variant = stencil::KernelVariant::Naive;
        auto s = stencil::make_solver(cfg);
        for (int i = 0; i < steps; ++i) s->step();
        stencil::HostGrid h(s->dims());
        s->download(h);
        std::memcpy(out, h.ptr(), h.bytes());
        return 0;
    } catch (...) {
        return -1;
    }
}

// The reference's Config::make_grid time step (config.hpp:75-87).
double ref_make_grid_dt(double dx, double velocity) {
    stencil::Config cfg;
    cfg.dx = cfg.dy = cfg.dz = static_cast<real_t>(dx);
    cfg.velocity = static_cast<real_t>(velocity);
    return static_cast<double>(cfg.make_grid().dt);
}

// The reference's initial condition (grid.hpp:57-78) into out.
void ref_init_gaussian(real_t* out, int64_t nx, int64_t ny, int64_t nz, double cx, double cy,
                       double cz, double sigma) {
    GridDims g;
    g.nx = static_cast<std::size_t>(nx);
    g.ny = static_cast<std::size_t>(ny);
    g.nz = static_cast<std::size_t>(nz);
    stencil::HostGrid h(g);
    stencil::init_gaussian(h, static_cast<real_t>(cx), static_cast<real_t>(cy),
                           static_cast<real_t>(cz), static_cast<real_t>(sigma));
    std::memcpy(out, h.ptr(), h.bytes());
}

// Threads an OpenMP region of the reference's CPU launcher uses in this process.
int ref_omp_threads() { return omp_get_max_threads(); }

}  // extern "C"
