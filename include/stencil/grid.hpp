#pragma once
/**
 * stencil/grid.hpp -- host and device field storage, initial conditions, norms.
 *
 * Source-compatible with the reference's include/stencil/grid.hpp: HostGrid,
 * init_gaussian / init_constant_velocity / init_layered_velocity, DeviceGrid
 * (three time levels + vel2 with rotate()), validate_grid, print_grid_info,
 * l2_error (an RMS) and max_abs_error.  Device buffers are cudaMalloc'd by
 * DeviceGrid (the launchers themselves never allocate).
 */
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "stencil/types.hpp"

namespace stencil {

/// A field in host memory: flat vector in the GridDims layout.
struct HostGrid {
    std::vector<real_t> data;
    GridDims dims;

    explicit HostGrid(const GridDims& g, real_t fill = real_t{0}) : data(g.size(), fill), dims(g) {}

    real_t& at(std::size_t x, std::size_t y, std::size_t z) { return data[dims.idx(x, y, z)]; }
    const real_t& at(std::size_t x, std::size_t y, std::size_t z) const {
        return data[dims.idx(x, y, z)];
    }
    real_t* ptr() noexcept { return data.data(); }
    const real_t* ptr() const noexcept { return data.data(); }
    std::size_t bytes() const noexcept { return data.size() * sizeof(real_t); }
};

/// Gaussian pulse exp(-r^2 / (2 sigma^2)) on the interior, centred at
/// (cx*(nx-1), cy*(ny-1), cz*(nz-1)) with sigma in cells; halo cells are left
/// untouched (zero for a fresh HostGrid), as the walls are fixed at zero.
void init_gaussian(HostGrid& g, real_t cx, real_t cy, real_t cz, real_t sigma);

/// Fills a velocity-squared field with v^2 everywhere.
void init_constant_velocity(HostGrid& g, real_t v_ms);

/// Two layers: v_top^2 for z < nz/2, v_bot^2 below.
void init_layered_velocity(HostGrid& g, real_t v_top, real_t v_bot);

/// Seeded layered model (sb200_model_layered) as v^2; returns the largest velocity.
real_t init_seeded_layered_velocity(HostGrid& g, std::uint64_t seed, int layers = 8,
                                    real_t v_top = 1500, real_t v_bottom = 4500,
                                    real_t perturbation = 0.05f, real_t corr_cells = 20);

/// Seeded U[0,1) on the interior, halo zero.
void init_uniform_random(HostGrid& g, std::uint64_t seed);

/// Device storage of one solver instance: three time levels and vel2.
/// rotate() advances the ring (next -> cur -> prev) without copies.
class DeviceGrid {
public:
    explicit DeviceGrid(const GridDims& g);
    ~DeviceGrid();
    DeviceGrid(const DeviceGrid&) = delete;
    DeviceGrid& operator=(const DeviceGrid&) = delete;
    DeviceGrid(DeviceGrid&& o) noexcept;

    const GridDims& dims() const noexcept { return dims_; }
    real_t* prev() noexcept { return buf_[slot(0)]; }
    real_t* cur() noexcept { return buf_[slot(1)]; }
    real_t* next() noexcept { return buf_[slot(2)]; }
    real_t* vel2() noexcept { return vel2_; }
    const real_t* prev() const noexcept { return buf_[slot(0)]; }
    const real_t* cur() const noexcept { return buf_[slot(1)]; }

    void rotate() noexcept { head_ = (head_ + 1) % 3; }
    void clear();
    void upload_cur(const HostGrid& h, cudaStream_t s = nullptr);
    void upload_prev(const HostGrid& h, cudaStream_t s = nullptr);
    void upload_vel2(const HostGrid& h, cudaStream_t s = nullptr);
    void download_cur(HostGrid& h, cudaStream_t s = nullptr) const;

private:
    int slot(int k) const noexcept { return (head_ + k) % 3; }
    GridDims dims_;
    int head_ = 0;
    real_t* buf_[3] = {nullptr, nullptr, nullptr};
    real_t* vel2_ = nullptr;
};

/// Throws std::invalid_argument unless every extent exceeds 2R, spacings and
/// dt are positive, and (v_max > 0) v_max*dt/min(dx) <= CFL_LIMIT.
void validate_grid(const GridDims& g, real_t v_max = real_t{0});

/// Prints extents, spacing, dt and memory footprint.
void print_grid_info(const GridDims& g, const char* label = "");

/// Root-mean-square difference over all cells, accumulated in double.
double l2_error(const HostGrid& a, const HostGrid& b);

/// Largest absolute difference over all cells.
double max_abs_error(const HostGrid& a, const HostGrid& b);

}  // namespace stencil
