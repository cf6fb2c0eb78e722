#pragma once
/**
 * stencil/types.hpp -- core types of the C++ stencil API, B200 build.
 *
 * Source-compatible with the reference's include/stencil/types.hpp: the same
 * names, field layout and semantics (real_t, GridDims, FDCoeffs<R>, the
 * per-step byte/flop models, CUDA_CHECK and NVTX macros), so code written
 * against the reference compiles unchanged against libstencil_b200.
 *
 * The B200 library computes in FP32 at radius 4 only; building with
 * STENCIL_FP64, STENCIL_CPU_FALLBACK or another STENCIL_RADIUS is rejected.
 */
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#ifdef __CUDACC__
#define STENCIL_HD __host__ __device__
#define STENCIL_D __device__
#define STENCIL_FI __forceinline__
#else
#define STENCIL_HD
#define STENCIL_D
#define STENCIL_FI inline
#endif

#if defined(STENCIL_FP64)
#error "libstencil_b200 computes in FP32; FP64 is used only inside its reductions"
#endif
#if defined(STENCIL_CPU_FALLBACK)
#error "libstencil_b200 has no CPU fallback; the oracle under oracle/ is the CPU checker"
#endif

using real_t = float;

#ifndef STENCIL_RADIUS
#define STENCIL_RADIUS 4
#endif
#if STENCIL_RADIUS != 4
#error "libstencil_b200 implements the radius-4 (8th-order) stencil only"
#endif

// Tile knobs of the reference's tiled kernel, kept so code that reads them
// compiles.  The B200 pencil kernel picks its tile at run time (the default is
// 32 x 32 columns marching the whole z extent: PENCIL_Z = 0).
#ifndef TILE_X
#define TILE_X 32
#endif
#ifndef TILE_Y
#define TILE_Y 32
#endif
#ifndef PENCIL_Z
#define PENCIL_Z 0
#endif

#include <cuda_runtime.h>

#define CUDA_CHECK(call)                                                                  \
    do {                                                                                  \
        const cudaError_t stencil_err_ = (call);                                          \
        if (stencil_err_ != cudaSuccess) {                                                \
            std::fprintf(stderr, "[CUDA ERROR] %s:%d  %s\n", __FILE__, __LINE__,          \
                         cudaGetErrorString(stencil_err_));                               \
            std::exit(EXIT_FAILURE);                                                      \
        }                                                                                 \
    } while (0)

#define CUDA_CHECK_LAST() CUDA_CHECK(cudaGetLastError())

#ifdef ENABLE_NVTX
#include <nvtx3/nvtx3.hpp>
#define NVTX_RANGE(name) nvtx3::scoped_range stencil_nvtx_##__LINE__{name}
#define NVTX_PUSH(name) nvtxRangePushA(name)
#define NVTX_POP() nvtxRangePop()
#else
#define NVTX_RANGE(name) \
    do {                 \
    } while (0)
#define NVTX_PUSH(name) \
    do {                \
    } while (0)
#define NVTX_POP() \
    do {           \
    } while (0)
#endif

namespace stencil {

/// Halo-inclusive 3-D grid: extents include STENCIL_RADIUS halo cells on every
/// face; the interior is [R, n-R) per axis; z is slowest (idx = z*nx*ny + y*nx + x).
struct GridDims {
    std::size_t nx = 0;
    std::size_t ny = 0;
    std::size_t nz = 0;
    real_t dx = 1;  ///< spacing [m]
    real_t dy = 1;
    real_t dz = 1;
    real_t dt = 1;  ///< time step [s]

    STENCIL_HD std::size_t size() const noexcept { return nx * ny * nz; }
    STENCIL_HD std::size_t idx(std::size_t x, std::size_t y, std::size_t z) const noexcept {
        return (z * ny + y) * nx + x;
    }
    STENCIL_HD std::size_t interior_nx() const noexcept { return nx - 2 * STENCIL_RADIUS; }
    STENCIL_HD std::size_t interior_ny() const noexcept { return ny - 2 * STENCIL_RADIUS; }
    STENCIL_HD std::size_t interior_nz() const noexcept { return nz - 2 * STENCIL_RADIUS; }
    STENCIL_HD std::size_t interior_size() const noexcept {
        return interior_nx() * interior_ny() * interior_nz();
    }

    /// Acoustic stability limit used to derive dt: dt <= CFL_LIMIT * min(dx) / v_max.
    static constexpr real_t CFL_LIMIT = static_cast<real_t>(0.45);
};

/// Centred second-derivative weights: u'' ~ c0*u[i] + sum_r c[r-1]*(u[i+r] + u[i-r]).
template <int R>
struct FDCoeffs;

template <>
struct FDCoeffs<1> {
    static constexpr real_t c0 = static_cast<real_t>(-2.0);
    static constexpr real_t c[1] = {static_cast<real_t>(1.0)};
};
template <>
struct FDCoeffs<2> {
    static constexpr real_t c0 = static_cast<real_t>(-5.0 / 2.0);
    static constexpr real_t c[2] = {static_cast<real_t>(4.0 / 3.0),
                                    static_cast<real_t>(-1.0 / 12.0)};
};
template <>
struct FDCoeffs<3> {
    static constexpr real_t c0 = static_cast<real_t>(-49.0 / 18.0);
    static constexpr real_t c[3] = {static_cast<real_t>(3.0 / 2.0),
                                    static_cast<real_t>(-3.0 / 20.0),
                                    static_cast<real_t>(1.0 / 90.0)};
};
template <>
struct FDCoeffs<4> {
    static constexpr real_t c0 = static_cast<real_t>(-205.0 / 72.0);
    static constexpr real_t c[4] = {static_cast<real_t>(8.0 / 5.0), static_cast<real_t>(-1.0 / 5.0),
                                    static_cast<real_t>(8.0 / 315.0),
                                    static_cast<real_t>(-1.0 / 560.0)};
};

/// No-reuse traffic model: (6R+4) reads/writes of real_t per interior point.
inline double bandwidth_bytes_per_step(const GridDims& g) {
    return static_cast<double>(g.interior_size()) * (6.0 * STENCIL_RADIUS + 4.0) *
           static_cast<double>(sizeof(real_t));
}

/// Compulsory DRAM traffic of the acoustic step: read p, p_prev, vel2 and write
/// p_next once per interior point (16 B in FP32).
inline double compulsory_bytes_per_step(const GridDims& g) {
    return static_cast<double>(g.interior_size()) * 4.0 * static_cast<double>(sizeof(real_t));
}

/// Compulsory DRAM traffic of the heat step with a scalar diffusivity: read u,
/// write u_next (8 B per interior point in FP32).
inline double heat_compulsory_bytes_per_step(const GridDims& g) {
    return static_cast<double>(g.interior_size()) * 2.0 * static_cast<double>(sizeof(real_t));
}

/// Flop model: 3 axes x (4R+1) + 5 for the time update, per interior point.
inline double flops_per_step(const GridDims& g) {
    return static_cast<double>(g.interior_size()) * (3.0 * (4 * STENCIL_RADIUS + 1) + 5.0);
}

}  // namespace stencil
