#pragma once
/**
 * stencil/kernels.cuh -- kernel launcher API, B200 build.
 *
 * Source-compatible with the reference's include/stencil/kernels.cuh.  Each
 * launcher enqueues one time step on `stream` and returns without
 * synchronising; device pointers are owned by the caller.  Errors follow the
 * reference: a CUDA failure prints and exits (CUDA_CHECK semantics); invalid
 * arguments (null or aliased fields, bad spacing) throw std::invalid_argument.
 *
 *   launch_naive : reference operation order, no FMA contraction -- bit-identical
 *                  to the reference CPU path built with -ffp-contract=off.
 *   launch_tiled : TMA z-marching pencil kernel (the fast path).
 *   launch_slab  : launch_tiled on a slab whose z-face halos the caller filled.
 * p_next may equal p_prev (in-place leapfrog); it must not equal p_cur.
 */
#include <cuda_runtime.h>

#include "stencil/config.hpp"
#include "stencil/types.hpp"

namespace stencil {

/// The radius-4 weights are compile-time constants of every kernel; this only
/// makes sure a CUDA device context exists (kept for call-site compatibility).
void upload_fd_coefficients();

void launch_naive(const real_t* d_p_cur, const real_t* d_p_prev, const real_t* d_vel2,
                  real_t* d_p_next, const GridDims& grid, cudaStream_t stream = nullptr);

void launch_tiled(const real_t* d_p_cur, const real_t* d_p_prev, const real_t* d_vel2,
                  real_t* d_p_next, const GridDims& grid, cudaStream_t stream = nullptr);

void launch_slab(const real_t* d_p_cur, const real_t* d_p_prev, const real_t* d_vel2,
                 real_t* d_p_next, const GridDims& dims, cudaStream_t stream = nullptr);

inline void launch(KernelVariant variant, const real_t* d_p_cur, const real_t* d_p_prev,
                   const real_t* d_vel2, real_t* d_p_next, const GridDims& grid,
                   cudaStream_t stream = nullptr) {
    if (variant == KernelVariant::Naive)
        launch_naive(d_p_cur, d_p_prev, d_vel2, d_p_next, grid, stream);
    else
        launch_tiled(d_p_cur, d_p_prev, d_vel2, d_p_next, grid, stream);
}

}  // namespace stencil
