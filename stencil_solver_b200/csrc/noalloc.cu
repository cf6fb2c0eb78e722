// sb200_field_stats_f32_noalloc: the FP64 field statistics (sum of squares,
// largest magnitude, non-finite count over the interior) with their per-block
// partials in a file-scope device array instead of a caller-supplied buffer.
//
// The entry point allocates nothing: no cudaMalloc / cudaFree and no library
// call that allocates.  It launches the same two kernels as
// sb200_field_stats_f32 (reduce.cu) with the same block count, so for the same
// field both entry points return the same bits.
//
// Scratch: kStaticPartials doubles (3 per block of pass 1, 28,416 bytes).  A
// grid needs 3 * stats_blocks(grid) of them; stats_blocks is capped at
// kMaxStatsBlocks, so every grid fits today, and the size check below turns any
// future mismatch into SB200_ERR_INVALID instead of an overrun.
// Nothing in the scratch has to start at zero: pass 1 writes every partial that
// pass 2 reads, in the same call.
// The array is one per device, shared by every caller in the process: two calls
// that overlap on the device (different streams without ordering between them)
// race on it.  Calls on one stream, or ordered by events, are safe.
// Set-up: the device address of the array is taken with cudaGetSymbolAddress
// once per device, on the first call; make that first call before any stream
// capture starts, since symbol lookup may load the module.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "dispatch.h"
#include "kernels.h"
#include "stencil_b200.h"

namespace sb200 {
namespace {

constexpr int kStaticPartials = 3 * kMaxStatsBlocks;

static __device__ __align__(256) double g_stats_partials[kStaticPartials];

std::mutex g_noalloc_mu;
double* g_partials_ptr[64] = {};

// Device address of g_stats_partials on the current device (cached), or an
// error status with the message set.
int static_partials(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return set_error(SB200_ERR_CUDA, std::string("sb200_field_stats_f32_noalloc: ") +
                                             cudaGetErrorString(e));
    if (dev < 0 || dev >= 64)
        return set_error(SB200_ERR_UNSUPPORTED,
                         "sb200_field_stats_f32_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_partials_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_stats_partials);
        if (e != cudaSuccess || !p)
            return set_error(SB200_ERR_CUDA,
                             std::string("sb200_field_stats_f32_noalloc: cudaGetSymbolAddress: ") +
                                 cudaGetErrorString(e));
        g_partials_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_partials_ptr[dev];
    return SB200_OK;
}

}  // namespace
}  // namespace sb200

extern "C" int sb200_field_stats_f32_noalloc(const float* field, const sb200_grid* grid,
                                             double* out3, void* stream) {
    using namespace sb200;
    const char* where = "sb200_field_stats_f32_noalloc";
    if (!grid || !field || !out3) return set_error(SB200_ERR_INVALID, std::string(where) + ": NULL pointer");
    GridDesc g;
    g.nx = grid->nx;
    g.ny = grid->ny;
    g.nz = grid->nz;
    if (g.nx > (1 << 30) || g.ny > (1 << 30) || g.nz > (1 << 30))
        return set_error(SB200_ERR_INVALID, std::string(where) + ": grid extent above 2^30");
    if (!g.has_interior()) return set_error(SB200_ERR_INVALID, std::string(where) + ": no interior");
    const int64_t need = 3 * static_cast<int64_t>(stats_blocks(g));
    if (need > kStaticPartials)
        return set_error(SB200_ERR_INVALID,
                         std::string(where) + ": grid needs " + std::to_string(need) +
                             " partial sums, the static scratch holds " +
                             std::to_string(kStaticPartials));
    double* partials = nullptr;
    if (int rc = static_partials(&partials)) return rc;
    const cudaError_t e = launch_field_stats(field, false, g, 1.0f, out3, partials,
                                             static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess)
        return set_error(SB200_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
    return SB200_OK;
}
