#pragma once
/**
 * stencil/io.hpp -- JSON result files, B200 build.
 *
 * Source-compatible with the reference's include/stencil/io.hpp; the results
 * schema keeps every reference key and adds per-result "gpts", "dtype" and
 * "hbm_fraction".
 */
#include <string>
#include <vector>

#include "stencil/timer.hpp"

namespace stencil {

struct ScalingResult {
    std::string mode;  ///< "weak" or "strong"
    int ngpu = 1;
    double time_ms = 0.0;
    double efficiency = 0.0;
};

/// Writes benchmark results (no-op for an empty path); throws std::runtime_error
/// when the file cannot be opened.
void write_results_json(const std::string& path, const std::vector<PerfResult>& results, int device,
                        int steps, int warmup);

void write_scaling_json(const std::string& path, const std::vector<ScalingResult>& results);

}  // namespace stencil
