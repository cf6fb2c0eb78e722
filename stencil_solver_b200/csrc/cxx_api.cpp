// C++ drop-in API (include/stencil/*.hpp) over the C ABI: launchers, grid
// utilities, initial conditions and result reporting.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>

#include "stencil/grid.hpp"
#include "stencil/io.hpp"
#include "stencil/kernels.cuh"
#include "stencil/timer.hpp"
#include "stencil/types.hpp"
#include "stencil_b200.h"

namespace stencil {

namespace {

sb200_grid to_c(const GridDims& g) {
    sb200_grid c;
    c.nx = static_cast<int64_t>(g.nx);
    c.ny = static_cast<int64_t>(g.ny);
    c.nz = static_cast<int64_t>(g.nz);
    c.dx = g.dx;
    c.dy = g.dy;
    c.dz = g.dz;
    c.dt = g.dt;
    return c;
}

// The reference's error behaviour: CUDA failures print and exit (CUDA_CHECK),
// argument errors throw.
void check(int status, const char* where) {
    if (status == SB200_OK) return;
    if (status == SB200_ERR_INVALID || status == SB200_ERR_UNSUPPORTED)
        throw std::invalid_argument(std::string(where) + ": " + sb200_last_error());
    std::fprintf(stderr, "[CUDA ERROR] %s: %s\n", where, sb200_last_error());
    std::exit(EXIT_FAILURE);
}

}  // namespace

// ── launchers (kernels.cuh) ───────────────────────────────────────────────────

void upload_fd_coefficients() { check(sb200_upload_fd_coefficients(), "upload_fd_coefficients"); }

void launch_naive(const real_t* d_p_cur, const real_t* d_p_prev, const real_t* d_vel2,
                  real_t* d_p_next, const GridDims& grid, cudaStream_t stream) {
    NVTX_RANGE("launch_naive");
    const sb200_grid g = to_c(grid);
    check(sb200_launch_naive(d_p_cur, d_p_prev, d_vel2, d_p_next, &g, stream), "launch_naive");
}

void launch_tiled(const real_t* d_p_cur, const real_t* d_p_prev, const real_t* d_vel2,
                  real_t* d_p_next, const GridDims& grid, cudaStream_t stream) {
    NVTX_RANGE("launch_tiled");
    const sb200_grid g = to_c(grid);
    check(sb200_launch_tiled(d_p_cur, d_p_prev, d_vel2, d_p_next, &g, stream), "launch_tiled");
}

void launch_slab(const real_t* d_p_cur, const real_t* d_p_prev, const real_t* d_vel2,
                 real_t* d_p_next, const GridDims& dims, cudaStream_t stream) {
    NVTX_RANGE("launch_slab");
    const sb200_grid g = to_c(dims);
    check(sb200_launch_slab(d_p_cur, d_p_prev, d_vel2, d_p_next, &g, stream), "launch_slab");
}

// ── initial conditions (grid.hpp) ─────────────────────────────────────────────

void init_gaussian(HostGrid& g, real_t cx, real_t cy, real_t cz, real_t sigma) {
    const GridDims& d = g.dims;
    const std::size_t R = STENCIL_RADIUS;
    if (d.nx <= 2 * R || d.ny <= 2 * R || d.nz <= 2 * R) return;
    // Centre at c*(n-1) and 1/(2 sigma^2), evaluated in real_t like the
    // reference's initial condition so both produce the same field.
    const real_t px = cx * static_cast<real_t>(d.nx - 1);
    const real_t py = cy * static_cast<real_t>(d.ny - 1);
    const real_t pz = cz * static_cast<real_t>(d.nz - 1);
    const real_t k = real_t{1} / (real_t{2} * sigma * sigma);
    for (std::size_t z = R; z < d.nz - R; ++z) {
        const real_t rz = static_cast<real_t>(z) - pz;
        for (std::size_t y = R; y < d.ny - R; ++y) {
            const real_t ry = static_cast<real_t>(y) - py;
            for (std::size_t x = R; x < d.nx - R; ++x) {
                const real_t rx = static_cast<real_t>(x) - px;
                g.at(x, y, z) = std::exp(-(rx * rx + ry * ry + rz * rz) * k);
            }
        }
    }
}

void init_constant_velocity(HostGrid& g, real_t v_ms) {
    std::fill(g.data.begin(), g.data.end(), v_ms * v_ms);
}

void init_layered_velocity(HostGrid& g, real_t v_top, real_t v_bot) {
    const GridDims& d = g.dims;
    const std::size_t plane = d.nx * d.ny;
    for (std::size_t z = 0; z < d.nz; ++z) {
        const real_t v = z < d.nz / 2 ? v_top : v_bot;
        std::fill(g.data.begin() + z * plane, g.data.begin() + (z + 1) * plane, v * v);
    }
}

real_t init_seeded_layered_velocity(HostGrid& g, std::uint64_t seed, int layers, real_t v_top,
                                    real_t v_bottom, real_t perturbation, real_t corr_cells) {
    float vmax = 0.f;
    const GridDims& d = g.dims;
    const int rc = sb200_model_layered(g.ptr(), static_cast<int64_t>(d.nx),
                                       static_cast<int64_t>(d.ny), static_cast<int64_t>(d.nz),
                                       seed, layers, v_top, v_bottom, perturbation, corr_cells,
                                       &vmax);
    if (rc != SB200_OK) throw std::invalid_argument("init_seeded_layered_velocity: bad model");
    return vmax;
}

void init_uniform_random(HostGrid& g, std::uint64_t seed) {
    const GridDims& d = g.dims;
    const std::size_t R = STENCIL_RADIUS;
    std::mt19937_64 rng(seed);
    std::fill(g.data.begin(), g.data.end(), real_t{0});
    if (d.nx <= 2 * R || d.ny <= 2 * R || d.nz <= 2 * R) return;
    for (std::size_t z = R; z < d.nz - R; ++z)
        for (std::size_t y = R; y < d.ny - R; ++y)
            for (std::size_t x = R; x < d.nx - R; ++x)
                g.at(x, y, z) = static_cast<real_t>(static_cast<double>(rng() >> 40) *
                                                    (1.0 / 16777216.0));  // 24-bit U[0,1)
}

// ── DeviceGrid ────────────────────────────────────────────────────────────────

DeviceGrid::DeviceGrid(const GridDims& g) : dims_(g) {
    const std::size_t n = g.size() * sizeof(real_t);
    for (auto& b : buf_) CUDA_CHECK(cudaMalloc(&b, n));
    CUDA_CHECK(cudaMalloc(&vel2_, n));
    CUDA_CHECK(cudaMemset(vel2_, 0, n));
    clear();
}

DeviceGrid::~DeviceGrid() {
    for (auto& b : buf_)
        if (b) cudaFree(b);
    if (vel2_) cudaFree(vel2_);
}

DeviceGrid::DeviceGrid(DeviceGrid&& o) noexcept : dims_(o.dims_), head_(o.head_), vel2_(o.vel2_) {
    for (int i = 0; i < 3; ++i) {
        buf_[i] = o.buf_[i];
        o.buf_[i] = nullptr;
    }
    o.vel2_ = nullptr;
}

void DeviceGrid::clear() {
    const std::size_t n = dims_.size() * sizeof(real_t);
    for (auto& b : buf_) CUDA_CHECK(cudaMemset(b, 0, n));
}

void DeviceGrid::upload_cur(const HostGrid& h, cudaStream_t s) {
    CUDA_CHECK(cudaMemcpyAsync(cur(), h.ptr(), h.bytes(), cudaMemcpyHostToDevice, s));
}
void DeviceGrid::upload_prev(const HostGrid& h, cudaStream_t s) {
    CUDA_CHECK(cudaMemcpyAsync(prev(), h.ptr(), h.bytes(), cudaMemcpyHostToDevice, s));
}
void DeviceGrid::upload_vel2(const HostGrid& h, cudaStream_t s) {
    CUDA_CHECK(cudaMemcpyAsync(vel2_, h.ptr(), h.bytes(), cudaMemcpyHostToDevice, s));
}
void DeviceGrid::download_cur(HostGrid& h, cudaStream_t s) const {
    CUDA_CHECK(cudaMemcpyAsync(h.ptr(), cur(), h.bytes(), cudaMemcpyDeviceToHost, s));
}

// ── validation and norms ──────────────────────────────────────────────────────

void validate_grid(const GridDims& g, real_t v_max) {
    const std::size_t two_r = 2 * STENCIL_RADIUS;
    std::ostringstream why;
    if (g.nx <= two_r) why << "  nx must be > 2 * STENCIL_RADIUS\n";
    if (g.ny <= two_r) why << "  ny must be > 2 * STENCIL_RADIUS\n";
    if (g.nz <= two_r) why << "  nz must be > 2 * STENCIL_RADIUS\n";
    if (!(g.dx > 0)) why << "  dx must be positive\n";
    if (!(g.dy > 0)) why << "  dy must be positive\n";
    if (!(g.dz > 0)) why << "  dz must be positive\n";
    if (!(g.dt > 0)) why << "  dt must be positive\n";
    if (why.str().empty() && v_max > 0) {
        const real_t h = std::min(g.dx, std::min(g.dy, g.dz));
        const real_t courant = v_max * g.dt / h;
        if (courant > GridDims::CFL_LIMIT)
            why << "  CFL violated: v*dt/dx = " << courant << " > " << GridDims::CFL_LIMIT << "\n";
    }
    if (!why.str().empty()) throw std::invalid_argument("Invalid grid:\n" + why.str());
}

void print_grid_info(const GridDims& g, const char* label) {
    std::printf("\n-- Grid: %s --\n", label);
    std::printf("  Total cells   : %zu x %zu x %zu = %.2f M\n", g.nx, g.ny, g.nz,
                static_cast<double>(g.size()) / 1e6);
    if (g.nx > 8 && g.ny > 8 && g.nz > 8)
        std::printf("  Interior      : %zu x %zu x %zu = %.2f M\n", g.interior_nx(),
                    g.interior_ny(), g.interior_nz(), static_cast<double>(g.interior_size()) / 1e6);
    std::printf("  Spacing       : dx=%.3f dy=%.3f dz=%.3f m\n", double(g.dx), double(g.dy),
                double(g.dz));
    std::printf("  Time step     : dt=%.4e s\n", double(g.dt));
    std::printf("  Stencil radius: R=%d (%d-th order)\n", STENCIL_RADIUS, 2 * STENCIL_RADIUS);
    std::printf("  Memory/field  : %.2f MB\n", double(g.size() * sizeof(real_t)) / 1e6);
    std::printf("\n");
}

double l2_error(const HostGrid& a, const HostGrid& b) {
    if (a.data.size() != b.data.size())
        throw std::invalid_argument("l2_error: grid size mismatch");
    const std::size_t n = a.data.size();
    double s = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        const double d = double(a.data[i]) - double(b.data[i]);
        s += d * d;
    }
    return n ? std::sqrt(s / double(n)) : 0.0;
}

double max_abs_error(const HostGrid& a, const HostGrid& b) {
    if (a.data.size() != b.data.size())
        throw std::invalid_argument("max_abs_error: grid size mismatch");
    double m = 0.0;
    for (std::size_t i = 0; i < a.data.size(); ++i)
        m = std::max(m, std::fabs(double(a.data[i]) - double(b.data[i])));
    return m;
}

// ── reporting (timer.hpp, io.hpp) ─────────────────────────────────────────────

void format_perf_table(const std::vector<PerfResult>& results) {
    if (results.empty()) return;
    std::printf("\n%-26s  %8s  %10s  %10s  %12s  %10s\n", "Kernel", "Grid", "ms/step", "GB/s",
                "GFLOP/s", "Gpts/s");
    for (const auto& r : results)
        std::printf("  %-24s  %6zu^3  %8.3f ms  %8.1f     %10.1f  %10.1f\n", r.label.c_str(),
                    r.grid_size, r.time_ms, r.bandwidth_gbs, r.gflops, r.gpts);
    std::printf("\n");
}

namespace {

std::string json_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

std::string gpu_name(int device) {
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device) == cudaSuccess) return p.name;
    cudaGetLastError();
    return "unknown";
}

std::string cuda_version() {
    int v = 0;
    cudaRuntimeGetVersion(&v);
    return std::to_string(v / 1000) + "." + std::to_string((v % 1000) / 10);
}

}  // namespace

void write_results_json(const std::string& path, const std::vector<PerfResult>& results, int device,
                        int steps, int warmup) {
    if (path.empty()) return;
    std::ostringstream js;
    js << "{\n";
    js << "  \"gpu_name\": \"" << json_escape(gpu_name(device)) << "\",\n";
    js << "  \"cuda_version\": \"" << cuda_version() << "\",\n";
    js << "  \"stencil_radius\": " << STENCIL_RADIUS << ",\n";
    js << "  \"precision\": \"fp32\",\n";
    js << "  \"tile_x\": " << TILE_X << ",\n";
    js << "  \"tile_y\": " << TILE_Y << ",\n";
    js << "  \"pencil_z\": " << PENCIL_Z << ",\n";
    js << "  \"steps\": " << steps << ",\n";
    js << "  \"warmup\": " << warmup << ",\n";
    js << "  \"results\": [\n";
    for (std::size_t i = 0; i < results.size(); ++i) {
        const PerfResult& r = results[i];
        js << "    {\n";
        js << "      \"label\": \"" << json_escape(r.label) << "\",\n";
        js << "      \"grid_size\": " << r.grid_size << ",\n";
        js << "      \"time_ms\": " << r.time_ms << ",\n";
        js << "      \"bandwidth_gbs\": " << r.bandwidth_gbs << ",\n";
        js << "      \"model_bandwidth_gbs\": " << r.model_bandwidth_gbs << ",\n";
        js << "      \"gflops\": " << r.gflops << ",\n";
        js << "      \"gpts\": " << r.gpts << ",\n";
        js << "      \"dtype\": \"" << json_escape(r.dtype) << "\",\n";
        js << "      \"hbm_fraction\": " << r.hbm_fraction << "\n";
        js << "    }" << (i + 1 < results.size() ? "," : "") << "\n";
    }
    js << "  ]\n}\n";
    std::ofstream f(path);
    if (!f) throw std::runtime_error("io: cannot open output file: " + path);
    f << js.str();
}

void write_scaling_json(const std::string& path, const std::vector<ScalingResult>& results) {
    if (path.empty()) return;
    std::ostringstream js;
    js << "{\n  \"results\": [\n";
    for (std::size_t i = 0; i < results.size(); ++i) {
        const ScalingResult& r = results[i];
        js << "    {\n      \"mode\": \"" << json_escape(r.mode) << "\",\n      \"ngpu\": " << r.ngpu
           << ",\n      \"time_ms\": " << r.time_ms << ",\n      \"efficiency\": " << r.efficiency
           << "\n    }" << (i + 1 < results.size() ? "," : "") << "\n";
    }
    js << "  ]\n}\n";
    std::ofstream f(path);
    if (!f) throw std::runtime_error("io: cannot open scaling output: " + path);
    f << js.str();
}

}  // namespace stencil
