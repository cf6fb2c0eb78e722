// C ABI of the library (include/stencil_b200.h): argument checks, kernel choice,
// tensor-map setup and error reporting around the sm_100a kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "kernels.h"
#include "stencil_b200.h"

// Library-wide device error word (one per device context); kernels receive its
// address and record bounded-wait failures in it.
__device__ int g_sb200_device_error = 0;

namespace sb200 {

namespace {

thread_local std::string t_last_error;

int fail(int code, const std::string& msg) {
    t_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    return fail(SB200_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

std::mutex g_dev_mu;
int* g_err_ptr[64] = {};

int* device_error_ptr() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(g_dev_mu);
    if (!g_err_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sb200_device_error) != cudaSuccess) return nullptr;
        g_err_ptr[dev] = static_cast<int*>(p);
    }
    return g_err_ptr[dev];
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int to_desc(const sb200_grid* g, GridDesc* d) {
    if (!g) return fail(SB200_ERR_INVALID, "grid descriptor is NULL");
    if (g->nx < 0 || g->ny < 0 || g->nz < 0)
        return fail(SB200_ERR_INVALID, "negative grid extent");
    if (g->nx > (1 << 30) || g->ny > (1 << 30) || g->nz > (1 << 30))
        return fail(SB200_ERR_INVALID, "grid extent above 2^30");
    if (!(g->dx > 0.f) || !(g->dy > 0.f) || !(g->dz > 0.f) || !std::isfinite(g->dx) ||
        !std::isfinite(g->dy) || !std::isfinite(g->dz))
        return fail(SB200_ERR_INVALID, "grid spacing must be positive and finite");
    if (!std::isfinite(g->dt)) return fail(SB200_ERR_INVALID, "dt must be finite");
    d->nx = g->nx;
    d->ny = g->ny;
    d->nz = g->nz;
    d->dx = g->dx;
    d->dy = g->dy;
    d->dz = g->dz;
    d->dt = g->dt;
    return SB200_OK;
}

// ── pencil configuration: override or heuristic ──────────────────────────────

struct Override {
    int variant = -1;
    int zchunks = 1;
};
std::mutex g_cfg_mu;
Override g_override[4];

bool valid_kind(int kind) {
    return kind == SB200_KIND_WAVE_F32 || kind == SB200_KIND_HEAT_F32 ||
           kind == SB200_KIND_WAVE_F16 || kind == SB200_KIND_WAVE2_F32;
}

int variant_count(int kind) {
    if (kind == SB200_KIND_WAVE2_F32) return leap2_variant_count();
    return kind == SB200_KIND_WAVE_F16 ? pencil_f16_variant_count()
                                       : pencil_f32_variant_count(kind == SB200_KIND_HEAT_F32);
}

const char* variant_name(int kind, int v) {
    if (kind == SB200_KIND_WAVE2_F32) return leap2_variant_name(v);
    if (kind == SB200_KIND_WAVE_F16) return pencil_f16_variant_name(v);
    return pencil_f32_variant_name(kind == SB200_KIND_HEAT_F32, v);
}

int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

// Untuned default tile of a kind: the tuner's usual pick on large grids
// (1024^3 acoustic: t64x32_r2_s8_a3; 512^3 heat: t64x16_r2_s8; FP16 1024^3:
// h64x16_s8_a4), found by name so the tables can be reordered.
int default_variant(int kind) {
    const char* want = kind == SB200_KIND_WAVE_F32   ? "t64x32_r2_s8_a3"
                       : kind == SB200_KIND_HEAT_F32 ? "t64x16_r2_s8"
                       : kind == SB200_KIND_WAVE_F16 ? "h64x16_s8_a4"
                                                     : "l32x32_r1_s8";
    const int n = variant_count(kind);
    for (int v = 0; v < n; ++v) {
        const char* name = variant_name(kind, v);
        if (name && std::strcmp(name, want) == 0) return v;
    }
    return 0;
}

PencilConfig choose(int kind, const GridDesc& g) {
    {
        std::lock_guard<std::mutex> lock(g_cfg_mu);
        const Override& o = g_override[kind];
        if (o.variant >= 0) {
            PencilConfig c;
            c.variant = o.variant;
            c.zchunks = std::max(1, o.zchunks);
            return c;
        }
    }
    PencilConfig c;
    if (tuned_choice(kind, g, &c)) return c;
    // Heuristic pick, memoised per (kind, extents, device): launches stay cheap
    // on the host.
    static std::mutex memo_mu;
    static std::map<std::tuple<int, int64_t, int64_t, int64_t, int>, PencilConfig> memo;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(kind, g.nx, g.ny, g.nz, dev);
    std::lock_guard<std::mutex> lock(memo_mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
    c.variant = default_variant(kind);
    c.zchunks = zchunk_ranking(kind, c.variant, g, 1).front();
    memo[key] = c;
    return c;
}

bool pencil_ok(const GridDesc& g, std::initializer_list<const void*> ptrs) {
    if (g.nx % 4 != 0) return false;
    for (const void* p : ptrs)
        if (p && !aligned16(p)) return false;
    return true;
}

int finish_launch(cudaError_t e, const char* where) {
    if (e != cudaSuccess) return cuda_fail(e, where);
    return SB200_OK;
}

// Encodes the tensor maps a pencil variant reads: the haloed box over the
// stencil field and, where the variant stages them by TMA, the tile box over
// p_prev and vel2.
int pencil_maps(bool heat, int v, const GridDesc& g, const void* field, const void* prev,
                const void* vel2, PencilMaps* m, const char* where) {
    const PencilBoxes b = pencil_f32_boxes(heat, v);
    int rc = tensor_map_3d(&m->p, field, g.nx, g.ny, g.nz, 4, b.halo_x, b.halo_y);
    m->prev = m->p;
    m->vel2 = m->p;
    if (!rc && b.aux_tma) {
        rc = tensor_map_3d(&m->prev, prev, g.nx, g.ny, g.nz, 4, b.tile_x, b.tile_y);
        if (!rc) rc = tensor_map_3d(&m->vel2, vel2, g.nx, g.ny, g.nz, 4, b.tile_x, b.tile_y);
    }
    if (rc)
        return fail(SB200_ERR_CUDA, std::string(where) + ": tensor map encode failed (" +
                                        std::to_string(rc) + ")");
    return SB200_OK;
}

int wave_step(const float* p, const float* p_prev, const float* vel2, float* p_next,
              const sb200_grid* grid, const SourceDesc& src, void* stream, bool allow_pencil,
              const char* where) {
    const int64_t src_index = src.idx;
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!p || !p_prev || !vel2 || !p_next)
        return fail(SB200_ERR_INVALID, std::string(where) + ": NULL field pointer");
    if (p_next == p)
        return fail(SB200_ERR_INVALID, std::string(where) + ": p_next must not alias p_cur");
    if (src_index >= g.size())
        return fail(SB200_ERR_INVALID, std::string(where) + ": source index outside the grid");
    if (!g.has_interior()) return SB200_OK;  // no interior point: nothing to update
    auto st = static_cast<cudaStream_t>(stream);
    if (allow_pencil && pencil_ok(g, {p, p_prev, vel2, p_next})) {
        const PencilConfig cfg = choose(SB200_KIND_WAVE_F32, g);
        PencilMaps maps;
        if (int rc = pencil_maps(false, cfg.variant, g, p, p_prev, vel2, &maps, where)) return rc;
        return finish_launch(launch_wave_pencil_f32(maps, p_prev, vel2, p_next, g, src, cfg,
                                                    device_error_ptr(), st),
                             where);
    }
    return finish_launch(launch_wave_naive(p, p_prev, vel2, p_next, g, src, st), where);
}

// Two acoustic steps in one sweep (leap2_f32.cu).  outputs_may_alias lets the
// tuner time it with one scratch buffer for both outputs (their values unused).
int wave_step2(const float* p, const float* p_prev, const float* vel2, float* out1, float* out2,
               const sb200_grid* grid, const SourceDesc& src, float w1, void* stream,
               bool outputs_may_alias, const char* where) {
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!p || !p_prev || !vel2 || !out1 || !out2)
        return fail(SB200_ERR_INVALID, std::string(where) + ": NULL field pointer");
    if (p == p_prev || (out1 == out2 && !outputs_may_alias))
        return fail(SB200_ERR_INVALID, std::string(where) + ": the five fields must be distinct");
    for (const float* o : {static_cast<const float*>(out1), static_cast<const float*>(out2)})
        if (o == p || o == p_prev || o == vel2)
            return fail(SB200_ERR_INVALID,
                        std::string(where) + ": an output aliases an input (five distinct fields)");
    if (src.idx >= g.size())
        return fail(SB200_ERR_INVALID, std::string(where) + ": source index outside the grid");
    if (!g.has_interior()) return SB200_OK;
    if (!pencil_ok(g, {p, p_prev, vel2, out1, out2}))
        return fail(SB200_ERR_UNSUPPORTED,
                    std::string(where) + ": needs nx % 4 == 0 and 16-byte aligned fields");
    const PencilConfig cfg = choose(SB200_KIND_WAVE2_F32, g);
    const PencilBoxes b = leap2_boxes(cfg.variant);
    PencilMaps maps;
    int rc = tensor_map_3d(&maps.p, p, g.nx, g.ny, g.nz, 4, b.halo_x, b.halo_y);
    if (!rc) rc = tensor_map_3d(&maps.prev, p_prev, g.nx, g.ny, g.nz, 4, b.tile_x, b.tile_y);
    if (!rc) rc = tensor_map_3d(&maps.vel2, vel2, g.nx, g.ny, g.nz, 4, b.tile_x, b.tile_y);
    if (rc)
        return fail(SB200_ERR_CUDA, std::string(where) + ": tensor map encode failed (" +
                                        std::to_string(rc) + ")");
    return finish_launch(launch_leap2_f32(maps, out1, out2, g, src, w1, cfg, device_error_ptr(),
                                          static_cast<cudaStream_t>(stream)),
                         where);
}

SourceDesc host_source(int64_t idx, float amp) {
    SourceDesc s;
    s.idx = idx;
    s.w = amp;
    return s;
}

int wave_step_f16(const uint16_t* p, uint16_t* p_prev_next, const uint16_t* k,
                  const sb200_grid* grid, const SourceDesc& src, const sb200_f16_scale* scale,
                  int phase, void* stream) {
    const char* where = "sb200_wave_step_f16";
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!p || !p_prev_next || !k || !scale)
        return fail(SB200_ERR_INVALID, std::string(where) + ": NULL pointer");
    if (p == p_prev_next)
        return fail(SB200_ERR_INVALID, std::string(where) + ": p_next must not alias p");
    if (phase < 0 || phase > 2) return fail(SB200_ERR_INVALID, std::string(where) + ": bad phase");
    if (src.idx >= g.size())
        return fail(SB200_ERR_INVALID, std::string(where) + ": source index outside the grid");
    if (src.idx >= 0 && src.wavelet && !src.step)
        return fail(SB200_ERR_INVALID, std::string(where) + ": wavelet without step pointer");
    if (!g.has_interior()) return SB200_OK;
    if (g.nx % 8 != 0 || !aligned16(p) || !aligned16(p_prev_next) || !aligned16(k))
        return fail(SB200_ERR_UNSUPPORTED,
                    std::string(where) + ": needs nx % 8 == 0 and 16-byte aligned fields");
    const PencilConfig cfg = choose(SB200_KIND_WAVE_F16, g);
    const PencilBoxes b = pencil_f16_boxes(cfg.variant);
    PencilMaps maps;
    int rc = tensor_map_3d(&maps.p, p, g.nx, g.ny, g.nz, 2, b.halo_x, b.halo_y);
    if (!rc) rc = tensor_map_3d(&maps.prev, p_prev_next, g.nx, g.ny, g.nz, 2, b.tile_x, b.tile_y);
    if (!rc) rc = tensor_map_3d(&maps.vel2, k, g.nx, g.ny, g.nz, 2, b.tile_x, b.tile_y);
    if (rc)
        return fail(SB200_ERR_CUDA, std::string(where) + ": tensor map encode failed (" +
                                        std::to_string(rc) + ")");
    return finish_launch(
        launch_wave_pencil_f16(maps, p_prev_next, g, src, reinterpret_cast<const F16Scale*>(scale),
                               phase, cfg, device_error_ptr(), static_cast<cudaStream_t>(stream)),
        where);
}

}  // namespace

// Step dispatch with a full source descriptor (trace included), for the run
// engine; the public entry points wrap these.
int dispatch_wave_f32(const float* p, const float* p_prev, const float* vel2, float* p_next,
                      const sb200_grid* grid, const SourceDesc& src, void* stream, bool exact) {
    return wave_step(p, p_prev, vel2, p_next, grid, src, stream, !exact,
                     exact ? "sb200_wave_step_exact_f32" : "sb200_wave_step_f32");
}

int dispatch_wave2_f32(const float* p, const float* p_prev, const float* vel2, float* out1,
                       float* out2, const sb200_grid* grid, const SourceDesc& src, float w1,
                       void* stream, bool outputs_may_alias) {
    return wave_step2(p, p_prev, vel2, out1, out2, grid, src, w1, stream, outputs_may_alias,
                      "sb200_wave_step2_f32");
}

int dispatch_wave_f16(const uint16_t* p, uint16_t* p_prev_next, const uint16_t* k,
                      const sb200_grid* grid, const SourceDesc& src, const sb200_f16_scale* scale,
                      int phase, void* stream) {
    return wave_step_f16(p, p_prev_next, k, grid, src, scale, phase, stream);
}

int set_error(int code, const std::string& msg) { return fail(code, msg); }

int* device_error_word() { return device_error_ptr(); }

// A wave is SMs x resident CTAs; a split whose CTA count leaves the last wave
// mostly empty wastes that fraction of the machine, and every extra split
// re-reads 8 halo planes of p (p is 1 of 4 streams for the acoustic kernels,
// 1 of 2 for heat).
std::vector<int> zchunk_ranking(int kind, int v, const GridDesc& g, int max_n) {
    const bool f16 = kind == SB200_KIND_WAVE_F16;
    const bool heat = kind == SB200_KIND_HEAT_F32;
    const bool two = kind == SB200_KIND_WAVE2_F32;
    const int inz = static_cast<int>(g.nz - 8);
    const int resident = two ? leap2_resident(v)
                             : (f16 ? pencil_f16_resident(v) : pencil_f32_resident(heat, v));
    const double slots = double(sm_count()) * std::max(1, resident);
    std::vector<std::pair<double, int>> scored;
    for (int zc = 1; zc <= 16 && zc <= inz; ++zc) {
        const double ctas = double(two ? leap2_ctas(v, g, zc)
                                       : (f16 ? pencil_f16_ctas(v, g, zc)
                                              : pencil_f32_ctas(heat, v, g, zc)));
        const double waves = std::ceil(ctas / slots);
        const double fill = ctas / (waves * slots);
        const int zlen = (inz + zc - 1) / zc;
        // two steps: p is 4 of the pair's 20 B and a chunk reads 16 halo planes
        const double pshare = two ? 0.2 : (heat ? 0.5 : 0.25);
        const int hplanes = two ? 16 : 8;
        const double halo = double(zlen) / double(zlen + hplanes) * pshare + (1.0 - pshare);
        scored.emplace_back(-(fill * halo), zc);
    }
    std::stable_sort(scored.begin(), scored.end());
    std::vector<int> out;
    for (const auto& s : scored) {
        if (static_cast<int>(out.size()) >= max_n) break;
        out.push_back(s.second);
    }
    if (out.empty()) out.push_back(1);
    return out;
}

}  // namespace sb200

using namespace sb200;

extern "C" {

int sb200_version(void) { return 100; }

const char* sb200_last_error(void) { return t_last_error.c_str(); }

int sb200_device_error(int clear) {
    int* p = device_error_ptr();
    if (!p) return fail(SB200_ERR_CUDA, "sb200_device_error: no usable CUDA device");
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_sb200_device_error, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "sb200_device_error");
    if (clear && v) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(g_sb200_device_error, &zero, sizeof(int));
        if (e != cudaSuccess) return cuda_fail(e, "sb200_device_error");
    }
    return v;
}

int sb200_upload_fd_coefficients(void) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaSetDevice(dev);  // initialises the primary context
    if (e != cudaSuccess) return cuda_fail(e, "sb200_upload_fd_coefficients");
    return SB200_OK;
}

int sb200_launch_naive(const float* p_cur, const float* p_prev, const float* vel2,
                       float* p_next, const sb200_grid* grid, void* stream) {
    return wave_step(p_cur, p_prev, vel2, p_next, grid, host_source(-1, 0.f), stream, false,
                     "sb200_launch_naive");
}

int sb200_launch_tiled(const float* p_cur, const float* p_prev, const float* vel2,
                       float* p_next, const sb200_grid* grid, void* stream) {
    return wave_step(p_cur, p_prev, vel2, p_next, grid, host_source(-1, 0.f), stream, true,
                     "sb200_launch_tiled");
}

int sb200_launch_slab(const float* p_cur, const float* p_prev, const float* vel2,
                      float* p_next, const sb200_grid* grid, void* stream) {
    return wave_step(p_cur, p_prev, vel2, p_next, grid, host_source(-1, 0.f), stream, true,
                     "sb200_launch_slab");
}

int sb200_wave_step_f32(const float* p, const float* p_prev, const float* vel2, float* p_next,
                        const sb200_grid* grid, int64_t src_index, float src_amp,
                        void* stream) {
    return wave_step(p, p_prev, vel2, p_next, grid, host_source(src_index, src_amp), stream,
                     true, "sb200_wave_step_f32");
}

int sb200_wave_step2_f32(const float* p, const float* p_prev, const float* vel2, float* p_next,
                         float* p_next2, const sb200_grid* grid, int64_t src_index,
                         float src_amp0, float src_amp1, void* stream) {
    return wave_step2(p, p_prev, vel2, p_next, p_next2, grid, host_source(src_index, src_amp0),
                      src_amp1, stream, false, "sb200_wave_step2_f32");
}

int sb200_wave_step2_dev_f32(const float* p, const float* p_prev, const float* vel2,
                             float* p_next, float* p_next2, const sb200_grid* grid,
                             int64_t src_index, const float* wavelet, const int* step,
                             int step_offset, float* trace, void* stream) {
    if (src_index >= 0 && (!wavelet || !step))
        return fail(SB200_ERR_INVALID, "sb200_wave_step2_dev_f32: NULL wavelet / step pointer");
    SourceDesc s;
    s.idx = src_index;
    s.wavelet = wavelet;
    s.step = step;
    s.step_offset = step_offset;
    s.trace = trace;
    return wave_step2(p, p_prev, vel2, p_next, p_next2, grid, s, 0.f, stream, false,
                      "sb200_wave_step2_dev_f32");
}

int sb200_wave_step_exact_f32(const float* p, const float* p_prev, const float* vel2,
                              float* p_next, const sb200_grid* grid, int64_t src_index,
                              float src_amp, void* stream) {
    return wave_step(p, p_prev, vel2, p_next, grid, host_source(src_index, src_amp), stream,
                     false, "sb200_wave_step_exact_f32");
}

int sb200_wave_step_dev_f32(const float* p, const float* p_prev, const float* vel2,
                            float* p_next, const sb200_grid* grid, int64_t src_index,
                            const float* wavelet, const int* step, int step_offset, int exact,
                            void* stream) {
    if (src_index >= 0 && (!wavelet || !step))
        return fail(SB200_ERR_INVALID, "sb200_wave_step_dev_f32: NULL wavelet / step pointer");
    SourceDesc s;
    s.idx = src_index;
    s.wavelet = wavelet;
    s.step = step;
    s.step_offset = step_offset;
    return wave_step(p, p_prev, vel2, p_next, grid, s, stream, exact == 0,
                     "sb200_wave_step_dev_f32");
}

int sb200_set_device_int(int* dst, int value, void* stream) {
    if (!dst) return fail(SB200_ERR_INVALID, "sb200_set_device_int: NULL pointer");
    return finish_launch(launch_set_int(dst, value, static_cast<cudaStream_t>(stream)),
                         "sb200_set_device_int");
}

int sb200_heat_step_exact_f32(const float* u, float* u_next, const sb200_grid* grid,
                              float alpha, void* stream) {
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!u || !u_next)
        return fail(SB200_ERR_INVALID, "sb200_heat_step_exact_f32: NULL field pointer");
    if (u == u_next)
        return fail(SB200_ERR_INVALID, "sb200_heat_step_exact_f32: u_next must not alias u");
    if (!std::isfinite(alpha))
        return fail(SB200_ERR_INVALID, "sb200_heat_step_exact_f32: alpha must be finite");
    if (!g.has_interior()) return SB200_OK;
    return finish_launch(
        launch_heat_naive(u, u_next, g, alpha * g.dt, static_cast<cudaStream_t>(stream)),
        "sb200_heat_step_exact_f32");
}

int sb200_heat_step_f32(const float* u, float* u_next, const sb200_grid* grid, float alpha,
                        void* stream) {
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!u || !u_next) return fail(SB200_ERR_INVALID, "sb200_heat_step_f32: NULL field pointer");
    if (u == u_next)
        return fail(SB200_ERR_INVALID, "sb200_heat_step_f32: u_next must not alias u");
    if (!std::isfinite(alpha))
        return fail(SB200_ERR_INVALID, "sb200_heat_step_f32: alpha must be finite");
    if (!g.has_interior()) return SB200_OK;
    const float alpha_dt = alpha * g.dt;
    auto st = static_cast<cudaStream_t>(stream);
    if (pencil_ok(g, {u, u_next})) {
        const PencilConfig cfg = choose(SB200_KIND_HEAT_F32, g);
        PencilMaps maps;
        if (int rc = pencil_maps(true, cfg.variant, g, u, nullptr, nullptr, &maps,
                                 "sb200_heat_step_f32"))
            return rc;
        return finish_launch(
            launch_heat_pencil_f32(maps, u_next, g, alpha_dt, cfg, device_error_ptr(), st),
            "sb200_heat_step_f32");
    }
    return finish_launch(launch_heat_naive(u, u_next, g, alpha_dt, st), "sb200_heat_step_f32");
}

int sb200_wave_prepass_f32(const float* p, float* p_prev, const float* vel2, float* r,
                           const sb200_grid* grid, float beta, void* stream) {
    const char* where = "sb200_wave_prepass_f32";
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!p || !p_prev || !vel2 || !r)
        return fail(SB200_ERR_INVALID, std::string(where) + ": NULL field pointer");
    if (r == p || r == p_prev || p == p_prev)
        return fail(SB200_ERR_INVALID, std::string(where) + ": r, p and p_prev must be distinct");
    if (!std::isfinite(beta))
        return fail(SB200_ERR_INVALID, std::string(where) + ": beta must be finite");
    if (!g.has_interior()) return SB200_OK;
    if (!pencil_ok(g, {p, p_prev, vel2, r}))
        return fail(SB200_ERR_UNSUPPORTED,
                    std::string(where) + ": needs nx % 4 == 0 and 16-byte aligned fields");
    const PencilConfig cfg = choose(SB200_KIND_WAVE_F32, g);
    PencilMaps maps;
    if (int rc = pencil_maps(false, cfg.variant, g, p, p_prev, vel2, &maps, where)) return rc;
    return finish_launch(launch_prepass_pencil_f32(maps, p_prev, vel2, r, g, beta, cfg,
                                                   device_error_ptr(),
                                                   static_cast<cudaStream_t>(stream)),
                         where);
}

int sb200_f16_pack(const float* src, uint16_t* dst, int64_t n, float scale, void* stream) {
    if (!src || !dst || n < 0) return fail(SB200_ERR_INVALID, "sb200_f16_pack: bad arguments");
    if (!(scale > 0.f) || !std::isfinite(scale))
        return fail(SB200_ERR_INVALID, "sb200_f16_pack: scale must be positive");
    if (n == 0) return SB200_OK;
    return finish_launch(launch_f16_pack(src, dst, n, scale, static_cast<cudaStream_t>(stream)),
                         "sb200_f16_pack");
}

int sb200_f16_unpack(const uint16_t* src, float* dst, int64_t n, float scale, void* stream) {
    if (!src || !dst || n < 0)
        return fail(SB200_ERR_INVALID, "sb200_f16_unpack: bad arguments");
    if (!(scale > 0.f) || !std::isfinite(scale))
        return fail(SB200_ERR_INVALID, "sb200_f16_unpack: scale must be positive");
    if (n == 0) return SB200_OK;
    return finish_launch(launch_f16_unpack(src, dst, n, scale, static_cast<cudaStream_t>(stream)),
                         "sb200_f16_unpack");
}

int sb200_k_field_bf16(const float* vel2, uint16_t* k, const sb200_grid* grid, void* stream) {
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!vel2 || !k) return fail(SB200_ERR_INVALID, "sb200_k_field_bf16: NULL pointer");
    if (!(g.dt > 0.f)) return fail(SB200_ERR_INVALID, "sb200_k_field_bf16: dt must be positive");
    if (g.size() == 0) return SB200_OK;
    const float f = static_cast<float>(double(g.dt) * g.dt / (double(g.dx) * g.dx));
    return finish_launch(launch_k_bf16(vel2, k, g.size(), f, static_cast<cudaStream_t>(stream)),
                         "sb200_k_field_bf16");
}

int sb200_wave_step_f16(const uint16_t* p, uint16_t* p_prev_next, const uint16_t* k,
                        const sb200_grid* grid, int64_t src_index, float src_amp,
                        const float* wavelet, const int* step, int step_offset,
                        const sb200_f16_scale* scale, int phase, void* stream) {
    SourceDesc src;
    src.idx = src_index;
    src.w = src_amp;
    src.wavelet = wavelet;
    src.step = step;
    src.step_offset = step_offset;
    return wave_step_f16(p, p_prev_next, k, grid, src, scale, phase, stream);
}

int sb200_f16_renorm(const double* stats3, sb200_f16_scale* scale, const float* bound,
                     const int* step, float bound_host, float target, void* stream) {
    if (!stats3 || !scale || (bound && !step))
        return fail(SB200_ERR_INVALID, "sb200_f16_renorm: NULL pointer");
    if (!(target > 0.f) || !(bound_host >= 0.f))
        return fail(SB200_ERR_INVALID, "sb200_f16_renorm: bad target / bound");
    return finish_launch(launch_f16_renorm(stats3, reinterpret_cast<F16Scale*>(scale), bound,
                                           step, bound_host, target,
                                           static_cast<cudaStream_t>(stream)),
                         "sb200_f16_renorm");
}

int64_t sb200_field_stats_scratch_len(const sb200_grid* grid) {
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!g.has_interior()) return fail(SB200_ERR_INVALID, "grid has no interior");
    return 3 * static_cast<int64_t>(stats_blocks(g));
}

namespace {
int field_stats(const void* field, bool half, const sb200_grid* grid, float scale, double* out3,
                double* scratch, int64_t scratch_len, void* stream, const char* where) {
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!field || !out3 || !scratch)
        return fail(SB200_ERR_INVALID, std::string(where) + ": NULL pointer");
    if (!g.has_interior()) return fail(SB200_ERR_INVALID, std::string(where) + ": no interior");
    if (!(scale > 0.f) || !std::isfinite(scale))
        return fail(SB200_ERR_INVALID, std::string(where) + ": scale must be positive");
    if (scratch_len < 3 * static_cast<int64_t>(stats_blocks(g)))
        return fail(SB200_ERR_INVALID, std::string(where) + ": scratch too small (need " +
                                           std::to_string(3 * stats_blocks(g)) + " doubles)");
    return finish_launch(launch_field_stats(field, half, g, scale, out3, scratch,
                                            static_cast<cudaStream_t>(stream)),
                         where);
}
}  // namespace

int sb200_field_stats_f32(const float* field, const sb200_grid* grid, double* out3,
                          double* scratch, int64_t scratch_len, void* stream) {
    return field_stats(field, false, grid, 1.0f, out3, scratch, scratch_len, stream,
                       "sb200_field_stats_f32");
}

int sb200_field_stats_f16(const uint16_t* field, const sb200_grid* grid, float scale,
                          double* out3, double* scratch, int64_t scratch_len, void* stream) {
    return field_stats(field, true, grid, scale, out3, scratch, scratch_len, stream,
                       "sb200_field_stats_f16");
}

int sb200_pencil_variant_count(int kind) {
    if (!valid_kind(kind)) return fail(SB200_ERR_INVALID, "unknown kernel kind");
    return variant_count(kind);
}

const char* sb200_pencil_variant_name(int kind, int variant) {
    if (!valid_kind(kind)) return nullptr;
    return variant_name(kind, variant);
}

int sb200_set_pencil_override(int kind, int variant, int zchunks) {
    if (!valid_kind(kind)) return fail(SB200_ERR_INVALID, "unknown kernel kind");
    if (variant >= variant_count(kind))
        return fail(SB200_ERR_INVALID, "variant out of range");
    if (zchunks < 1) return fail(SB200_ERR_INVALID, "zchunks must be >= 1");
    std::lock_guard<std::mutex> lock(g_cfg_mu);
    g_override[kind].variant = variant;
    g_override[kind].zchunks = zchunks;
    return SB200_OK;
}

int sb200_pencil_choice(int kind, const sb200_grid* grid, int* variant, int* zchunks) {
    if (!valid_kind(kind)) return fail(SB200_ERR_INVALID, "unknown kernel kind");
    GridDesc g;
    if (int rc = to_desc(grid, &g)) return rc;
    if (!variant || !zchunks) return fail(SB200_ERR_INVALID, "NULL output pointer");
    if (!g.has_interior()) return fail(SB200_ERR_INVALID, "grid has no interior");
    const PencilConfig c = choose(kind, g);
    *variant = c.variant;
    *zchunks = c.zchunks;
    return SB200_OK;
}

}  // extern "C"
