// Seeded synthetic velocity models and source wavelets (host side).
//
// The reference has no velocity-model or source generator (its solver uses a
// constant velocity and a Gaussian initial pulse, include/stencil/grid.hpp:57-99).
// The benchmark configurations need one, so it is defined here once and every
// consumer -- the CUDA path, the CPU oracle runs in the tests, the benchmark --
// uses the same arrays.  Deterministic on every host: std::mt19937_64's output
// sequence is fixed by the standard and the normal deviates come from our own
// Box-Muller transform (std::normal_distribution is implementation-defined).
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "stencil_b200.h"

namespace {

double uniform01(std::mt19937_64& g) {
    return static_cast<double>(g() >> 11) * (1.0 / 9007199254740992.0);  // 53 bits
}

// Correlated field on a coarse lattice: white noise smoothed by a separable
// Gaussian of standard deviation sigma_c (lattice cells), truncated at 3 sigma.
std::vector<double> smoothed_noise(std::mt19937_64& g, int64_t cx, int64_t cy, int64_t cz,
                                   double sigma_c) {
    const int64_t n = cx * cy * cz;
    std::vector<double> a(n);
    for (int64_t i = 0; i < n; i += 2) {  // Box-Muller pairs
        double u1 = uniform01(g);
        const double u2 = uniform01(g);
        if (u1 < 1e-300) u1 = 1e-300;
        const double rr = std::sqrt(-2.0 * std::log(u1));
        a[i] = rr * std::cos(2.0 * M_PI * u2);
        if (i + 1 < n) a[i + 1] = rr * std::sin(2.0 * M_PI * u2);
    }
    const int hw = std::max(1, static_cast<int>(std::ceil(3.0 * sigma_c)));
    std::vector<double> k(2 * hw + 1);
    double ks = 0;
    for (int i = -hw; i <= hw; ++i) ks += (k[i + hw] = std::exp(-0.5 * i * i / (sigma_c * sigma_c)));
    for (auto& v : k) v /= ks;
    std::vector<double> b(n);
    const int64_t ext[3] = {cx, cy, cz};
    const int64_t str[3] = {1, cx, cx * cy};
    for (int axis = 0; axis < 3; ++axis) {
        const int64_t L = ext[axis], s = str[axis];
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            const int64_t c = (i / s) % L;
            double acc = 0;
            for (int t = -hw; t <= hw; ++t) {
                int64_t cc = c + t;
                cc = cc < 0 ? -cc : (cc >= L ? 2 * L - 2 - cc : cc);  // mirror at the edges
                cc = std::min<int64_t>(std::max<int64_t>(cc, 0), L - 1);
                acc += k[t + hw] * a[i + (cc - c) * s];
            }
            b[i] = acc;
        }
        a.swap(b);
    }
    return a;
}

}  // namespace

extern "C" {

/* See include/stencil_b200.h. */
int sb200_model_layered(float* vel2, int64_t nx, int64_t ny, int64_t nz, uint64_t seed,
                        int n_layers, float v_top, float v_bottom, float perturbation,
                        float corr_cells, float* v_max_out) {
    if (!vel2 || nx < 1 || ny < 1 || nz < 1 || n_layers < 1 || !(v_top > 0) ||
        !(v_bottom > 0) || !(perturbation >= 0) || !(perturbation < 1) || !(corr_cells > 0))
        return SB200_ERR_INVALID;
    std::mt19937_64 g(seed);
    // Layer interfaces: n_layers-1 depths uniform over the interior z range, sorted.
    std::vector<double> iface(n_layers - 1);
    const double z0 = 4.0, z1 = std::max(5.0, static_cast<double>(nz) - 4.0);
    for (auto& d : iface) d = z0 + (z1 - z0) * uniform01(g);
    std::sort(iface.begin(), iface.end());
    std::vector<float> vz(nz);
    for (int64_t z = 0; z < nz; ++z) {
        const int layer = static_cast<int>(
            std::upper_bound(iface.begin(), iface.end(), static_cast<double>(z)) - iface.begin());
        const double t = n_layers > 1 ? static_cast<double>(layer) / (n_layers - 1) : 0.0;
        vz[z] = static_cast<float>(v_top + (v_bottom - v_top) * t);
    }
    // Perturbation: Gaussian-correlated field with correlation function
    // exp(-r^2 / L^2) (L = corr_cells), i.e. white noise smoothed by a Gaussian
    // of sigma = L/2, built on a lattice of spacing h = max(1, L/5) and
    // interpolated trilinearly; scaled so max|g| over the lattice is 1.
    const double h = std::max(1.0, static_cast<double>(corr_cells) / 5.0);
    const int64_t cx = static_cast<int64_t>(std::ceil((nx - 1) / h)) + 2;
    const int64_t cy = static_cast<int64_t>(std::ceil((ny - 1) / h)) + 2;
    const int64_t cz = static_cast<int64_t>(std::ceil((nz - 1) / h)) + 2;
    std::vector<double> lat;
    if (perturbation > 0) {
        lat = smoothed_noise(g, cx, cy, cz, 0.5 * corr_cells / h);
        double m = 0;
        for (double v : lat) m = std::max(m, std::fabs(v));
        if (m > 0)
            for (double& v : lat) v /= m;
    }
    float vmax = 0.f;
#pragma omp parallel for schedule(static) reduction(max : vmax)
    for (int64_t z = 0; z < nz; ++z) {
        for (int64_t y = 0; y < ny; ++y) {
            float* row = vel2 + (z * ny + y) * nx;
            for (int64_t x = 0; x < nx; ++x) {
                double gv = 0;
                if (!lat.empty()) {
                    const double fx = x / h, fy = y / h, fz = z / h;
                    const int64_t ix = static_cast<int64_t>(fx), iy = static_cast<int64_t>(fy),
                                  iz = static_cast<int64_t>(fz);
                    const double tx = fx - ix, ty = fy - iy, tz = fz - iz;
                    auto L = [&](int64_t a, int64_t b, int64_t c) {
                        return lat[(c * cy + b) * cx + a];
                    };
                    const double c00 = L(ix, iy, iz) * (1 - tx) + L(ix + 1, iy, iz) * tx;
                    const double c10 = L(ix, iy + 1, iz) * (1 - tx) + L(ix + 1, iy + 1, iz) * tx;
                    const double c01 = L(ix, iy, iz + 1) * (1 - tx) + L(ix + 1, iy, iz + 1) * tx;
                    const double c11 =
                        L(ix, iy + 1, iz + 1) * (1 - tx) + L(ix + 1, iy + 1, iz + 1) * tx;
                    gv = (c00 * (1 - ty) + c10 * ty) * (1 - tz) + (c01 * (1 - ty) + c11 * ty) * tz;
                }
                const float v = static_cast<float>(vz[z] * (1.0 + perturbation * gv));
                vmax = std::max(vmax, v);
                row[x] = v * v;
            }
        }
    }
    if (v_max_out) *v_max_out = vmax;
    return SB200_OK;
}

/* See include/stencil_b200.h. */
int sb200_ricker(double freq, double t0, double dt, int64_t n_steps, float* out) {
    if (!out || n_steps < 0 || !(freq > 0) || !(dt > 0)) return SB200_ERR_INVALID;
    for (int64_t n = 0; n < n_steps; ++n) {
        const double tau = static_cast<double>(n) * dt - t0;
        const double a = M_PI * M_PI * freq * freq * tau * tau;
        out[n] = static_cast<float>((1.0 - 2.0 * a) * std::exp(-a));
    }
    return SB200_OK;
}

}  // extern "C"
