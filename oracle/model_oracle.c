/*
 * oracle/model_oracle.c -- CPU restatement of the seeded layered velocity model.
 *
 * TEST INFRASTRUCTURE ONLY.  It lets bench.py's reference arm and the tests
 * build the benchmark's velocity model without loading the product library.
 * The product's generator is stencil_solver_b200/csrc/model.cpp
 * (sb200_model_layered); the reference has no velocity-model generator of its
 * own (its tests use a constant velocity, include/stencil/grid.hpp:83-99), so
 * this is a project-defined input and tests/test_oracle.py pins the two
 * generators bit for bit against each other.
 *
 * Definition restated here:
 *   - random source: the 64-bit Mersenne Twister MT19937-64 (Matsumoto and
 *     Nishimura, 2000; the engine C++ names std::mt19937_64, whose output
 *     sequence the C++ standard fixes), seeded with `seed`;
 *     uniform01 = (x >> 11) * 2^-53;
 *   - n_layers - 1 interface depths uniform over [4, max(5, nz - 4)), sorted;
 *     the layer of plane z is the number of interfaces <= z, and its velocity
 *     v_top + (v_bottom - v_top) * layer / (n_layers - 1);
 *   - perturbation g: white normal noise (Box-Muller pairs) on a lattice of
 *     spacing h = max(1, corr_cells / 5), smoothed per axis by a Gaussian of
 *     sigma = corr_cells / (2 h) lattice cells truncated at ceil(3 sigma) with
 *     mirrored edges, scaled so max |g| = 1 over the lattice, interpolated
 *     trilinearly to the grid;
 *   - vel2 = (float(v_z * (1 + perturbation * g)))^2, and v_max the largest v.
 * Compiled with -ffp-contract=off: every product and sum rounds where written,
 * as in the product's host build (which targets x86-64 without FMA).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MT_N 312
#define MT_M 156
#define MT_MATRIX_A 0xB5026F5AA96619E9ULL
#define MT_UPPER 0xFFFFFFFF80000000ULL
#define MT_LOWER 0x000000007FFFFFFFULL

typedef struct {
    uint64_t s[MT_N];
    int i;
} mt64_t;

static void mt64_seed(mt64_t* g, uint64_t seed) {
    g->s[0] = seed;
    for (int k = 1; k < MT_N; ++k)
        g->s[k] = 6364136223846793005ULL * (g->s[k - 1] ^ (g->s[k - 1] >> 62)) + (uint64_t)k;
    g->i = MT_N;
}

static uint64_t mt64_twist_word(uint64_t hi, uint64_t lo, uint64_t far) {
    const uint64_t x = (hi & MT_UPPER) | (lo & MT_LOWER);
    return far ^ (x >> 1) ^ ((x & 1ULL) ? MT_MATRIX_A : 0ULL);
}

static uint64_t mt64_next(mt64_t* g) {
    if (g->i >= MT_N) {
        for (int k = 0; k < MT_N; ++k)
            g->s[k] = mt64_twist_word(g->s[k], g->s[(k + 1) % MT_N], g->s[(k + MT_M) % MT_N]);
        g->i = 0;
    }
    uint64_t x = g->s[g->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= x >> 43;
    return x;
}

/* The 10000th output for seed 5489 is a known answer of the engine
 * (9981545732273789042); tests/test_oracle.py checks it. */
uint64_t oracle_mt64_nth(uint64_t seed, int64_t n) {
    mt64_t* g = (mt64_t*)malloc(sizeof(mt64_t));
    mt64_seed(g, seed);
    uint64_t x = 0;
    for (int64_t k = 0; k < n; ++k) x = mt64_next(g);
    free(g);
    return x;
}

static double uniform01(mt64_t* g) {
    return (double)(mt64_next(g) >> 11) * (1.0 / 9007199254740992.0);
}

static int cmp_double(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return (x > y) - (x < y);
}

/* White normal noise on a cx x cy x cz lattice, smoothed per axis (x, then y,
 * then z) by a normalised Gaussian of sigma_c lattice cells; returns a malloc'd
 * array the caller frees. */
static double* smoothed_noise(mt64_t* g, int64_t cx, int64_t cy, int64_t cz, double sigma_c) {
    const double pi = 3.14159265358979323846;
    const int64_t n = cx * cy * cz;
    double* a = (double*)malloc((size_t)n * sizeof(double));
    double* b = (double*)malloc((size_t)n * sizeof(double));
    for (int64_t i = 0; i < n; i += 2) {
        double u1 = uniform01(g);
        const double u2 = uniform01(g);
        if (u1 < 1e-300) u1 = 1e-300;
        const double rr = sqrt(-2.0 * log(u1));
        a[i] = rr * cos(2.0 * pi * u2);
        if (i + 1 < n) a[i + 1] = rr * sin(2.0 * pi * u2);
    }
    int hw = (int)ceil(3.0 * sigma_c);
    if (hw < 1) hw = 1;
    double* k = (double*)malloc((size_t)(2 * hw + 1) * sizeof(double));
    double ks = 0;
    for (int i = -hw; i <= hw; ++i) ks += (k[i + hw] = exp(-0.5 * i * i / (sigma_c * sigma_c)));
    for (int i = 0; i < 2 * hw + 1; ++i) k[i] /= ks;
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
                cc = cc < 0 ? -cc : (cc >= L ? 2 * L - 2 - cc : cc);
                if (cc < 0) cc = 0;
                if (cc > L - 1) cc = L - 1;
                acc += k[t + hw] * a[i + (cc - c) * s];
            }
            b[i] = acc;
        }
        double* t = a;
        a = b;
        b = t;
    }
    free(b);
    free(k);
    return a;
}

/* vel2 (nz, ny, nx) float32 and *v_max_out; returns 0, or -1 on bad arguments. */
int oracle_model_layered(float* vel2, int64_t nx, int64_t ny, int64_t nz, uint64_t seed,
                         int n_layers, float v_top, float v_bottom, float perturbation,
                         float corr_cells, float* v_max_out) {
    if (!vel2 || nx < 1 || ny < 1 || nz < 1 || n_layers < 1 || !(v_top > 0) ||
        !(v_bottom > 0) || !(perturbation >= 0) || !(perturbation < 1) || !(corr_cells > 0))
        return -1;
    mt64_t* g = (mt64_t*)malloc(sizeof(mt64_t));
    mt64_seed(g, seed);
    double* iface = (double*)malloc((size_t)(n_layers > 1 ? n_layers - 1 : 1) * sizeof(double));
    const double z0 = 4.0;
    const double z1 = (double)nz - 4.0 > 5.0 ? (double)nz - 4.0 : 5.0;
    for (int i = 0; i < n_layers - 1; ++i) iface[i] = z0 + (z1 - z0) * uniform01(g);
    qsort(iface, (size_t)(n_layers - 1), sizeof(double), cmp_double);
    float* vz = (float*)malloc((size_t)nz * sizeof(float));
    for (int64_t z = 0; z < nz; ++z) {
        int layer = 0;
        while (layer < n_layers - 1 && iface[layer] <= (double)z) ++layer;
        const double t = n_layers > 1 ? (double)layer / (n_layers - 1) : 0.0;
        vz[z] = (float)(v_top + (v_bottom - v_top) * t);
    }
    const double h = (double)corr_cells / 5.0 > 1.0 ? (double)corr_cells / 5.0 : 1.0;
    const int64_t cx = (int64_t)ceil((nx - 1) / h) + 2;
    const int64_t cy = (int64_t)ceil((ny - 1) / h) + 2;
    const int64_t cz = (int64_t)ceil((nz - 1) / h) + 2;
    double* lat = NULL;
    if (perturbation > 0) {
        lat = smoothed_noise(g, cx, cy, cz, 0.5 * corr_cells / h);
        double m = 0;
        for (int64_t i = 0; i < cx * cy * cz; ++i) m = fabs(lat[i]) > m ? fabs(lat[i]) : m;
        if (m > 0)
            for (int64_t i = 0; i < cx * cy * cz; ++i) lat[i] /= m;
    }
    float vmax = 0.f;
#pragma omp parallel for schedule(static) reduction(max : vmax)
    for (int64_t z = 0; z < nz; ++z) {
        for (int64_t y = 0; y < ny; ++y) {
            float* row = vel2 + (z * ny + y) * nx;
            for (int64_t x = 0; x < nx; ++x) {
                double gv = 0;
                if (lat) {
                    const double fx = x / h, fy = y / h, fz = z / h;
                    const int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
                    const double tx = fx - ix, ty = fy - iy, tz = fz - iz;
#define LAT(A, B, C) lat[((C) * cy + (B)) * cx + (A)]
                    const double c00 = LAT(ix, iy, iz) * (1 - tx) + LAT(ix + 1, iy, iz) * tx;
                    const double c10 = LAT(ix, iy + 1, iz) * (1 - tx) + LAT(ix + 1, iy + 1, iz) * tx;
                    const double c01 = LAT(ix, iy, iz + 1) * (1 - tx) + LAT(ix + 1, iy, iz + 1) * tx;
                    const double c11 =
                        LAT(ix, iy + 1, iz + 1) * (1 - tx) + LAT(ix + 1, iy + 1, iz + 1) * tx;
#undef LAT
                    gv = (c00 * (1 - ty) + c10 * ty) * (1 - tz) + (c01 * (1 - ty) + c11 * ty) * tz;
                }
                const float v = (float)(vz[z] * (1.0 + perturbation * gv));
                vmax = v > vmax ? v : vmax;
                row[x] = v * v;
            }
        }
    }
    if (v_max_out) *v_max_out = vmax;
    free(lat);
    free(vz);
    free(iface);
    free(g);
    return 0;
}
