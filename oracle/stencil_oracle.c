/*
 * oracle/stencil_oracle.c -- CPU restatement of the reference stencil time-stepper.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: it is
 * loaded by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline /
 * reference legs, never by the product library.  It is compiled with
 * -ffp-contract=off so every multiply and add rounds exactly where the C source
 * says, which makes the FP32 variant bit-identical to the reference's own CPU
 * path built with the same flag (pinned in tests/test_oracle.py against the
 * reference sources compiled into oracle/_ref/, and against tests/golden/).
 *
 * Algorithm followed (somya2703/stencil_solver):
 *   - coefficients: include/stencil/types.hpp:175-181 (FDCoeffs<4>)
 *   - wave step:    src/kernels/stencil_naive.cu:136-170 (CPU launch_naive)
 *                   and tests/integration/test_kernel_correctness.cpp:43-75
 *                   (cpu_reference_step): per axis
 *                       lap_a  = c0*p*inv_da2
 *                       lap_a += c_r*(p[+r]+p[-r])*inv_da2      r = 1..4
 *                   then next = 2*p - prev + dt2*vel2*(lap_x+lap_y+lap_z)
 *                   over the interior [R, n-R) of each axis; halo never written.
 *   - heat step:    src/solver/heat_diffusion.cpp:73-122 -- the wave step with
 *                   prev == cur and vel2 == alpha, dt_eff^2 in place of dt^2.
 *   - norms:        src/utils/grid.cpp:86-115 (l2_error is an RMS, max_abs_error).
 * Project-defined pieces (no reference counterpart; identical rule in the CUDA
 * path): Ricker wavelet samples and the source rule
 *       next[src] += (dt2*vel2[src]) * w(t_n)    after the update of step n.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define R 4

/* include/stencil/types.hpp:175-181, evaluated in double then rounded. */
static const double C0_D = -205.0 / 72.0;
static const double C_D[R] = {8.0 / 5.0, -1.0 / 5.0, 8.0 / 315.0, -1.0 / 560.0};

void oracle_fd_coefficients(double out[R + 1]) {
    out[0] = C0_D;
    for (int r = 0; r < R; ++r) out[r + 1] = C_D[r];
}

/* One leapfrog step, generic over the element type via a macro so that the
 * FP32 and FP64 variants share one statement of the arithmetic. */
#define DEFINE_WAVE_STEP(NAME, T)                                                        \
    void NAME(const T* cur, const T* prev, const T* vel2, T* next, int64_t nx,          \
              int64_t ny, int64_t nz, T dx, T dy, T dz, T dt) {                          \
        const T c0 = (T)C0_D;                                                            \
        T c[R];                                                                          \
        for (int r = 0; r < R; ++r) c[r] = (T)C_D[r];                                    \
        const T inv_dx2 = (T)1 / (dx * dx);                                              \
        const T inv_dy2 = (T)1 / (dy * dy);                                              \
        const T inv_dz2 = (T)1 / (dz * dz);                                              \
        const T dt2 = dt * dt;                                                           \
        const int64_t sy = nx, sz = nx * ny;                                             \
        _Pragma("omp parallel for collapse(2) schedule(static)")                         \
        for (int64_t iz = R; iz < nz - R; ++iz)                                          \
            for (int64_t iy = R; iy < ny - R; ++iy)                                      \
                for (int64_t ix = R; ix < nx - R; ++ix) {                                \
                    const int64_t ci = iz * sz + iy * sy + ix;                           \
                    const T p = cur[ci];                                                 \
                    T lx = c0 * p * inv_dx2;                                             \
                    T ly = c0 * p * inv_dy2;                                             \
                    T lz = c0 * p * inv_dz2;                                             \
                    for (int r = 1; r <= R; ++r) {                                       \
                        lx += c[r - 1] * (cur[ci + r] + cur[ci - r]) * inv_dx2;          \
                        ly += c[r - 1] * (cur[ci + r * sy] + cur[ci - r * sy]) * inv_dy2; \
                        lz += c[r - 1] * (cur[ci + r * sz] + cur[ci - r * sz]) * inv_dz2; \
                    }                                                                    \
                    next[ci] = (T)2 * p - prev[ci] + dt2 * vel2[ci] * (lx + ly + lz);    \
                }                                                                        \
    }

DEFINE_WAVE_STEP(oracle_wave_step_f32, float)
DEFINE_WAVE_STEP(oracle_wave_step_f64, double)

/* Heat step with a scalar diffusivity, in the reference's arithmetic
 * (heat_diffusion.cpp:103-118): next = 2*u - u + (dt_eff^2*alpha)*lap(u).
 * 2*u - u is exact in binary floating point, so this equals
 * u + (dt_eff^2*alpha)*lap(u) with lap in the reference's per-axis order. */
#define DEFINE_HEAT_STEP(NAME, T)                                                        \
    void NAME(const T* u, T* u_next, int64_t nx, int64_t ny, int64_t nz, T dx, T dy,    \
              T dz, T dt_eff, T alpha) {                                                 \
        const T c0 = (T)C0_D;                                                            \
        T c[R];                                                                          \
        for (int r = 0; r < R; ++r) c[r] = (T)C_D[r];                                    \
        const T inv_dx2 = (T)1 / (dx * dx);                                              \
        const T inv_dy2 = (T)1 / (dy * dy);                                              \
        const T inv_dz2 = (T)1 / (dz * dz);                                              \
        const T dt2 = dt_eff * dt_eff;                                                   \
        const int64_t sy = nx, sz = nx * ny;                                             \
        _Pragma("omp parallel for collapse(2) schedule(static)")                         \
        for (int64_t iz = R; iz < nz - R; ++iz)                                          \
            for (int64_t iy = R; iy < ny - R; ++iy)                                      \
                for (int64_t ix = R; ix < nx - R; ++ix) {                                \
                    const int64_t ci = iz * sz + iy * sy + ix;                           \
                    const T p = u[ci];                                                   \
                    T lx = c0 * p * inv_dx2;                                             \
                    T ly = c0 * p * inv_dy2;                                             \
                    T lz = c0 * p * inv_dz2;                                             \
                    for (int r = 1; r <= R; ++r) {                                       \
                        lx += c[r - 1] * (u[ci + r] + u[ci - r]) * inv_dx2;              \
                        ly += c[r - 1] * (u[ci + r * sy] + u[ci - r * sy]) * inv_dy2;    \
                        lz += c[r - 1] * (u[ci + r * sz] + u[ci - r * sz]) * inv_dz2;    \
                    }                                                                    \
                    u_next[ci] = (T)2 * p - p + dt2 * alpha * (lx + ly + lz);            \
                }                                                                        \
    }

DEFINE_HEAT_STEP(oracle_heat_step_f32, float)
DEFINE_HEAT_STEP(oracle_heat_step_f64, double)

/* Project-defined source rule: after the update of step n,
 *   next[src] += (dt2 * vel2[src]) * w_n,  dt2 = dt*dt in the field's type. */
void oracle_inject_f32(float* next, const float* vel2, int64_t src, float dt, float w) {
    const float dt2 = dt * dt;
    const float k = dt2 * vel2[src];
    next[src] = next[src] + k * w;
}

void oracle_inject_f64(double* next, const double* vel2, int64_t src, double dt, double w) {
    const double dt2 = dt * dt;
    const double k = dt2 * vel2[src];
    next[src] = next[src] + k * w;
}

/* Ricker wavelet w(t) = (1 - 2 pi^2 f^2 tau^2) exp(-pi^2 f^2 tau^2), tau = t - t0,
 * sampled at t_n = n*dt for n = 0..n_steps-1 (project-defined; t0 = 1/f). */
void oracle_ricker(double f, double t0, double dt, int64_t n_steps, double* out) {
    const double pi = 3.14159265358979323846;
    for (int64_t n = 0; n < n_steps; ++n) {
        const double tau = (double)n * dt - t0;
        const double a = pi * pi * f * f * tau * tau;
        out[n] = (1.0 - 2.0 * a) * exp(-a);
    }
}

/* Runs n_steps of the acoustic scheme with a three-level ring, as the reference
 * solver does (wave_prop.cpp:67-75 + grid.hpp:144-153), with an optional source.
 * On return, cur holds the final field and prev the one before it.  trace
 * (optional) receives p at the source cell after every step. */
#define DEFINE_WAVE_RUN(NAME, STEP, INJ, T)                                             \
    void NAME(T* cur, T* prev, T* scratch, const T* vel2, int64_t nx, int64_t ny,       \
              int64_t nz, T dx, T dy, T dz, T dt, int64_t n_steps, int64_t src,          \
              const double* wavelet, T* trace) {                                         \
        T* bufs[3] = {prev, cur, scratch};                                               \
        int ip = 0, ic = 1, in = 2;                                                      \
        for (int64_t n = 0; n < n_steps; ++n) {                                          \
            STEP(bufs[ic], bufs[ip], vel2, bufs[in], nx, ny, nz, dx, dy, dz, dt);        \
            if (src >= 0 && wavelet) INJ(bufs[in], vel2, src, dt, (T)wavelet[n]);        \
            if (trace && src >= 0) trace[n] = bufs[in][src];                             \
            const int t = ip;                                                            \
            ip = ic;                                                                     \
            ic = in;                                                                     \
            in = t;                                                                      \
        }                                                                                \
        /* (cur, prev) <- (bufs[ic], bufs[ip]); the three names are a permutation  \
         * of the caller's buffers, so copy through temporaries. */                   \
        const size_t bytes = (size_t)(nx * ny * nz) * sizeof(T);                         \
        T* tc = (T*)malloc(bytes);                                                       \
        T* tp = (T*)malloc(bytes);                                                       \
        memcpy(tc, bufs[ic], bytes);                                                     \
        memcpy(tp, bufs[ip], bytes);                                                     \
        memcpy(cur, tc, bytes);                                                          \
        memcpy(prev, tp, bytes);                                                         \
        free(tc);                                                                        \
        free(tp);                                                                        \
    }

DEFINE_WAVE_RUN(oracle_wave_run_f32, oracle_wave_step_f32, oracle_inject_f32, float)
DEFINE_WAVE_RUN(oracle_wave_run_f64, oracle_wave_step_f64, oracle_inject_f64, double)

/* Norms, accumulated in double (src/utils/grid.cpp:86-115). */
double oracle_rms_diff_f32(const float* a, const float* b, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double d = (double)a[i] - (double)b[i];
        s += d * d;
    }
    return n > 0 ? sqrt(s / (double)n) : 0.0;
}

double oracle_max_abs_diff_f32(const float* a, const float* b, int64_t n) {
    double m = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double d = fabs((double)a[i] - (double)b[i]);
        if (d > m) m = d;
    }
    return m;
}

/* ── FP16-storage scheme (the B200 precision variant; no reference counterpart) ──
 * Conversions follow the IEEE 754 binary16 / bfloat16 definitions with round to
 * nearest even.  The step evaluates, in FP32 and the reference's per-axis order,
 *   out = m_out * (2 p - m_q q + K * L'(p)),  L' = sum_a (dx/d_a)^2 (c0 p + sum_r c_r (p+r + p-r)),
 * with p, q decoded from FP16 and K from BF16, then rounds out to FP16; the
 * source adds ((K[src] * dx^2) * w) * a before the rounding. */
static uint32_t f32_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static float bits_f32(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

float oracle_f16_to_f32(uint16_t h) {
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    if (e == 0) { /* zero / subnormal: m * 2^-24 */
        const float v = (float)m * 5.9604644775390625e-8f;
        return sign ? -v : v;
    }
    if (e == 31) return bits_f32(sign | 0x7f800000u | (m << 13));
    return bits_f32(sign | ((e + 112u) << 23) | (m << 13));
}

uint16_t oracle_f32_to_f16(float f) {
    const uint32_t u = f32_bits(f);
    const uint16_t sign = (uint16_t)((u >> 16) & 0x8000u);
    const uint32_t a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return sign | (a > 0x7f800000u ? 0x7e00u : 0x7c00u);
    const float af = bits_f32(a);
    if (af >= 65520.0f) return sign | 0x7c00u; /* rounds to infinity */
    if (af < 6.103515625e-05f) { /* subnormal result: quantum 2^-24, exact scaling */
        const float q = af * 16777216.0f; /* af / 2^-24 */
        const float r = nearbyintf(q);    /* round half to even (default mode) */
        return sign | (uint16_t)r;
    }
    /* normal: keep 10 mantissa bits, round to nearest even on the 13 dropped */
    uint32_t e = (a >> 23) - 112u, m = a & 0x7fffffu;
    uint32_t hm = m >> 13, rest = m & 0x1fffu;
    if (rest > 0x1000u || (rest == 0x1000u && (hm & 1u))) {
        if (++hm == 0x400u) { hm = 0; ++e; }
    }
    return sign | (uint16_t)((e << 10) | hm);
}

float oracle_bf16_to_f32(uint16_t b) { return bits_f32((uint32_t)b << 16); }

uint16_t oracle_f32_to_bf16(float f) {
    const uint32_t u = f32_bits(f);
    if ((u & 0x7f800000u) == 0x7f800000u && (u & 0x7fffffu)) return (uint16_t)((u >> 16) | 0x40u);
    return (uint16_t)((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

void oracle_wave_step_f16(const uint16_t* P, const uint16_t* Q, const uint16_t* K, uint16_t* out,
                          int64_t nx, int64_t ny, int64_t nz, float dx, float dy, float dz,
                          float m_out, float m_q, int64_t src, float w, float a) {
    const float ry = (float)((double)dx * dx / ((double)dy * dy));
    const float rz = (float)((double)dx * dx / ((double)dz * dz));
    const float c0 = (float)C0_D;
    float c[R];
    for (int r = 0; r < R; ++r) c[r] = (float)C_D[r];
    const int64_t sy = nx, sz = nx * ny;
    const float dx2 = dx * dx;
#pragma omp parallel for collapse(2) schedule(static)
    for (int64_t iz = R; iz < nz - R; ++iz)
        for (int64_t iy = R; iy < ny - R; ++iy)
            for (int64_t ix = R; ix < nx - R; ++ix) {
                const int64_t ci = iz * sz + iy * sy + ix;
                const float p = oracle_f16_to_f32(P[ci]);
                float lx = c0 * p, ly = c0 * p * ry, lz = c0 * p * rz;
                for (int r = 1; r <= R; ++r) {
                    lx += c[r - 1] * (oracle_f16_to_f32(P[ci + r]) + oracle_f16_to_f32(P[ci - r]));
                    ly += c[r - 1] * (oracle_f16_to_f32(P[ci + r * sy]) +
                                      oracle_f16_to_f32(P[ci - r * sy])) * ry;
                    lz += c[r - 1] * (oracle_f16_to_f32(P[ci + r * sz]) +
                                      oracle_f16_to_f32(P[ci - r * sz])) * rz;
                }
                const float kk = oracle_bf16_to_f32(K[ci]);
                float o = m_out * ((2.0f * p - m_q * oracle_f16_to_f32(Q[ci])) +
                                   kk * ((lx + ly) + lz));
                if (ci == src) o = o + ((kk * dx2) * w) * a;
                out[ci] = oracle_f32_to_f16(o);
            }
}

/* ── learned coarse correction (no reference counterpart) ──────────────────────
 * Restates the library's MLP path (stencil_solver_b200/csrc/mlp.cu) for the
 * gradient check: features of a 25-point star, the 26 -> 32 -> 32 -> 1 ReLU
 * network and the gradient of mean (y - t)^2.  Parameters in the library's
 * layout: W1[32][32] (out x in), b1[32], W2[32][32], b2[32], w3[32], b3.
 * With round_bf16 != 0 the operands are rounded to BF16 where the GPU's mma
 * reads them (W1, W2, x, h1 for layer 2, dh2 and dh1 for the weight-gradient
 * products, W2 for dh1); every sum is in double.  With round_bf16 == 0 all of
 * it is exact FP64 arithmetic (for finite-difference checks). */
#define MLP_H 32
#define MLP_F 32
#define MLP_OFF_B1 (MLP_H * MLP_F)
#define MLP_OFF_W2 (MLP_OFF_B1 + MLP_H)
#define MLP_OFF_B2 (MLP_OFF_W2 + MLP_H * MLP_H)
#define MLP_OFF_W3 (MLP_OFF_B2 + MLP_H)
#define MLP_OFF_B3 (MLP_OFF_W3 + MLP_H)
#define MLP_NPARAM (MLP_OFF_B3 + 1)

int oracle_mlp_nparam(void) { return MLP_NPARAM; }

static double mlp_rnd(double v, int on) {
    return on ? (double)oracle_bf16_to_f32(oracle_f32_to_bf16((float)v)) : v;
}

/* Feature row (32 BF16) and scale of the star at flat cell c, as the library
 * builds it: the difference basis / s in FP32, then BF16; feature 25 =
 * sqrtf(vel2) * dt_over_dx. */
float oracle_mlp_features(const float* p, const float* vel2, int64_t nx, int64_t ny, int64_t c,
                          float dt_over_dx, uint16_t* row) {
    float v[25];
    int k = 1;
    const int64_t sy = nx, sz = nx * ny;
    v[0] = p[c];
    for (int r = -4; r <= 4; ++r)
        if (r) v[k++] = p[c + r];
    for (int r = -4; r <= 4; ++r)
        if (r) v[k++] = p[c + r * sy];
    for (int r = -4; r <= 4; ++r)
        if (r) v[k++] = p[c + r * sz];
    float m = 0.f;
    for (int j = 0; j < 25; ++j) m = fabsf(v[j]) > m ? fabsf(v[j]) : m;
    /* s: the smallest power of two above m (0 for m = 0), from m's exponent
     * field (subnormal m counts as 2^-126; clamped below 2^126) */
    float s = 0.f;
    if (m > 0.f) {
        uint32_t e = f32_bits(m) & 0x7f800000u;
        if (e < 0x00800000u) e = 0x00800000u;
        if (e > 0x7e000000u) e = 0x7e000000u;
        s = bits_f32(e + 0x00800000u);
    }
    const float inv = s > 0.f ? 1.f / s : 0.f;
    /* difference basis: per axis a and radius r the pair (p_+r - p_-r,
     * p_+r + p_-r - 2 p_c) at features 2k, 2k + 1 (k = 4a + r - 1), then p_c, all
     * / s; v[1 + 8a + k] holds axis a's offset k - 4 (k < 4) or k - 3 (k >= 4) */
    for (int a = 0; a < 3; ++a)
        for (int r = 1; r <= 4; ++r) {
            const float up = v[1 + 8 * a + 3 + r], dn = v[1 + 8 * a + 4 - r];
            const int k = 4 * a + r - 1;
            row[2 * k] = oracle_f32_to_bf16((up - dn) * inv);
            row[2 * k + 1] = oracle_f32_to_bf16(((up + dn) - 2.f * v[0]) * inv);
        }
    row[24] = oracle_f32_to_bf16(v[0] * inv);
    row[25] = oracle_f32_to_bf16(sqrtf(vel2[c]) * dt_over_dx);
    for (int j = 26; j < 32; ++j) row[j] = 0;
    return s;
}

/* Forward of one row; h1, h2 (optional) receive the activations. */
static double mlp_row(const float* prm, const uint16_t* x, int rb, double* h1, double* h2) {
    double a1[MLP_H], a2[MLP_H];
    for (int o = 0; o < MLP_H; ++o) {
        double acc = prm[MLP_OFF_B1 + o];
        for (int i = 0; i < MLP_F; ++i)
            acc += mlp_rnd(prm[o * MLP_F + i], rb) * (double)oracle_bf16_to_f32(x[i]);
        a1[o] = acc > 0.0 ? acc : 0.0;
    }
    double y = prm[MLP_OFF_B3];
    for (int o = 0; o < MLP_H; ++o) {
        double acc = prm[MLP_OFF_B2 + o];
        for (int i = 0; i < MLP_H; ++i)
            acc += mlp_rnd(prm[MLP_OFF_W2 + o * MLP_H + i], rb) * mlp_rnd(a1[i], rb);
        a2[o] = acc > 0.0 ? acc : 0.0;
        y += (double)prm[MLP_OFF_W3 + o] * a2[o];
    }
    if (h1) memcpy(h1, a1, sizeof(a1));
    if (h2) memcpy(h2, a2, sizeof(a2));
    return y;
}

void oracle_mlp_forward(const float* prm, const uint16_t* X, int64_t n, int round_bf16,
                        double* y) {
    for (int64_t r = 0; r < n; ++r) y[r] = mlp_row(prm, X + r * MLP_F, round_bf16, NULL, NULL);
}

/* grad[0..NPARAM) = d/dparam of mean_r (y_r - t_r)^2; returns the loss. */
double oracle_mlp_grad(const float* prm, const uint16_t* X, const float* t, int64_t n,
                       int round_bf16, double* grad) {
    const int rb = round_bf16;
    double loss = 0.0;
    memset(grad, 0, sizeof(double) * MLP_NPARAM);
    for (int64_t r = 0; r < n; ++r) {
        const uint16_t* x = X + r * MLP_F;
        double h1[MLP_H], h2[MLP_H], dh2[MLP_H], dh1[MLP_H];
        const double y = mlp_row(prm, x, rb, h1, h2);
        const double e = y - (double)t[r];
        loss += e * e / (double)n;
        const double dy = 2.0 * e / (double)n;
        grad[MLP_OFF_B3] += dy;
        for (int o = 0; o < MLP_H; ++o) {
            grad[MLP_OFF_W3 + o] += dy * h2[o];
            dh2[o] = h2[o] > 0.0 ? dy * (double)prm[MLP_OFF_W3 + o] : 0.0;
            grad[MLP_OFF_B2 + o] += dh2[o];
        }
        for (int o = 0; o < MLP_H; ++o)
            for (int i = 0; i < MLP_H; ++i)
                grad[MLP_OFF_W2 + o * MLP_H + i] += mlp_rnd(dh2[o], rb) * mlp_rnd(h1[i], rb);
        for (int i = 0; i < MLP_H; ++i) {
            double acc = 0.0;
            for (int o = 0; o < MLP_H; ++o)
                acc += mlp_rnd(dh2[o], rb) * mlp_rnd(prm[MLP_OFF_W2 + o * MLP_H + i], rb);
            dh1[i] = h1[i] > 0.0 ? acc : 0.0;
            grad[MLP_OFF_B1 + i] += dh1[i];
        }
        for (int o = 0; o < MLP_H; ++o)
            for (int i = 0; i < MLP_F; ++i)
                grad[o * MLP_F + i] += mlp_rnd(dh1[o], rb) * (double)oracle_bf16_to_f32(x[i]);
    }
    return loss;
}
