"""Pins the oracle (CPU restatement) before anything is checked against it.

1. Known-answer tests of the reference (tests/unit/test_fd_coeffs.cpp,
   tests/unit/test_kernels.cpp, tests/integration/test_kernel_correctness.cpp).
2. Bit-exact agreement with the golden fixtures in tests/golden/, which were
   produced by the reference's own CPU path (tests/golden/make_golden.py).
3. Bit-exact agreement with the reference's CPU path compiled here
   (oracle/_ref/, -ffp-contract=off build) on random inputs, when available.
"""
from __future__ import annotations

import hashlib
import json
import math
import pathlib

import numpy as np
import pytest

import oracle
from tests.conftest import gaussian_field

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLDEN / "manifest.json").read_text())


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ── 1. known answers ──────────────────────────────────────────────────────────

def test_fd_coefficients_known_values():
    # test_fd_coeffs.cpp:55-62
    c = oracle.fd_coefficients()
    assert c[0] == pytest.approx(-205.0 / 72.0, abs=1e-12)
    assert list(c[1:]) == pytest.approx([8 / 5, -1 / 5, 8 / 315, -1 / 560], abs=1e-12)


def test_fd_coefficients_consistency():
    # test_fd_coeffs.cpp:18-39: c0 + 2*sum(c) = 0
    c = oracle.fd_coefficients()
    assert c[0] + 2 * c[1:].sum() == pytest.approx(0.0, abs=1e-12)


def _lap_error(n):
    """Max |FD lap - exact| of sin(x) on [0, 2pi) with n points, FP64 oracle."""
    h = 2 * math.pi / n
    nx = n
    x = np.arange(nx) * h
    u = np.broadcast_to(np.sin(x), (9, 9, nx)).astype(np.float64).copy()
    one = np.ones_like(u)
    # next = 2u - u + dt^2*1*lap  with dt = 1  =>  lap = next - u
    nxt = oracle.wave_step(u, u, one, h, 1e30, 1e30, 1.0)
    lap = (nxt - u)[4, 4, 4:nx - 4]
    return np.abs(lap + np.sin(x[4:nx - 4])).max()


def test_fd_convergence_order_8():
    # test_fd_coeffs.cpp:121-126 (rate > 3.8 between 32 and 64 points)
    rate = math.log2(_lap_error(32) / _lap_error(64))
    assert rate > 7.5


def test_flat_field_fixed_point():
    # test_kernel_correctness.cpp:160-184
    d = (24, 24, 24)
    p = np.ones(d, np.float32)
    out = oracle.wave_step(p, p, np.ones(d, np.float32), 10, 10, 10, 1e-3)
    np.testing.assert_allclose(out[4:-4, 4:-4, 4:-4], 1.0, atol=1e-5)


def test_linear_field_zero_laplacian():
    # test_kernel_correctness.cpp:189-213
    n = 24
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    p = (np.float32(0.1) * x + np.float32(0.2) * y + np.float32(0.3) * z).astype(np.float32)
    out = oracle.wave_step(p, p, np.ones_like(p), 10, 10, 10, 1e-3)
    i = out[4:-4, 4:-4, 4:-4]
    e = p[4:-4, 4:-4, 4:-4]
    assert np.all(np.abs(i - e) <= np.abs(e) * 1e-4 + 1e-6)


def test_halo_never_written():
    # test_kernels.cpp:202-215
    p = gaussian_field((24, 24, 24), sigma=3.0)
    out = np.full_like(p, 7.0)
    oracle.wave_step(p, p, np.ones_like(p), 10, 10, 10, 1e-3, out=out)
    halo = np.ones(out.shape, bool)
    halo[4:-4, 4:-4, 4:-4] = False
    assert np.all(out[halo] == 7.0)


def test_rms_is_root_mean_square():
    # tests/unit/test_grid.cpp:149-157 (l2_error is an RMS)
    a = np.zeros(8, np.float32)
    b = np.full(8, 2.0, np.float32)
    assert oracle.rms_diff(a, b) == pytest.approx(2.0)
    assert oracle.max_abs_diff(a, b) == pytest.approx(2.0)


def test_gaussian_helper_matches_reference_ic():
    # Input generator only (both paths always get identical arrays); it agrees
    # with init_gaussian (grid.hpp:57-78) to within float exp rounding.
    g = np.load(GOLDEN / "wave_solver32.npz")["p"]
    h = gaussian_field((32, 32, 32), sigma=4.0)
    assert np.abs(h - g).max() <= 2e-7
    assert np.array_equal(h == 0, g == 0)


# ── 2. golden fixtures from the reference's CPU path ─────────────────────────

def test_golden_wave_gauss24():
    f = np.load(GOLDEN / "wave_gauss24.npz")
    out = oracle.wave_step(f["p"], f["p"], f["vel2"], 10, 10, 10, 1e-3)
    assert np.array_equal(out, f["out"])
    assert sha(out) == MANIFEST["wave_gauss24"]["sha256_out"]


def test_golden_wave_solver32():
    f = np.load(GOLDEN / "wave_solver32.npz")
    v2 = np.full(f["p"].shape, np.float32(1500.0) * np.float32(1500.0), np.float32)
    out = oracle.wave_step(f["p"], f["p"], v2, 10, 10, 10, float(f["dt"]))
    assert np.array_equal(out, f["out"])


def test_golden_wave_source_run():
    f = np.load(GOLDEN / "wave_src_44x36x28.npz")
    shape = f["vel2"].shape
    cur, prev, _ = oracle.wave_run(np.zeros(shape, np.float32), np.zeros(shape, np.float32),
                                   f["vel2"], 10, 10, 10, 1e-3, int(f["steps"]), int(f["src"]),
                                   f["wavelet"])
    assert np.array_equal(cur, f["cur"]) and np.array_equal(prev, f["prev"])
    c64, _, _ = oracle.wave_run(np.zeros(shape), np.zeros(shape), f["vel2"].astype(np.float64),
                                10, 10, 10, 1e-3, int(f["steps"]), int(f["src"]), f["wavelet"])
    assert np.array_equal(c64, f["cur64"])


def test_golden_wave_odd_extents():
    f = np.load(GOLDEN / "wave_odd_25x31x37.npz")
    cur, prev, _ = oracle.wave_run(f["p"].copy(), f["p"].copy(), f["vel2"], 10, 10, 10, 1e-3,
                                   int(f["steps"]))
    assert np.array_equal(cur, f["cur"]) and np.array_equal(prev, f["prev"])


def test_golden_heat_solver32():
    f = np.load(GOLDEN / "heat_solver32.npz")
    dt_eff = np.float32(math.sqrt(float(f["dt"])))  # heat_diffusion.cpp:86-87
    u = f["u0"].copy()
    for _ in range(int(f["steps"])):
        u = oracle.heat_step(u, 1, 1, 1, dt_eff, np.float32(f["alpha"]), out=u.copy())
    assert np.array_equal(u, f["out"])


def test_golden_acoustic_config_trace_and_hash():
    f = np.load(GOLDEN / "acoustic128_300.npz")
    n, steps = 128, 300
    shape = (n, n, n)
    vel2 = np.full(shape, 2000.0 ** 2, np.float32)
    cur, prev, tr = oracle.wave_run(np.zeros(shape, np.float32), np.zeros(shape, np.float32),
                                    vel2, 10, 10, 10, 1e-3, steps, int(f["src"]), f["wavelet"],
                                    trace=True)
    assert np.array_equal(tr, f["trace32"])
    assert np.array_equal(cur[n // 2], f["mid32"])
    assert sha(cur) == MANIFEST["acoustic128_300"]["sha256_final32"]


def test_ricker_matches_golden():
    f = np.load(GOLDEN / "acoustic128_300.npz")
    np.testing.assert_array_equal(oracle.ricker(15.0, 1 / 15.0, 1e-3, 300), f["wavelet"])


# ── 3. the reference CPU path compiled here ───────────────────────────────────

needs_ref = pytest.mark.skipif(not oracle.ref_available("f32_strict"),
                               reason="reference CPU path not built (no reference checkout)")


@needs_ref
@pytest.mark.parametrize("shape", [(20, 24, 28), (17, 29, 13), (40, 12, 33)])
def test_oracle_matches_reference_cpu_path(shape):
    rng = np.random.default_rng(sum(shape))
    cur = rng.standard_normal(shape).astype(np.float32)
    prev = rng.standard_normal(shape).astype(np.float32)
    vel2 = rng.uniform(1e6, 2e7, shape).astype(np.float32)
    a = oracle.wave_step(cur, prev, vel2, 7.5, 10.0, 12.5, 1.3e-3)
    b = oracle.ref_wave_step(cur, prev, vel2, 7.5, 10.0, 12.5, 1.3e-3)
    assert np.array_equal(a, b)


@needs_ref
def test_oracle_f64_matches_reference_f64():
    rng = np.random.default_rng(5)
    shape = (18, 22, 26)
    cur = rng.standard_normal(shape)
    prev = rng.standard_normal(shape)
    vel2 = rng.uniform(1e6, 2e7, shape)
    a = oracle.wave_step(cur, prev, vel2, 10.0, 10.0, 10.0, 1e-3)
    b = oracle.ref_wave_step(cur, prev, vel2, 10.0, 10.0, 10.0, 1e-3, variant="f64")
    assert np.array_equal(a, b)


# ── 4. the project-defined inputs: velocity model and wavelet ─────────────────

def test_mt19937_64_known_answer():
    # The engine's published check value: the 10000th output for seed 5489.
    assert oracle.mt64_nth(5489, 10000) == 9981545732273789042


@pytest.mark.parametrize("dims,seed", [((40, 33, 29), 7), ((128, 128, 128), 1234),
                                       ((96, 200, 320), 1334), ((9, 9, 9), 0)])
def test_model_layered_matches_library(dims, seed):
    """The oracle's restatement of the seeded layered model is bit-equal to the
    library's generator (host code; no GPU), so the reference arm of the
    benchmark builds the same velocity field without loading the library."""
    import stencil_solver_b200 as sb

    nx, ny, nz = dims
    a, va = oracle.model_layered(nx, ny, nz, seed)
    b, vb = sb.model_layered(nx, ny, nz, seed)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert va == vb
    # the same model with other layer / perturbation settings
    a2, _ = oracle.model_layered(nx, ny, nz, seed, n_layers=3, perturbation=0.0)
    b2, _ = sb.model_layered(nx, ny, nz, seed, n_layers=3, perturbation=0.0)
    assert np.array_equal(a2.view(np.uint32), b2.view(np.uint32))


def test_ricker_matches_library():
    import stencil_solver_b200 as sb

    dt = float(np.float32(0.4 * 10.0 / 4680.1))
    w1 = oracle.ricker(15.0, 1.0 / 15.0, dt, 3000).astype(np.float32)
    w2 = sb.ricker(15.0, 1.0 / 15.0, dt, 3000)
    assert np.array_equal(w1.view(np.uint32), w2.view(np.uint32))
