"""GPU parity of the FP32 kernels against the oracle, through the C ABI.

Tolerances (the acoustic parity bar, FP32 vs the reference CPU path on identical
inputs): relative L2 <= 1e-6 after one step and <= 1e-5 after a full run.  The
reference-order kernels (launch_naive, wave_step_exact) are held to bit
equality with the oracle / golden fixtures.
"""
from __future__ import annotations

import pathlib

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb
from tests.conftest import gaussian_field

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
STEP_TOL = 1e-6
RUN_TOL = 1e-5


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    sb.upload_fd_coefficients()
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0
    for k in (sb.KIND_WAVE_F32, sb.KIND_HEAT_F32):
        sb.set_pencil_override(k, -1, 1)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def rel(a, b):
    return oracle.rel_l2(a, b)


def run_gpu(torch, step, p0, prev0, vel2, grid, steps, src=-1, wavelet=None):
    """steps of `step` in place (p_next over p_prev); returns (p, p_prev) on host."""
    p, q, v = dev(torch, p0), dev(torch, prev0), dev(torch, vel2)
    for n in range(steps):
        amp = float(np.float32(wavelet[n])) if wavelet is not None else 0.0
        step(p, q, v, q, grid, src, amp)
        p, q = q, p
    return host(p), host(q)


def random_case(shape, seed):
    rng = np.random.default_rng(seed)
    cur = gaussian_field(shape, 0.45, 0.55, 0.5, 3.0) + \
        0.1 * rng.standard_normal(shape).astype(np.float32)
    prev = cur + 0.01 * rng.standard_normal(shape).astype(np.float32)
    for a in (cur, prev):  # halos are walls: zero
        m = np.ones(shape, bool)
        m[4:-4, 4:-4, 4:-4] = False
        a[m] = 0
    vel2 = rng.uniform(1500.0, 4500.0, shape).astype(np.float32) ** 2
    return cur.astype(np.float32), prev.astype(np.float32), vel2.astype(np.float32)


# ── reference-order kernel: bit equality ──────────────────────────────────────

def test_naive_bitexact_golden_gauss24(torch_cuda):
    f = np.load(GOLDEN / "wave_gauss24.npz")
    g = sb.Grid(24, 24, 24, 10, 10, 10, 1e-3)
    out = dev(torch_cuda, np.zeros_like(f["p"]))
    sb.launch_naive(dev(torch_cuda, f["p"]), dev(torch_cuda, f["p"]),
                    dev(torch_cuda, f["vel2"]), out, g)
    assert np.array_equal(host(out), f["out"])


def test_naive_bitexact_golden_solver32(torch_cuda):
    f = np.load(GOLDEN / "wave_solver32.npz")
    g = sb.Grid(32, 32, 32, 10, 10, 10, float(f["dt"]))
    v2 = np.full(f["p"].shape, np.float32(1500.0) * np.float32(1500.0), np.float32)
    out = dev(torch_cuda, np.zeros_like(f["p"]))
    sb.launch_naive(dev(torch_cuda, f["p"]), dev(torch_cuda, f["p"]), dev(torch_cuda, v2), out,
                    g)
    assert np.array_equal(host(out), f["out"])


def test_exact_step_bitexact_golden_source_run(torch_cuda):
    f = np.load(GOLDEN / "wave_src_44x36x28.npz")
    nz, ny, nx = f["vel2"].shape
    g = sb.Grid(nx, ny, nz, 10, 10, 10, 1e-3)
    z = np.zeros(f["vel2"].shape, np.float32)
    p, q = run_gpu(torch_cuda, sb.wave_step_exact, z, z, f["vel2"], g, int(f["steps"]),
                   int(f["src"]), f["wavelet"])
    assert np.array_equal(p, f["cur"]) and np.array_equal(q, f["prev"])


def test_tiled_odd_extents_falls_back_bitexact(torch_cuda):
    # nx = 25: row pitch not a multiple of 16 bytes -> reference-order kernel.
    f = np.load(GOLDEN / "wave_odd_25x31x37.npz")
    g = sb.Grid(25, 31, 37, 10, 10, 10, 1e-3)

    def step(p, q, v, o, grid, src, amp):
        sb.launch_tiled(p, q, v, o, grid)

    p, q = run_gpu(torch_cuda, step, f["p"], f["p"], f["vel2"], g, int(f["steps"]))
    assert np.array_equal(p, f["cur"]) and np.array_equal(q, f["prev"])


# ── pencil kernel: tolerance against the oracle ───────────────────────────────

@pytest.mark.parametrize("zchunks", [1, 3])
@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE_F32))))
def test_tiled_variants_one_step(torch_cuda, variant, zchunks):
    sb.set_pencil_override(sb.KIND_WAVE_F32, variant, zchunks)
    shape = (45, 70, 76)  # nz, ny, nx: ragged against every tile shape
    cur, prev, vel2 = random_case(shape, 11 + variant)
    g = sb.Grid(76, 70, 45, 10, 10, 10, 1e-3)
    ref = oracle.wave_step(cur, prev, vel2, 10, 10, 10, 1e-3)
    out = dev(torch_cuda, np.zeros(shape, np.float32))
    sb.launch_tiled(dev(torch_cuda, cur), dev(torch_cuda, prev), dev(torch_cuda, vel2), out, g)
    o = host(out)
    assert rel(o, ref) <= STEP_TOL
    halo = np.ones(shape, bool)
    halo[4:-4, 4:-4, 4:-4] = False
    assert np.all(o[halo] == 0)


def test_tiled_in_place_equals_out_of_place(torch_cuda):
    shape = (40, 40, 48)
    cur, prev, vel2 = random_case(shape, 3)
    g = sb.Grid(48, 40, 40, 10, 10, 10, 1e-3)
    out = dev(torch_cuda, np.zeros(shape, np.float32))
    sb.launch_tiled(dev(torch_cuda, cur), dev(torch_cuda, prev), dev(torch_cuda, vel2), out, g)
    q = dev(torch_cuda, prev)
    sb.launch_tiled(dev(torch_cuda, cur), q, dev(torch_cuda, vel2), q, g)
    a, b = host(out), host(q)
    inner = (slice(4, -4),) * 3
    assert np.array_equal(a[inner], b[inner])


def test_tiled_source_run_vs_golden(torch_cuda):
    f = np.load(GOLDEN / "wave_src_44x36x28.npz")
    nz, ny, nx = f["vel2"].shape
    g = sb.Grid(nx, ny, nz, 10, 10, 10, 1e-3)
    z = np.zeros(f["vel2"].shape, np.float32)
    p, _ = run_gpu(torch_cuda, sb.wave_step, z, z, f["vel2"], g, int(f["steps"]),
                   int(f["src"]), f["wavelet"])
    assert rel(p, f["cur"]) <= RUN_TOL


def test_acoustic_config_full_run(torch_cuda):
    """128^3 (120^3 interior), dx 10 m, v 2000 m/s, dt 1 ms, 15 Hz Ricker at the
    centre, 300 steps: the whole final field and the centre trace against the
    reference CPU path, and the whole field against the FP64 oracle."""
    f = np.load(GOLDEN / "acoustic128_300.npz")
    n, steps = 128, 300
    g = sb.Grid(n, n, n, 10, 10, 10, 1e-3)
    shape = (n, n, n)
    src = int(f["src"])
    w = f["wavelet"]
    p = dev(torch_cuda, np.zeros(shape, np.float32))
    q = dev(torch_cuda, np.zeros(shape, np.float32))
    v = dev(torch_cuda, np.full(shape, 2000.0 ** 2, np.float32))
    trace = torch_cuda.empty(steps, dtype=torch_cuda.float32, device="cuda")
    for s in range(steps):
        sb.wave_step(p, q, v, q, g, src, float(np.float32(w[s])))
        trace[s] = q.view(-1)[src]  # device-side copy of the sample
        p, q = q, p
    tr = host(trace)
    fin = host(p)
    assert rel(fin[n // 2], f["mid32"]) <= RUN_TOL
    assert rel(tr, f["trace32"]) <= RUN_TOL
    # The whole field: the oracle's FP32 run (bit-equal to the reference CPU
    # path, pinned here by its mid plane and trace against the golden fixture)
    # and its FP64 run (bar: the order of the reference's own FP32 error).
    vel2 = np.full(shape, 2000.0 ** 2, np.float32)
    z32 = np.zeros(shape, np.float32)
    ref32, _, tr32 = oracle.wave_run(z32.copy(), z32.copy(), vel2, 10, 10, 10, 1e-3, steps, src,
                                     w, trace=True)
    assert np.array_equal(ref32[n // 2], f["mid32"]) and np.array_equal(tr32, f["trace32"])
    assert rel(fin, ref32) <= RUN_TOL
    z64 = np.zeros(shape, np.float64)
    ref64, _, _ = oracle.wave_run(z64.copy(), z64.copy(), vel2.astype(np.float64), 10.0, 10.0,
                                  10.0, 1e-3, steps, src, w)
    assert rel(ref64[n // 2], f["mid64"]) <= 1e-12
    assert rel(fin, ref64) <= 5e-5


def test_tuner_choice_is_applied_and_correct(torch_cuda):
    shape = (72, 68, 80)
    cur, prev, vel2 = random_case(shape, 21)
    g = sb.Grid(80, 68, 72, 10, 10, 10, 1e-3)
    d = [dev(torch_cuda, a) for a in (cur, prev, vel2)]
    scratch = dev(torch_cuda, np.zeros(shape, np.float32))
    v, z, ms = sb.tune(sb.KIND_WAVE_F32, g, d[0], d[1], d[2], scratch, reps=2)
    assert ms > 0 and 0 <= v < len(sb.variant_names()) and z >= 1
    assert sb.pencil_choice(sb.KIND_WAVE_F32, g) == (v, z)
    # the tuner wrote only the scratch buffer
    assert np.array_equal(host(d[1]), prev) and np.array_equal(host(d[0]), cur)
    out = dev(torch_cuda, np.zeros(shape, np.float32))
    sb.launch_tiled(d[0], d[1], d[2], out, g)
    assert rel(host(out), oracle.wave_step(cur, prev, vel2, 10, 10, 10, 1e-3)) <= STEP_TOL


# ── heat ──────────────────────────────────────────────────────────────────────

def test_heat_one_step_vs_oracle(torch_cuda):
    shape = (36, 44, 52)
    rng = np.random.default_rng(7)
    u = rng.uniform(0, 1, shape).astype(np.float32)
    m = np.ones(shape, bool)
    m[4:-4, 4:-4, 4:-4] = False
    u[m] = 0
    g = sb.Grid(52, 44, 36, 1.0, 1.0, 1.0, 0.05)
    k = np.float32(np.float32(1.0) * np.float32(0.05))
    ref = oracle.heat_step(u, 1, 1, 1, 1.0, k)
    out = dev(torch_cuda, np.zeros(shape, np.float32))
    sb.heat_step(dev(torch_cuda, u), out, g, 1.0)
    assert rel(host(out), ref) <= STEP_TOL


@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_HEAT_F32))))
def test_heat_variants_20_steps(torch_cuda, variant):
    sb.set_pencil_override(sb.KIND_HEAT_F32, variant, 2)
    shape = (30, 41, 44)
    rng = np.random.default_rng(variant)
    u = rng.uniform(0, 1, shape).astype(np.float32)
    m = np.ones(shape, bool)
    m[4:-4, 4:-4, 4:-4] = False
    u[m] = 0
    g = sb.Grid(44, 41, 30, 1.0, 1.0, 1.0, 0.05)
    a, b = dev(torch_cuda, u), dev(torch_cuda, np.zeros(shape, np.float32))
    ref = u.copy()
    for _ in range(20):
        sb.heat_step(a, b, g, 1.0)
        a, b = b, a
        ref = oracle.heat_step(ref, 1, 1, 1, 1.0, np.float32(0.05), out=ref.copy())
    assert rel(host(a), ref) <= RUN_TOL


def test_heat_vs_golden_reference_solver(torch_cuda):
    # Reference HeatDiffusionSolver: coefficient (sqrt(dt))^2 * alpha in float.
    f = np.load(GOLDEN / "heat_solver32.npz")
    dt = float(f["dt"])
    g = sb.Grid(32, 32, 32, 1.0, 1.0, 1.0, dt)
    a, b = dev(torch_cuda, f["u0"]), dev(torch_cuda, np.zeros_like(f["u0"]))
    for _ in range(int(f["steps"])):
        sb.heat_step(a, b, g, float(f["alpha"]))
        a, b = b, a
    assert rel(host(a), f["out"]) <= RUN_TOL


# ── reference invariants (test_kernels.cpp, test_wave_3d.cpp) on the GPU ─────────

@pytest.mark.parametrize("launch", ["naive", "tiled"])
def test_flat_field_fixed_point(torch_cuda, launch):
    n = 32
    g = sb.Grid(n, n, n, 10, 10, 10, 1e-3)
    p = dev(torch_cuda, np.full((n, n, n), 3.0, np.float32))
    v = dev(torch_cuda, np.ones((n, n, n), np.float32))
    out = dev(torch_cuda, np.zeros((n, n, n), np.float32))
    getattr(sb, f"launch_{launch}")(p, p, v, out, g)
    np.testing.assert_allclose(host(out)[4:-4, 4:-4, 4:-4], 3.0, atol=1e-5)


@pytest.mark.parametrize("launch", ["naive", "tiled"])
def test_linear_field_zero_laplacian(torch_cuda, launch):
    n = 24
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    p = (np.float32(0.1) * x + np.float32(0.2) * y + np.float32(0.3) * z).astype(np.float32)
    g = sb.Grid(n, n, n, 10, 10, 10, 1e-3)
    out = dev(torch_cuda, np.zeros_like(p))
    getattr(sb, f"launch_{launch}")(dev(torch_cuda, p), dev(torch_cuda, p),
                                   dev(torch_cuda, np.ones_like(p)), out, g)
    o = host(out)[4:-4, 4:-4, 4:-4]
    e = p[4:-4, 4:-4, 4:-4]
    assert np.all(np.abs(o - e) <= np.abs(e) * 1e-4 + 1e-6)


def test_tiled_deterministic_and_symmetric(torch_cuda):
    n = 48
    g = sb.Grid(n, n, n, 10, 10, 10, 3e-3)
    p0 = gaussian_field((n, n, n), 0.5, 0.5, 0.5, 4.0)
    vel2 = np.full((n, n, n), 1500.0 ** 2, np.float32)

    def step(p, q, v, o, grid, src, amp):
        sb.launch_tiled(p, q, v, o, grid)

    a, _ = run_gpu(torch_cuda, step, p0, p0, vel2, g, 8)
    b, _ = run_gpu(torch_cuda, step, p0, p0, vel2, g, 8)
    assert np.array_equal(a, b)  # test_wave_3d.cpp:177-192
    i = slice(4, n - 4)
    inner = a[i, i, i]
    for axis in range(3):  # test_wave_3d.cpp:121-150
        assert np.abs(inner - np.flip(inner, axis)).max() < 1e-4


def test_halo_untouched_many_steps(torch_cuda):
    n = 40
    g = sb.Grid(n, n, n, 10, 10, 10, 1e-3)
    cur, prev, vel2 = random_case((n, n, n), 9)
    p, q = run_gpu(torch_cuda, sb.wave_step, cur, prev, vel2, g, 10)
    halo = np.ones((n, n, n), bool)
    halo[4:-4, 4:-4, 4:-4] = False
    assert np.all(p[halo] == 0) and np.all(q[halo] == 0)
