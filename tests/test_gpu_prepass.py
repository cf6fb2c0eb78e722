"""sb200_wave_prepass_f32 (the coarse step's composition pre-pass) against the
FP64 oracle, through the C ABI.

The pre-pass writes r = p + beta dt^2 L p and p_prev + 2 beta dt^2 L p
(L = vel2 lap); a plain acoustic step of (r, p_prev) must then equal
2 p - p_prev + dt^2 L p + beta dt^4 L^2 p.  L is evaluated by the oracle's FP64
restatement of the reference CPU step (src/kernels/stencil_naive.cu:136-170)
with dt = 1 and prev = cur: next - cur = vel2 lap(cur).  Tolerance: the FP32
one-step parity bar, relative L2 <= 1e-6.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb
from tests.test_gpu_parity import STEP_TOL, dev, host, random_case, rel

pytestmark = pytest.mark.gpu


def _interior(shape):
    m = np.zeros(shape, bool)
    m[4:-4, 4:-4, 4:-4] = True
    return m


def lap_v(f, vel2, d):
    """vel2 * lap(f) in float64 on the interior (halo zero)."""
    f64 = np.asarray(f, np.float64)
    return oracle.wave_step(f64, f64, np.asarray(vel2, np.float64), *d, 1.0) - \
        np.where(_interior(f.shape), f64, 0.0)


@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE_F32))))
def test_prepass_against_fp64(torch_cuda, variant):
    torch = torch_cuda
    sb.set_pencil_override(sb.KIND_WAVE_F32, variant, 2)
    try:
        shape = (40, 52, 68)  # nz, ny, nx: ragged against the tiles
        d = (9.0, 12.0, 10.0)  # dx, dy, dz
        dt, beta = 1.2e-3, 1.0 / 16.0
        cur, prev, vel2 = random_case(shape, 31 + variant)
        g = sb.Grid(shape[2], shape[1], shape[0], *d, dt)
        p, q, v = dev(torch, cur), dev(torch, prev), dev(torch, vel2)
        r = torch.zeros_like(p)
        sb.wave_prepass(p, q, v, r, g, beta)
        lp = beta * dt * dt * lap_v(cur, vel2, d)
        assert rel(host(r), cur + lp) <= STEP_TOL
        assert rel(host(q), prev + 2 * lp) <= STEP_TOL
        assert np.array_equal(host(p), cur)  # p is read only
        halo = ~_interior(shape)
        assert np.all(host(r)[halo] == 0) and np.array_equal(host(q)[halo], prev[halo])
        # the plain step of (r, p_prev') carries the beta dt^4 L^2 term
        sb.wave_step(r, q, v, q, g)
        L1 = lap_v(cur, vel2, d)
        L2 = lap_v(L1, vel2, d)
        want = np.where(_interior(shape),
                        2.0 * cur - prev + dt * dt * L1 + beta * dt ** 4 * L2, prev)
        assert rel(host(q), want) <= STEP_TOL
    finally:
        sb.set_pencil_override(sb.KIND_WAVE_F32, -1, 1)
    assert sb.device_error() == 0


def test_prepass_rejects_bad_arguments(torch_cuda):
    torch = torch_cuda
    g = sb.Grid(32, 32, 32, 10, 10, 10, 1e-3)
    a = torch.zeros(g.shape, device="cuda")
    b = torch.zeros_like(a)
    with pytest.raises(sb.StencilError) as e:
        sb.wave_prepass(a, b, a, a, g)  # r aliases p
    assert e.value.status == sb.SB200_ERR_INVALID
    odd = sb.Grid(30, 32, 32, 10, 10, 10, 1e-3)  # nx % 4 != 0: no pencil kernel
    x = torch.zeros(odd.shape, device="cuda")
    with pytest.raises(sb.StencilError) as e:
        sb.wave_prepass(x, x.clone(), x.clone(), x.clone(), odd)
    assert e.value.status == sb.SB200_ERR_UNSUPPORTED
