"""Minimal and thin grids on every tile of every kernel family: one interior plane,
four interior columns, a single tile row or column, z splits deeper than the
interior.  FP32 acoustic and heat against the oracle (the parity tolerances),
FP16 storage against its oracle restatement, two steps per sweep bit for bit
against two one-step launches; halo cells are never written."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb
from tests.test_gpu_f16 import compare_f16, f16_case, scale_state, step_magnitude

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-6
# (nz, ny, nx): nx % 4 == 0 for the FP32 pencils
SHAPES32 = [(9, 12, 12), (9, 9, 40), (10, 33, 12), (12, 9, 16), (40, 10, 9 * 4)]
# nx % 8 == 0 for FP16 storage
SHAPES16 = [(9, 12, 16), (9, 9, 40), (10, 33, 16), (12, 9, 24)]


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    sb.upload_fd_coefficients()
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0
    for k in (sb.KIND_WAVE_F32, sb.KIND_HEAT_F32, sb.KIND_WAVE_F16, sb.KIND_WAVE2_F32):
        sb.set_pencil_override(k, -1, 1)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def halo_mask(shape):
    m = np.ones(shape, bool)
    m[4:-4, 4:-4, 4:-4] = False
    return m


def case(shape, seed):
    rng = np.random.default_rng(seed)
    m = halo_mask(shape)
    cur = np.where(m, 0, rng.standard_normal(shape)).astype(np.float32)
    prev = np.where(m, 0, cur + 0.01 * rng.standard_normal(shape)).astype(np.float32)
    vel2 = (rng.uniform(1500.0, 4500.0, shape) ** 2).astype(np.float32)
    return cur, prev, vel2


def grid_of(shape, d=10.0, dt=1e-3):
    nz, ny, nx = shape
    return sb.Grid(nx, ny, nz, d, d, d, dt)


@pytest.mark.parametrize("zchunks", [1, 5])
@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE_F32))))
@pytest.mark.parametrize("shape", SHAPES32)
def test_acoustic_thin_grids(torch_cuda, shape, variant, zchunks):
    sb.set_pencil_override(sb.KIND_WAVE_F32, variant, zchunks)
    cur, prev, vel2 = case(shape, 3 + variant)
    g = grid_of(shape)
    out = dev(torch_cuda, np.zeros(shape, np.float32))
    sb.launch_tiled(dev(torch_cuda, cur), dev(torch_cuda, prev), dev(torch_cuda, vel2), out, g)
    o = host(out)
    ref = oracle.wave_step(cur, prev, vel2, 10, 10, 10, 1e-3)
    assert oracle.rel_l2(o, ref) <= STEP_TOL
    assert np.all(o[halo_mask(shape)] == 0)


@pytest.mark.parametrize("zchunks", [1, 5])
@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_HEAT_F32))))
@pytest.mark.parametrize("shape", SHAPES32)
def test_heat_thin_grids(torch_cuda, shape, variant, zchunks):
    sb.set_pencil_override(sb.KIND_HEAT_F32, variant, zchunks)
    u, _, _ = case(shape, 5 + variant)
    g = grid_of(shape, 1.0, 0.05)
    k = np.float32(np.float32(1.0) * np.float32(0.05))
    ref = oracle.heat_step(u, 1, 1, 1, 1.0, k)
    out = dev(torch_cuda, np.zeros(shape, np.float32))
    sb.heat_step(dev(torch_cuda, u), out, g, 1.0)
    o = host(out)
    assert oracle.rel_l2(o, ref) <= STEP_TOL
    assert np.all(o[halo_mask(shape)] == 0)


@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE_F16))))
@pytest.mark.parametrize("shape", SHAPES16)
def test_fp16_thin_grids(torch_cuda, shape, variant):
    sb.set_pencil_override(sb.KIND_WAVE_F16, variant, 3)
    P, Q, K = f16_case(shape, 7 + variant)
    g = grid_of(shape)
    out = dev(torch_cuda, Q.view(np.int16))
    sb.wave_step_f16(dev(torch_cuda, P.view(np.int16)), out, dev(torch_cuda, K.view(np.int16)), g,
                     scale_state(torch_cuda, 1024.0), 0)
    got = host(out).view(np.uint16)
    ref = oracle.wave_step_f16(P, Q, K, 10.0, 10.0, 10.0)
    compare_f16(got, ref, step_magnitude(P, Q, K))
    m = halo_mask(shape)
    assert np.array_equal(got[m], Q[m])


@pytest.mark.parametrize("zchunks", [1, 5])
@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE2_F32))))
@pytest.mark.parametrize("shape", SHAPES32)
def test_two_step_thin_grids(torch_cuda, shape, variant, zchunks):
    sb.set_pencil_override(sb.KIND_WAVE2_F32, variant, zchunks)
    cur, prev, vel2 = case(shape, 9 + variant)
    g = grid_of(shape)
    p, q, v = dev(torch_cuda, cur), dev(torch_cuda, prev), dev(torch_cuda, vel2)
    src = g.index(shape[2] // 2, shape[1] // 2, shape[0] // 2)
    o1, o2 = torch_cuda.zeros_like(p), torch_cuda.zeros_like(p)
    sb.wave_step2(p, q, v, o1, o2, g, src, 0.5, -0.25)
    a, b = q.clone(), p.clone()
    sb.wave_step(p, a, v, a, g, src, 0.5)
    sb.wave_step(a, b, v, b, g, src, -0.25)
    torch_cuda.cuda.synchronize()
    assert torch_cuda.equal(o1, a) and torch_cuda.equal(o2, b)
