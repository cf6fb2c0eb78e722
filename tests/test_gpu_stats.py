"""FP64 field statistics (stability monitor / FP16 scale input) against NumPy."""
from __future__ import annotations

import numpy as np
import pytest

import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu


def interior(a):
    return a[4:-4, 4:-4, 4:-4]


def run_stats(torch, field, grid, scale=1.0):
    n = sb.field_stats_scratch_len(grid)
    scratch = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    sb.field_stats(field, grid, out, scratch, scale)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("shape", [(20, 24, 28), (37, 31, 25), (96, 80, 72)])
def test_stats_f32_match_numpy(torch_cuda, shape):
    rng = np.random.default_rng(sum(shape))
    a = rng.standard_normal(shape).astype(np.float32) * 3
    nz, ny, nx = shape
    g = sb.Grid(nx, ny, nz)
    s = run_stats(torch_cuda, torch_cuda.from_numpy(a).cuda(), g)
    i = interior(a).astype(np.float64)
    assert s[0] == pytest.approx(np.sum(i * i), rel=1e-12)
    assert s[1] == np.abs(i).max()
    assert s[2] == 0


def test_stats_ignore_halo_and_count_nonfinite(torch_cuda):
    shape = (24, 24, 24)
    a = np.ones(shape, np.float32)
    a[0, 0, 0] = 1e30          # halo: ignored
    a[10, 11, 12] = np.nan     # planted on the host
    a[5, 6, 7] = np.inf
    a[6, 6, 6] = -5.0
    s = run_stats(torch_cuda, torch_cuda.from_numpy(a).cuda(), sb.Grid(24, 24, 24))
    n_int = 16 ** 3
    assert s[2] == 2
    assert s[1] == 5.0
    assert s[0] == pytest.approx((n_int - 3) * 1.0 + 25.0)


def test_stats_f16_with_scale(torch_cuda):
    shape = (28, 30, 32)
    rng = np.random.default_rng(3)
    v = rng.uniform(-2, 2, shape).astype(np.float16)
    scale = 1024.0
    stored = (v.astype(np.float32) * scale).astype(np.float16)
    s = run_stats(torch_cuda, torch_cuda.from_numpy(stored).cuda(), sb.Grid(32, 30, 28), scale)
    i = interior(stored).astype(np.float64) / scale
    assert s[0] == pytest.approx(np.sum(i * i), rel=1e-12)
    assert s[1] == np.abs(i).max()


def test_stats_bit_reproducible(torch_cuda):
    a = torch_cuda.randn(64, 72, 80, device="cuda")
    g = sb.Grid(80, 72, 64)
    s1 = run_stats(torch_cuda, a, g)
    s2 = run_stats(torch_cuda, a, g)
    assert np.array_equal(s1, s2)


def test_stats_scratch_too_small_rejected(torch_cuda):
    g = sb.Grid(64, 64, 64)
    a = torch_cuda.zeros(64, 64, 64, device="cuda")
    out = torch_cuda.zeros(3, dtype=torch_cuda.float64, device="cuda")
    small = torch_cuda.zeros(2, dtype=torch_cuda.float64, device="cuda")
    with pytest.raises(sb.StencilError, match="scratch"):
        sb.field_stats(a, g, out, small)
