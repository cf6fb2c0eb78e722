"""sb200_field_stats_f32_noalloc (static device scratch, allocates nothing)
against sb200_field_stats_f32 (caller scratch): the same kernels and block
count, so the same bits, call after call.  Collected last on purpose: it must
pass after every other test has used the library, as well as alone."""
from __future__ import annotations

import numpy as np
import pytest

import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu


def _field(torch, g, seed, plant_nan=False):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(g.shape).astype(np.float32)
    if plant_nan:
        a[g.nz // 2, g.ny // 2, g.nx // 2] = np.nan
        a[5, 6, 7] = np.inf
    return torch.from_numpy(a).cuda()


def _with_scratch(torch, f, g):
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    scratch = torch.empty(sb.field_stats_scratch_len(g), dtype=torch.float64, device="cuda")
    sb.field_stats(f, g, out, scratch)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _noalloc(torch, f, g):
    out = torch.full((3,), -1.0, dtype=torch.float64, device="cuda")
    sb.field_stats_noalloc(f, g, out)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("shape", [(72, 44, 37), (264, 200, 136)])
def test_noalloc_matches_scratch_entry_point_twice(torch_cuda, shape):
    torch = torch_cuda
    nx, ny, nz = shape
    g = sb.Grid(nx, ny, nz)
    fa = _field(torch, g, 1)
    fb = _field(torch, g, 2, plant_nan=True)
    ref_a, ref_b = _with_scratch(torch, fa, g), _with_scratch(torch, fb, g)
    # Two calls in a row on different fields: nothing of the first call's
    # partials may leak into the second.
    got_a = _noalloc(torch, fa, g)
    got_b = _noalloc(torch, fb, g)
    assert np.array_equal(got_a, ref_a)
    assert np.array_equal(got_b, ref_b)
    assert got_b[2] == 2.0
    # and once more in the opposite order
    assert np.array_equal(_noalloc(torch, fb, g), ref_b)
    assert np.array_equal(_noalloc(torch, fa, g), ref_a)
    assert sb.device_error() == 0


def test_noalloc_on_a_stream_matches(torch_cuda):
    torch = torch_cuda
    g = sb.Grid(128, 96, 80)
    f = _field(torch, g, 3)
    ref = _with_scratch(torch, f, g)
    s = torch.cuda.Stream()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    s.wait_stream(torch.cuda.current_stream())  # f and out were written on the default stream
    with torch.cuda.stream(s):
        sb.field_stats_noalloc(f, g, out, stream=s)
        sb.field_stats_noalloc(f, g, out, stream=s)
    s.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)


def test_noalloc_allocates_nothing(torch_cuda):
    """After the first call on the device (which may load the library's module),
    further calls leave the device's free memory and torch's allocator as they
    were: the partials live in the static array."""
    torch = torch_cuda
    g = sb.Grid(200, 136, 96)
    f = _field(torch, g, 4)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    sb.field_stats_noalloc(f, g, out)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0, reserved0 = torch.cuda.memory_allocated(), torch.cuda.memory_reserved()
    for _ in range(20):
        sb.field_stats_noalloc(f, g, out)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert (torch.cuda.memory_allocated(), torch.cuda.memory_reserved()) == (alloc0, reserved0)
    assert np.array_equal(out.cpu().numpy(), _with_scratch(torch, f, g))


def test_noalloc_rejects_bad_arguments(torch_cuda):
    torch = torch_cuda
    z = torch.zeros(8 * 8 * 8, dtype=torch.float32, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    with pytest.raises(sb.StencilError) as e:
        sb.field_stats_noalloc(z, sb.Grid(8, 8, 8), out)  # no interior
    assert e.value.status == sb.SB200_ERR_INVALID
    assert "noalloc" in str(e.value)
