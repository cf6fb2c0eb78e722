"""Two acoustic steps per sweep (sb200_wave_step2_f32) against two one-step
launches of sb200_wave_step_f32: the same bits, fields and halos, on ragged grids,
every tile shape and z split, with a source near a tile corner; and the argument
checks."""
from __future__ import annotations

import numpy as np
import pytest

import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0


def fields(torch, g, seed):
    rng = np.random.default_rng(seed)
    shape = g.shape
    m = np.zeros(shape, bool)
    m[4:-4, 4:-4, 4:-4] = True
    p = np.where(m, rng.standard_normal(shape), 0).astype(np.float32)
    q = np.where(m, rng.standard_normal(shape), 0).astype(np.float32)
    v = rng.uniform(1500.0, 4500.0, shape).astype(np.float32) ** 2
    return [torch.from_numpy(a).cuda() for a in (p, q, v)]


def one_step_pair(torch, p, q, v, g, src, w0, w1):
    """Two in-place one-step launches: returns (p at t+dt, p at t+2dt)."""
    a, b = q.clone(), p.clone()
    sb.wave_step(p, a, v, a, g, src, w0)
    sb.wave_step(a, b, v, b, g, src, w1)
    return a, b


@pytest.mark.parametrize("zchunks", [1, 2, 3])
@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE2_F32))))
@pytest.mark.parametrize("shape", [(76, 45, 37), (44, 41, 30)])
def test_two_steps_match_two_one_step_launches(torch_cuda, variant, zchunks, shape):
    nx, ny, nz = shape
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 7e-4)
    p, q, v = fields(torch_cuda, g, 7 + variant)
    # a source one cell inside the first tile's corner: the neighbouring tiles'
    # widened regions hold it too
    src = g.index(5, 6, 9)
    sb.set_pencil_override(sb.KIND_WAVE2_F32, variant, zchunks)
    try:
        o1 = torch_cuda.zeros_like(p)
        o2 = torch_cuda.zeros_like(p)
        sb.wave_step2(p, q, v, o1, o2, g, src, 0.75, -0.5)
    finally:
        sb.set_pencil_override(sb.KIND_WAVE2_F32, -1, 1)
    r1, r2 = one_step_pair(torch_cuda, p, q, v, g, src, 0.75, -0.5)
    torch_cuda.cuda.synchronize()
    assert torch_cuda.equal(o1, r1)
    assert torch_cuda.equal(o2, r2)


def test_twenty_steps_match(torch_cuda):
    g = sb.Grid(72, 64, 48, 10.0, 12.0, 9.0, 6e-4)
    p, q, v = fields(torch_cuda, g, 3)
    src = g.index(30, 33, 20)
    w = np.sin(np.arange(20) * 0.3).astype(np.float32)
    a, b = p.clone(), q.clone()  # one-step: current a, previous b (in place)
    for k in range(20):
        sb.wave_step(a, b, v, b, g, src, float(w[k]))
        a, b = b, a
    bufs = [p.clone(), q.clone(), torch_cuda.zeros_like(p), torch_cuda.zeros_like(p)]
    cur, prev, o1, o2 = bufs
    for k in range(0, 20, 2):
        sb.wave_step2(cur, prev, v, o1, o2, g, src, float(w[k]), float(w[k + 1]))
        cur, prev, o1, o2 = o2, o1, cur, prev
    torch_cuda.cuda.synchronize()
    assert torch_cuda.equal(cur, a) and torch_cuda.equal(prev, b)


def test_device_wavelet_and_trace_match(torch_cuda):
    """The device-sample form reads wavelet[*step + off] and the next sample, and
    records the source cell after each step: the same field and trace as the run
    engine's two one-step launches."""
    g = sb.Grid(48, 40, 36, 10.0, 10.0, 10.0, 7e-4)
    p, q, v = fields(torch_cuda, g, 11)
    src = g.index(20, 21, 17)
    wav = torch_cuda.tensor([0.1, 0.2, 0.9, -0.4, 0.3], device="cuda")
    step = torch_cuda.tensor([1], dtype=torch_cuda.int32, device="cuda")
    trace = torch_cuda.full((5,), -7.0, device="cuda")
    o1, o2 = torch_cuda.zeros_like(p), torch_cuda.zeros_like(p)
    sb.wave_step2_dev(p, q, v, o1, o2, g, src, wav, step, 1, trace=trace)
    r1, r2 = one_step_pair(torch_cuda, p, q, v, g, src, 0.9, -0.4)
    torch_cuda.cuda.synchronize()
    assert torch_cuda.equal(o1, r1) and torch_cuda.equal(o2, r2)
    t = trace.cpu().numpy()
    assert t[0] == -7.0 and t[1] == -7.0 and t[4] == -7.0  # only indices 2 and 3 written
    with sb.Run(g, src_index=src, graph_chunk=0) as run:
        run.set_fields(p.cpu().numpy(), q.cpu().numpy(), v.cpu().numpy())
        run.set_wavelet(np.array([0.9, -0.4, 0.0], np.float32))
        run.steps(2)
        field, tr = run.field(), run.trace(2)
    assert np.array_equal(field, o2.cpu().numpy())
    assert np.array_equal(t[2:4], tr)


def test_argument_checks(torch_cuda):
    g = sb.Grid(40, 36, 32)
    p, q, v = fields(torch_cuda, g, 1)
    o1, o2 = torch_cuda.zeros_like(p), torch_cuda.zeros_like(p)
    for args in ((p, q, v, q, o2), (p, q, v, o1, p), (p, q, v, o1, o1), (p, p, v, o1, o2)):
        with pytest.raises(sb.StencilError) as e:
            sb.wave_step2(*args, g)
        assert e.value.status == sb.SB200_ERR_INVALID
    g2 = sb.Grid(42, 36, 32)  # nx % 4 != 0
    z = [torch_cuda.zeros(g2.shape, device="cuda") for _ in range(5)]
    with pytest.raises(sb.StencilError) as e:
        sb.wave_step2(*z, g2)
    assert e.value.status == sb.SB200_ERR_UNSUPPORTED
