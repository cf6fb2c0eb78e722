"""The run engine behind the C-ABI handle (sb200_run_*) and make_solver:
golden parity through CUDA graphs, bit-exact reference-order mode, graph vs
eager equivalence, heat, and the FP64 stability monitor."""
from __future__ import annotations

import pathlib

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb
from tests.conftest import gaussian_field

pytestmark = pytest.mark.gpu
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0


def acoustic128(**opts):
    f = np.load(GOLDEN / "acoustic128_300.npz")
    n = 128
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-3)
    z = np.zeros(g.shape, np.float32)
    v = np.full(g.shape, 2000.0 ** 2, np.float32)
    run = sb.Run(g, src_index=int(f["src"]), src_freq=15.0, **opts)
    run.set_fields(z, z, v)
    return f, run


def test_run_fp32_graphs_match_reference():
    f, run = acoustic128(graph_chunk=100)
    with run:
        run.steps(300)
        p, tr = run.field(), run.trace(300)
    assert oracle.rel_l2(p[64], f["mid32"]) <= 1e-5
    assert oracle.rel_l2(tr, f["trace32"]) <= 1e-5


def test_run_exact_mode_is_bit_identical_to_reference():
    f, run = acoustic128(graph_chunk=100, exact=1)
    with run:
        # The golden samples were taken at t = n * 1e-3 in double; the run's own
        # Ricker uses the grid's FP32 dt, a few ulps away.  Bit equality is about
        # the stepping, so both sides get the same samples.
        run.set_wavelet(f["wavelet"])
        run.steps(300)
        p, tr = run.field(), run.trace(300)
    assert np.array_equal(tr, f["trace32"])
    assert np.array_equal(p[64], f["mid32"])


def test_slices_hold_the_reference_mid_plane(tmp_path):
    """Frames written through the plane read-back (exact mode): the frame after
    300 steps is the reference's mid plane bit for bit, frame 0 the initial state."""
    from stencil_solver_b200.slices import read_slices, write_slices

    f, run = acoustic128(graph_chunk=100, exact=1)
    with run:
        run.set_wavelet(f["wavelet"])
        n = write_slices(run, tmp_path / "wave", 300, 100, velocity=2000.0)
        full = run.field()
    meta, frames = read_slices(tmp_path / "wave")
    assert n == 4 and meta["plane_index"] == 64
    assert not frames[0].any()
    assert np.array_equal(frames[3], f["mid32"])
    assert np.array_equal(frames[3], full[64])


def test_plane_readback_fp16_is_the_field_plane():
    n = 40
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-3)
    p0 = gaussian_field(g.shape, sigma=4.0)
    v = np.full(g.shape, 1800.0 ** 2, np.float32)
    with sb.Run(g, precision=sb.PRECISION_F16, graph_chunk=0) as r:
        r.set_fields(p0, p0, v)
        r.steps(7)
        full = r.field()
        for z in (0, 17, n - 1):
            assert np.array_equal(r.plane(z), full[z])
        with pytest.raises(sb.StencilError):
            r.plane(n)


def test_run_graph_and_eager_agree_across_parity():
    n = 48
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-3)
    p0 = gaussian_field(g.shape, sigma=4.0)
    v = np.full(g.shape, 1800.0 ** 2, np.float32)
    outs = []
    for chunk, pieces in ((0, [203]), (20, [3, 200]), (20, [1, 41, 161])):
        with sb.Run(g, graph_chunk=chunk, src_index=g.index(20, 21, 22), src_freq=20.0) as r:
            r.set_fields(p0, p0, v)
            for k in pieces:
                r.steps(k)
            outs.append((r.field(), r.trace(203)))
    for p, t in outs[1:]:
        assert np.array_equal(p, outs[0][0]) and np.array_equal(t, outs[0][1])


def test_run_heat_matches_reference_solver():
    f = np.load(GOLDEN / "heat_solver32.npz")
    g = sb.Grid(32, 32, 32, 1.0, 1.0, 1.0, float(f["dt"]))
    with sb.Run(g, physics=sb.PHYSICS_HEAT, diffusivity=float(f["alpha"]), graph_chunk=4) as r:
        r.set_fields(f["u0"])
        r.steps(int(f["steps"]))
        u = r.field()
    assert oracle.rel_l2(u, f["out"]) <= 1e-5


def test_monitor_trips_on_planted_nan():
    n = 32
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-3)
    p0 = gaussian_field(g.shape, sigma=3.0)
    p0[10, 12, 14] = np.nan  # planted on the host
    v = np.full(g.shape, 2000.0 ** 2, np.float32)
    with sb.Run(g, monitor_every=1, graph_chunk=0) as r:
        r.set_fields(p0, p0, v)
        r.steps(2)
        with pytest.raises(sb.StencilError) as e:
            r.synchronize()
        assert e.value.status == sb.SB200_ERR_MONITOR


def test_monitor_trips_on_blow_up_inside_graphs():
    n = 32
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-2)  # Courant 2.0: unstable
    p0 = gaussian_field(g.shape, sigma=3.0)
    v = np.full(g.shape, 2000.0 ** 2, np.float32)
    with sb.Run(g, graph_chunk=10, monitor_limit=1e6) as r:
        r.set_fields(p0, p0, v)
        r.steps(60)
        with pytest.raises(sb.StencilError) as e:
            r.synchronize()
        assert e.value.status == sb.SB200_ERR_MONITOR


def test_stats_of_run():
    n = 40
    g = sb.Grid(n, n, n)
    p0 = gaussian_field(g.shape, sigma=4.0)
    v = np.full(g.shape, 1500.0 ** 2, np.float32)
    with sb.Run(g) as r:
        r.set_fields(p0, p0, v)
        s = r.stats()
    i = p0[4:-4, 4:-4, 4:-4].astype(np.float64)
    assert s[0] == pytest.approx(np.sum(i * i), rel=1e-12) and s[1] == np.abs(i).max()


def test_caller_wavelet_is_kept_and_bounds_the_run():
    n = 24
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-3)
    z = np.zeros(g.shape, np.float32)
    v = np.full(g.shape, 2000.0 ** 2, np.float32)
    w = np.linspace(1.0, 2.0, 12).astype(np.float32)
    with sb.Run(g, src_index=g.index(12, 12, 12), src_freq=15.0, graph_chunk=0) as r:
        r.set_fields(z, z, v)
        r.set_wavelet(w)
        r.steps(12)
        tr = r.trace(12)
        with pytest.raises(sb.StencilError) as e:
            r.steps(1)
        assert e.value.status == sb.SB200_ERR_INVALID
    # first step from rest: p = dt^2 vel2 w[0] at the source
    k = np.float32(np.float32(1e-3) * np.float32(1e-3)) * np.float32(2000.0 ** 2)
    assert tr[0] == np.float32(k * w[0])
