"""Batched shots (sb200_batch_*): uneven grids advanced by one persistent launch
per step.  Each shot must match the single-grid run engine bit for bit (same
per-point arithmetic) and the FP32 oracle within the full-run bound, for every
tile variant and z-chunk length, eager and through CUDA graphs."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu

STEPS = 60


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    yield
    assert sb.device_error() == 0


def make_shots(seed=7, dims=((40, 48, 36), (64, 40, 56), (32, 32, 32), (56, 24, 44), (48, 64, 40))):
    rng = np.random.default_rng(seed)
    shots = []
    for nx, ny, nz in dims:
        g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 1e-3)
        vel2 = (rng.uniform(1500.0, 3000.0, g.shape) ** 2).astype(np.float32)
        src = g.index(int(rng.integers(4, nx - 4)), int(rng.integers(4, ny - 4)),
                      int(rng.integers(4, nz - 4)))
        f = float(rng.uniform(10.0, 25.0))
        w = oracle.ricker(f, 1.0 / f, 1e-3, STEPS).astype(np.float32)
        shots.append((g, src, vel2, w))
    return shots


def run_batch(shots, steps=STEPS, chunk=20, choice=None, split=(7, 53)):
    with sb.Batch([(g, s) for g, s, _, _ in shots], max_steps=steps, graph_chunk=chunk) as b:
        if choice is not None:
            b.set_choice(*choice)
        for i, (g, _, v, w) in enumerate(shots):
            z = np.zeros(g.shape, np.float32)
            b.set_fields(i, z, z, v)
            b.set_wavelet(i, w)
        for k in split:
            b.steps(k)
        b.synchronize()
        return [(b.field(i), b.trace(i, steps)) for i in range(len(shots))]


def test_batch_matches_single_grid_runs_bitwise():
    shots = make_shots()
    got = run_batch(shots)
    for (g, src, v, w), (p, tr) in zip(shots, got):
        z = np.zeros(g.shape, np.float32)
        with sb.Run(g, src_index=src, graph_chunk=0) as r:
            r.set_fields(z, z, v)
            r.set_wavelet(w)
            r.steps(STEPS)
            ref_p, ref_tr = r.field(), r.trace(STEPS)
        assert np.array_equal(p, ref_p)
        assert np.array_equal(tr, ref_tr)


def test_batch_matches_oracle():
    shots = make_shots(seed=11)
    got = run_batch(shots)
    for (g, src, v, w), (p, tr) in zip(shots, got):
        z = np.zeros(g.shape, np.float32)
        cur, _, otr = oracle.wave_run(z.copy(), z.copy(), v, 10.0, 10.0, 10.0, 1e-3, STEPS,
                                      src=src, wavelet=w.astype(np.float64), trace=True)
        assert oracle.rel_l2(p, cur) <= 1e-5
        assert oracle.rel_l2(tr, otr) <= 1e-5


@pytest.mark.parametrize("zlen", [0, 16])
def test_batch_every_variant_agrees(zlen):
    shots = make_shots(seed=3)
    base = run_batch(shots, choice=(0, 64))
    for v in range(sb.lib().sb200_batch_variant_count()):
        got = run_batch(shots, choice=(v, zlen), chunk=0, split=(STEPS,))
        for (p0, t0), (p, t) in zip(base, got):
            assert np.array_equal(p, p0) and np.array_equal(t, t0)


def test_batch_tune_then_run():
    shots = make_shots(seed=5, dims=((64, 64, 64), (40, 72, 48)))
    with sb.Batch([(g, s) for g, s, _, _ in shots], max_steps=STEPS, graph_chunk=20) as b:
        b.tune(reps=2)
        assert b.steps_done == 0
        c = b.choice()
        assert 0 <= c["variant"] < sb.lib().sb200_batch_variant_count() and c["items"] > 0
        assert np.count_nonzero(b.field(0)) == 0
        for i, (g, _, v, w) in enumerate(shots):
            z = np.zeros(g.shape, np.float32)
            b.set_fields(i, z, z, v)
            b.set_wavelet(i, w)
        b.steps(STEPS)
        p = b.field(1)
    ref = run_batch(shots)
    assert np.array_equal(p, ref[1][0])


def test_batch_rejects_bad_shots():
    g = sb.Grid(42, 40, 40)  # nx % 4 != 0
    with pytest.raises(sb.StencilError) as e:
        sb.Batch([(g, None)], max_steps=10)
    assert e.value.status == sb.SB200_ERR_UNSUPPORTED
    g = sb.Grid(40, 40, 40)
    with pytest.raises(sb.StencilError) as e:
        sb.Batch([(g, g.index(2, 20, 20))], max_steps=10)  # source in the halo
    assert e.value.status == sb.SB200_ERR_INVALID
    with sb.Batch([(g, g.index(20, 20, 20))], max_steps=10, graph_chunk=0) as b:
        b.steps(10)
        with pytest.raises(sb.StencilError) as e:
            b.steps(1)
        assert e.value.status == sb.SB200_ERR_INVALID


def run_batch_f16(shots, steps=120, chunk=50, choice=None, split=(7, 113)):
    with sb.Batch([(g, s) for g, s, _, _ in shots], max_steps=steps, graph_chunk=chunk,
                  precision=sb.PRECISION_F16) as b:
        if choice is not None:
            b.set_choice(*choice)
        for i, (g, _, v, w) in enumerate(shots):
            z = np.zeros(g.shape, np.float32)
            b.set_fields(i, z, z, v)
            b.set_wavelet(i, w)
        for k in split:
            b.steps(k)
        b.synchronize()
        return [(b.field(i), b.trace(i, steps)) for i in range(len(shots))]


def test_f16_batch_matches_single_grid_f16_runs_bitwise():
    """FP16-storage batch: per-shot power-of-two scales renormalised every 50
    steps (eager steps and a captured 50-step chunk), bit for bit the FP16 run
    engine on each shot alone."""
    steps = 120
    shots = make_shots(seed=21)
    shots = [(g, s, v, np.pad(w, (0, steps - len(w)))) for g, s, v, w in shots]
    got = run_batch_f16(shots, steps=steps)
    for (g, src, v, w), (p, tr) in zip(shots, got):
        z = np.zeros(g.shape, np.float32)
        with sb.Run(g, src_index=src, graph_chunk=0, precision=sb.PRECISION_F16) as r:
            r.set_fields(z, z, v)
            r.set_wavelet(w)
            r.steps(steps)
            ref_p, ref_tr = r.field(), r.trace(steps)
        assert np.abs(p).max() > 0
        assert np.array_equal(p, ref_p)
        assert np.array_equal(tr, ref_tr)


@pytest.mark.parametrize("zlen", [0, 16])
def test_f16_batch_every_variant_agrees(zlen):
    steps = 60
    shots = make_shots(seed=23)
    base = run_batch_f16(shots, steps=steps, choice=(0, 64), split=(60,))
    for v in range(sb.lib().sb200_batch_variant_count_f16()):
        got = run_batch_f16(shots, steps=steps, choice=(v, zlen), split=(60,))
        for (p0, t0), (p1, t1) in zip(base, got):
            assert np.array_equal(p0, p1), v
            assert np.array_equal(t0, t1), v


def test_f16_batch_tune_and_validation():
    shots = make_shots(seed=25)
    with sb.Batch([(g, s) for g, s, _, _ in shots], max_steps=20, graph_chunk=0,
                  precision=sb.PRECISION_F16) as b:
        b.tune(reps=1)
        c = b.choice()
        assert 0 <= c["variant"] < sb.lib().sb200_batch_variant_count_f16() and c["items"] > 0
    g = sb.Grid(36, 32, 32)  # nx % 8 != 0
    with pytest.raises(sb.StencilError):
        sb.Batch([(g, None)], max_steps=10, graph_chunk=0, precision=sb.PRECISION_F16)
    g = sb.Grid(40, 32, 32)
    with pytest.raises(sb.StencilError):  # a chunk that does not start on a renorm
        sb.Batch([(g, None)], max_steps=100, graph_chunk=30, precision=sb.PRECISION_F16)


@pytest.mark.parametrize("precision,chunk", [(sb.PRECISION_F32, 0), (sb.PRECISION_F32, 10),
                                             (sb.PRECISION_F16, 50)])
def test_batch_monitor_flags_the_shot_that_blows_up(precision, chunk):
    """A non-finite value in one shot trips that shot's monitor (eager steps,
    graph chunks, FP16 renormalisation statistics) and synchronize fails; the
    other shots stay clear, and new fields clear the flag."""
    shots = make_shots(seed=27)[:3]
    with sb.Batch([(g, s) for g, s, _, _ in shots], max_steps=120, graph_chunk=chunk,
                  precision=precision) as b:
        for i, (g, _, v, w) in enumerate(shots):
            p = np.zeros(g.shape, np.float32)
            if i == 1:
                p[g.nz // 2, g.ny // 2, g.nx // 2] = np.nan
            b.set_fields(i, p, p, v)
            b.set_wavelet(i, w)
        b.steps(60 if precision == sb.PRECISION_F16 else 20)
        with pytest.raises(sb.StencilError) as e:
            b.synchronize()
        assert e.value.status == sb.SB200_ERR_MONITOR and "shot 1" in str(e.value)
        assert list(b.monitor_flags()) == [0, 1, 0]
        g, _, v, _ = shots[1]
        z = np.zeros(g.shape, np.float32)
        b.set_fields(1, z, z, v)
        assert list(b.monitor_flags()) == [0, 0, 0]


def test_batch_monitor_limit():
    shots = make_shots(seed=29)[:2]
    with sb.Batch([(g, s) for g, s, _, _ in shots], max_steps=STEPS, graph_chunk=0) as b:
        for i, (g, _, v, w) in enumerate(shots):
            z = np.zeros(g.shape, np.float32)
            b.set_fields(i, z, z, v)
            b.set_wavelet(i, w)
        b.steps(20)
        b.synchronize()
        peak = max(float(np.abs(b.field(i)).max()) for i in range(2))
        assert peak > 0
        b.set_monitor_limit(peak / 2)
        b.steps(1)
        with pytest.raises(sb.StencilError) as e:
            b.synchronize()
        assert e.value.status == sb.SB200_ERR_MONITOR
        assert b.monitor_flags().sum() >= 1


THIN = ((12, 9, 9), (40, 12, 10), (16, 33, 9), (40, 36, 36))  # nx, ny, nz


@pytest.mark.parametrize("precision", [sb.PRECISION_F32, sb.PRECISION_F16])
def test_batch_thin_shots_match_single_grid_runs(precision):
    """Minimal shots (four interior columns, one interior plane, one tile row)
    beside a normal one, every tile variant and z-chunk length: each shot bit for
    bit the single-grid run engine on that grid alone."""
    f16 = precision == sb.PRECISION_F16
    steps = 24
    dims = tuple((max(16, nx) if f16 else nx, ny, nz) for nx, ny, nz in THIN)
    shots = [(g, s, v, w[:steps]) for g, s, v, w in make_shots(seed=31, dims=dims)]
    refs = []
    for g, src, v, w in shots:
        z = np.zeros(g.shape, np.float32)
        with sb.Run(g, src_index=src, graph_chunk=0, precision=precision) as r:
            r.set_fields(z, z, v)
            r.set_wavelet(np.pad(w, (0, 1)))
            r.steps(steps)
            refs.append((r.field(), r.trace(steps)))
    nvar = (sb.lib().sb200_batch_variant_count_f16() if f16
            else sb.lib().sb200_batch_variant_count())
    runner = run_batch_f16 if f16 else run_batch
    for v in range(nvar):
        for zlen in (0, 1):
            got = runner(shots, steps=steps, chunk=0, choice=(v, zlen), split=(5, steps - 5))
            for (p, tr), (rp, rtr) in zip(got, refs):
                assert np.array_equal(p, rp), (v, zlen)
                assert np.array_equal(tr, rtr), (v, zlen)
