"""FP16-storage acoustic path: conversions, one step against the FP16 oracle
(the same scheme restated in C), renormalisation phases, and a full run against
the FP64 oracle (error reported, bounded)."""
from __future__ import annotations

import pathlib

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu
GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def scale_state(torch, a=1.0, r=1.0):
    return torch.tensor([a, r], dtype=torch.float32, device="cuda")


def test_pack_unpack_and_k_field(torch_cuda):
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(100_003) * 3).astype(np.float32)
    h = torch_cuda.empty(x.size, dtype=torch_cuda.int16, device="cuda")
    sb.f16_pack(dev(torch_cuda, x), h, x.size, 256.0)
    assert np.array_equal(host(h).view(np.uint16), oracle.to_f16(x, 256.0))
    back = torch_cuda.empty(x.size, dtype=torch_cuda.float32, device="cuda")
    sb.f16_unpack(h, back, x.size, 256.0)
    ref = oracle.to_f16(x, 256.0).view(np.float16).astype(np.float32) / np.float32(256.0)
    assert np.array_equal(host(back), ref)
    g = sb.Grid(40, 36, 28, 10.0, 10.0, 10.0, 8.5e-4)
    vel2 = rng.uniform(1500, 4500, g.shape).astype(np.float32) ** 2
    k = torch_cuda.empty(g.shape, dtype=torch_cuda.int16, device="cuda")
    sb.k_field_bf16(dev(torch_cuda, vel2), k, g)
    f = np.float32(np.float64(np.float32(8.5e-4)) ** 2 / 100.0)
    assert np.array_equal(host(k).view(np.uint16), oracle.to_bf16(vel2 * f))


def f16_case(shape, seed, scale=1024.0):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal(shape).astype(np.float32)
    q = p + 0.05 * rng.standard_normal(shape).astype(np.float32)
    for a in (p, q):
        m = np.ones(shape, bool)
        m[4:-4, 4:-4, 4:-4] = False
        a[m] = 0
    K = oracle.to_bf16(rng.uniform(0.02, 0.16, shape).astype(np.float32))
    return oracle.to_f16(p, scale), oracle.to_f16(q, scale), K


def step_magnitude(P, Q, K, m_out=1.0, m_q=1.0):
    """|m_out| (2|p| + |m_q q| + K sum |c_i| |p_i|) per interior cell, in FP64: the
    scale of the FP32 rounding error any evaluation order of the step can make."""
    c = np.abs(oracle.fd_coefficients())
    p = np.abs(P.view(np.float16).astype(np.float64))
    q = np.abs(Q.view(np.float16).astype(np.float64))
    k = np.abs((K.astype(np.uint32) << 16).view(np.float32).astype(np.float64))
    s = (slice(4, -4),) * 3
    acc = 3 * c[0] * p[s]
    for r in range(1, 5):
        for ax in range(3):
            for sg in (1, -1):
                sl = [slice(4, -4)] * 3
                sl[ax] = slice(4 + sg * r, p.shape[ax] - 4 + sg * r)
                acc = acc + c[r] * p[tuple(sl)]
    return abs(m_out) * (2 * p[s] + abs(m_q) * q[s] + k[s] * acc)


def compare_f16(got, ref, mag):
    """The kernel and the oracle sum the stencil in different orders in FP32, so a
    stored half may differ by one ulp, or, where the sum cancels to far below its
    terms, by up to 64 FP32 ulps of the terms' magnitude (mag, interior cells)."""
    s = (slice(4, -4),) * 3
    g = got.view(np.float16)[s].astype(np.float64)
    r = ref.view(np.float16)[s].astype(np.float64)
    ulp = np.spacing(np.abs(r).astype(np.float16)).astype(np.float64)
    err = np.abs(g - r)
    assert np.all(err <= ulp + 64 * 2.0**-24 * mag)
    assert np.count_nonzero(err > ulp) <= 0.005 * err.size


@pytest.mark.parametrize("phase,r", [(0, 1.0), (1, 0.5), (2, 0.5), (1, 4.0)])
@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE_F16))))
def test_f16_step_matches_oracle(torch_cuda, phase, r, variant):
    sb.set_pencil_override(sb.KIND_WAVE_F16, variant, 2)
    try:
        shape = (37, 44, 72)  # nz, ny, nx (nx % 8 == 0, ragged against the tiles)
        P, Q, K = f16_case(shape, 5 + variant)
        g = sb.Grid(72, 44, 37, 10.0, 10.0, 10.0, 1e-3)
        out = dev(torch_cuda, Q.view(np.int16))
        st = scale_state(torch_cuda, 1024.0, r)
        sb.wave_step_f16(dev(torch_cuda, P.view(np.int16)), out, dev(torch_cuda, K.view(np.int16)),
                         g, st, phase)
        ref = oracle.wave_step_f16(P, Q, K, 10.0, 10.0, 10.0,
                                   m_out=r if phase == 1 else 1.0, m_q=r if phase == 2 else 1.0)
        got = host(out).view(np.uint16)
        compare_f16(got, ref, step_magnitude(P, Q, K, r if phase == 1 else 1.0,
                                             r if phase == 2 else 1.0))
        halo = np.ones(shape, bool)
        halo[4:-4, 4:-4, 4:-4] = False
        assert np.array_equal(got[halo], Q[halo])  # never written
    finally:
        sb.set_pencil_override(sb.KIND_WAVE_F16, -1, 1)


@pytest.mark.parametrize("spacing", [(10.0, 12.0, 9.0), (10.0, 10.0, 9.0)])
def test_f16_variants_agree_bitwise(torch_cuda, spacing):
    """The per-point arithmetic does not depend on the tile shape or z split (it
    depends on the grid: the exact-y form where dx == dy)."""
    shape = (45, 52, 80)
    P, Q, K = f16_case(shape, 21)
    g = sb.Grid(80, 52, 45, *spacing, 1e-3)
    n = len(sb.variant_names(sb.KIND_WAVE_F16))
    outs = {}
    try:
        for v in range(n):
            for phase in (0, 1, 2):
                sb.set_pencil_override(sb.KIND_WAVE_F16, v, 1 + v % 3)
                out = dev(torch_cuda, Q.view(np.int16))
                sb.wave_step_f16(dev(torch_cuda, P.view(np.int16)), out,
                                 dev(torch_cuda, K.view(np.int16)), g,
                                 scale_state(torch_cuda, 1024.0, 0.5), phase)
                outs[(v, phase)] = host(out)
    finally:
        sb.set_pencil_override(sb.KIND_WAVE_F16, -1, 1)
    for (v, phase), o in outs.items():
        assert np.array_equal(o, outs[(0, phase)]), (v, phase)


def test_f16_tuner_picks_a_variant(torch_cuda):
    import ctypes as C

    g = sb.Grid(96, 80, 72, 10.0, 10.0, 10.0, 1e-3)
    P, Q, K = f16_case(g.shape, 4)
    p, q, k = (dev(torch_cuda, x.view(np.int16)) for x in (P, Q, K))
    scratch = q.clone()
    v, zc, ms = C.c_int(-1), C.c_int(-1), C.c_float(0)
    rc = sb.lib().sb200_tune(sb.KIND_WAVE_F16, sb._g(g), p.data_ptr(), q.data_ptr(), k.data_ptr(),
                             scratch.data_ptr(), 2, C.byref(v), C.byref(zc), C.byref(ms))
    assert rc == 0, sb.last_error()
    assert 0 <= v.value < sb.lib().sb200_pencil_variant_count(sb.KIND_WAVE_F16)
    assert zc.value >= 1 and ms.value > 0


@pytest.mark.parametrize("variant", range(len(sb.variant_names(sb.KIND_WAVE_F16))))
def test_f16_source_injection(torch_cuda, variant):
    """Source injection under every tile shape."""
    shape = (24, 24, 32)
    P, Q, K = f16_case(shape, 9, scale=64.0)
    g = sb.Grid(32, 24, 24, 10.0, 10.0, 10.0, 1e-3)
    src = g.index(13, 11, 12)
    out = dev(torch_cuda, Q.view(np.int16))
    sb.set_pencil_override(sb.KIND_WAVE_F16, variant, 1)
    try:
        sb.wave_step_f16(dev(torch_cuda, P.view(np.int16)), out, dev(torch_cuda, K.view(np.int16)),
                         g, scale_state(torch_cuda, 64.0), 0, src, 0.75)
    finally:
        sb.set_pencil_override(sb.KIND_WAVE_F16, -1, 1)
    ref = oracle.wave_step_f16(P, Q, K, 10.0, 10.0, 10.0, src=src, w=0.75, a=64.0)
    mag = step_magnitude(P, Q, K)
    kk = float((K.astype(np.uint32) << 16).view(np.float32).ravel()[src])
    mag[12 - 4, 11 - 4, 13 - 4] += kk * 100.0 * 0.75 * 64.0
    compare_f16(host(out).view(np.uint16), ref, mag)
    assert host(out).view(np.uint16).ravel()[src] != Q.ravel()[src]


def test_f16_renorm_picks_power_of_two(torch_cuda):
    stats = torch_cuda.tensor([0.0, 3.0 * 256.0, 0.0], dtype=torch_cuda.float64, device="cuda")
    st = scale_state(torch_cuda, 256.0)
    sb.f16_renorm(stats, st, bound_host=1.0, target=4096.0)
    a, r = host(st)
    # max|p| = 3, + bound 1 -> 4096 / 4 = 1024
    assert a == 1024.0 and r == 4.0


def test_f16_rejects_unaligned_rows(torch_cuda):
    g = sb.Grid(36, 24, 24)  # nx % 8 != 0
    z = torch_cuda.zeros(g.shape, dtype=torch_cuda.int16, device="cuda")
    with pytest.raises(sb.StencilError) as e:
        sb.wave_step_f16(z, z.clone(), z.clone(), g, scale_state(torch_cuda))
    assert e.value.status == sb.SB200_ERR_UNSUPPORTED


def test_f16_run_accuracy_vs_fp64(torch_cuda):
    """The 128^3 acoustic case (Ricker at the centre, 300 steps) with FP16
    storage: relative L2 against the FP64 oracle's mid plane."""
    f = np.load(GOLDEN / "acoustic128_300.npz")
    n = 128
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 1e-3)
    z = np.zeros(g.shape, np.float32)
    v = np.full(g.shape, 2000.0 ** 2, np.float32)
    with sb.Run(g, precision=sb.PRECISION_F16, src_index=int(f["src"]), src_freq=15.0) as run:
        run.set_fields(z, z, v)
        run.steps(300)
        p = run.field()
        tr = run.trace(300)
    err = oracle.rel_l2(p[n // 2], f["mid64"])
    terr = oracle.rel_l2(tr, f["trace32"])
    print(f"FP16 storage, 300 steps: rel L2 vs FP64 {err:.3e}, trace {terr:.3e}")
    assert err < 3e-2 and terr < 3e-2
