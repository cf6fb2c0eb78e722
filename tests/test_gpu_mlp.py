"""The learned-correction kernels against the oracle: feature rows (bit-exact),
forward and gradients of the BF16 mma network (tolerances in the tests), the
fused correction kernel, restriction, box injection, and that Adam training
lowers the loss."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def net_and_rows(seed, n):
    rng = np.random.default_rng(seed)
    w = (rng.standard_normal(sb.MLP_NPARAM) * 0.3).astype(np.float32)
    w[:1024].reshape(32, 32)[:, 26:] = 0
    X = oracle.to_bf16(rng.uniform(-1, 1, (n, 32)).astype(np.float32))
    X[:, 26:] = 0
    t = rng.standard_normal(n).astype(np.float32)
    return w, X, t


def field_case(seed, shape=(40, 36, 44)):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal(shape).astype(np.float32)
    v2 = rng.uniform(1500, 4500, shape).astype(np.float32) ** 2
    m = np.ones(shape, bool)
    m[4:-4, 4:-4, 4:-4] = False
    p[m] = 0
    return p, v2


def interior_cells(shape):
    nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(4, nz - 4), np.arange(4, ny - 4), np.arange(4, nx - 4),
                          indexing="ij")
    return ((z * ny + y) * nx + x).ravel().astype(np.int64)


def test_samples_are_bit_exact(torch_cuda):
    torch = torch_cuda
    p, v2 = field_case(1)
    nz, ny, nx = p.shape
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 8e-4)
    rng = np.random.default_rng(2)
    pt = (p + 0.01 * rng.standard_normal(p.shape)).astype(np.float32)
    pp = (p + 0.01 * rng.standard_normal(p.shape)).astype(np.float32)
    cells = rng.choice(interior_cells(p.shape), 500, replace=False)
    X = torch.empty((500, 32), dtype=torch.int16, device="cuda")
    t = torch.empty(500, dtype=torch.float32, device="cuda")
    sb.mlp_samples(dev(torch, p), dev(torch, v2), dev(torch, pt), dev(torch, pp), g,
                   dev(torch, cells), X, t)
    torch.cuda.synchronize()
    Xh, th = X.cpu().numpy().view(np.uint16), t.cpu().numpy()
    dtdx = np.float32(np.float32(8e-4) / np.float32(10.0))
    for r, c in enumerate(cells):
        row, s = oracle.mlp_features(p, v2, c, dtdx)
        assert np.array_equal(Xh[r], row)
        assert th[r] == (np.float32(pt.flat[c] - pp.flat[c]) / np.float32(s))


def test_forward_matches_oracle(torch_cuda):
    torch = torch_cuda
    w, X, _ = net_and_rows(3, 1000)
    with sb.Mlp() as m:
        m.set_params(w)
        y = torch.empty(1000, dtype=torch.float32, device="cuda")
        m.forward(dev(torch, X.view(np.int16)), y)
        yg = y.cpu().numpy()
    ref = oracle.mlp_forward(w, X, round_bf16=True)
    # FP32 accumulation vs double; h1 rounds to BF16 on both sides, so an
    # FP32-level difference can move one h1 by a BF16 ulp: bounded by 2e-2 of the scale.
    assert np.max(np.abs(yg - ref)) <= 2e-2 * (1 + np.max(np.abs(ref)))
    assert np.median(np.abs(yg - ref)) <= 1e-5 * (1 + np.max(np.abs(ref)))


def test_gradients_match_oracle(torch_cuda):
    torch = torch_cuda
    w, X, t = net_and_rows(4, 4096)
    with sb.Mlp() as m:
        m.set_params(w)
        grad = torch.empty(sb.MLP_NPARAM + 1, dtype=torch.float32, device="cuda")
        m.gradients(dev(torch, X.view(np.int16)), dev(torch, t), grad)
        gg = grad.cpu().numpy().astype(np.float64)
    loss, ref = oracle.mlp_grad(w, X, t, round_bf16=True)
    assert abs(gg[-1] - loss) <= 1e-4 * loss
    # per parameter block: relative L2 of the difference
    blocks = {"W1": slice(0, 1024), "b1": slice(1024, 1056), "W2": slice(1056, 2080),
              "b2": slice(2080, 2112), "w3": slice(2112, 2144), "b3": slice(2144, 2145)}
    for name, sl in blocks.items():
        d = np.linalg.norm(gg[sl] - ref[sl]) / max(np.linalg.norm(ref[sl]), 1e-12)
        assert d <= 5e-3, (name, d)


def test_training_lowers_the_loss(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(5)
    n = 1 << 15
    F = rng.uniform(-1, 1, (n, 26)).astype(np.float32)
    target = (0.5 * F[:, 0] - 0.25 * F[:, 1:9].sum(1) + 0.1 * np.maximum(F[:, 9], 0)).astype(np.float32)
    X = np.zeros((n, 32), np.uint16)
    X[:, :26] = oracle.to_bf16(F)
    Xd, td = dev(torch, X.view(np.int16)), dev(torch, target)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    with sb.Mlp(seed=11) as m:
        losses = []
        for step in range(300):
            sl = slice((step * 4096) % n, (step * 4096) % n + 4096)
            m.train_step(Xd[sl], td[sl], 3e-3, loss)
            if step % 50 == 0 or step == 299:
                losses.append(float(loss.item()))
    assert losses[-1] < 0.1 * losses[0], losses


def test_correct_kernel_adds_scaled_mlp(torch_cuda):
    torch = torch_cuda
    p, v2 = field_case(6, (24, 20, 40))
    nz, ny, nx = p.shape
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 8e-4)
    w, _, _ = net_and_rows(7, 1)
    base = np.random.default_rng(8).standard_normal(p.shape).astype(np.float32)
    with sb.Mlp() as m:
        m.set_params(w)
        m.output_scale = 0.5
        out = dev(torch, base)
        m.correct(dev(torch, p), dev(torch, v2), out, g)
        got = out.cpu().numpy()
    dtdx = np.float32(np.float32(8e-4) / np.float32(10.0))
    cells = interior_cells(p.shape)
    rows = np.zeros((cells.size, 32), np.uint16)
    s = np.zeros(cells.size, np.float64)
    for r, c in enumerate(cells):
        rows[r], s[r] = oracle.mlp_features(p, v2, c, dtdx)
    ref = base.ravel().astype(np.float64).copy()
    ref[cells] += 0.5 * s * oracle.mlp_forward(w, rows, True)
    err = np.abs(got.ravel() - ref)
    assert np.max(err[cells]) <= 2e-2 * (1 + np.max(np.abs(s)))
    halo = np.ones(p.size, bool)
    halo[cells] = False
    assert np.array_equal(got.ravel()[halo], base.ravel()[halo])


def test_restrict2(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(9)
    fine = rng.standard_normal((56, 48, 40)).astype(np.float32)
    fg = sb.Grid(40, 48, 56, 5.0, 5.0, 5.0, 4e-4)
    cg = sb.Grid(24, 28, 32, 10.0, 10.0, 10.0, 8e-4)
    out = torch.full(cg.shape, 7.0, device="cuda")
    sb.restrict2(dev(torch, fine), fg, out, cg, -4)
    got = out.cpu().numpy()
    ref = np.zeros(cg.shape, np.float32)
    for z in range(4, 28):
        for y in range(4, 24):
            for x in range(4, 20):
                fz, fy, fx = 2 * z - 4, 2 * y - 4, 2 * x - 4
                if fz < 56 and fy < 48 and fx < 40:
                    ref[z, y, x] = fine[fz, fy, fx]
    assert np.array_equal(got, ref)


def test_add_box_skips_the_halo(torch_cuda):
    torch = torch_cuda
    g = sb.Grid(24, 20, 16)
    f = torch.zeros(g.shape, device="cuda")
    pat = torch.arange(1, 7 * 7 * 7 + 1, dtype=torch.float32, device="cuda")
    sb.add_box(f, g, (1, 2, 3), (7, 7, 7), pat, 0.5)
    got = f.cpu().numpy()
    ref = np.zeros(g.shape, np.float32)
    pv = pat.cpu().numpy().reshape(7, 7, 7)
    for k in range(7):
        for j in range(7):
            for i in range(7):
                x, y, z = 1 + i, 2 + j, 3 + k
                if 4 <= x < 20 and 4 <= y < 16 and 4 <= z < 12:
                    ref[z, y, x] += 0.5 * pv[k, j, i]
    assert np.array_equal(got, ref)


def test_tcgen05_and_mma_correction_agree(torch_cuda):
    """The tcgen05 (TMEM) correction and the mma.sync one: same BF16 operands, FP32
    accumulation in a different order, so equal up to FP32 rounding and the odd
    BF16 flip of a hidden activation."""
    torch = torch_cuda
    p, v2 = field_case(10, (40, 36, 72))
    nz, ny, nx = p.shape
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 8e-4)
    w, _, _ = net_and_rows(12, 1)
    outs = {}
    with sb.Mlp() as m:
        m.set_params(w)
        m.output_scale = 0.25
        for kern in ("mma", "tcgen05", "tcgen05"):
            out = torch.zeros(g.shape, device="cuda")
            m.set_kernel(kern)
            m.correct(dev(torch, p), dev(torch, v2), out, g)
            outs.setdefault(kern, []).append(out.cpu().numpy())
    a, b = outs["mma"][0], outs["tcgen05"][0]
    scale = np.max(np.abs(a))
    assert scale > 0
    assert np.max(np.abs(a - b)) <= 2e-2 * scale
    assert np.median(np.abs(a - b)) <= 1e-5 * scale
    assert np.array_equal(outs["tcgen05"][0], outs["tcgen05"][1])  # deterministic


@pytest.mark.parametrize("shape,mode", [((40, 36, 72), "dense"), ((29, 45, 40), "dense"),
                                        ((36, 52, 80), "sparse"), ((32, 40, 64), "wide")])
def test_learned_step_is_step_plus_correction(torch_cuda, shape, mode):
    """The fused learned step gives the same bits as the FP32 acoustic step
    followed by the tcgen05 correction: ragged tiles in x and y, unequal
    spacings, an all-zero slab whose planes skip the network, (sparse) a
    field that is zero but for a small blob, so most threads and warps of the
    active planes skip the features and epilogues, and (wide) magnitudes
    spread from 2^10 down into the FP32 subnormals, as in the tail of a wave
    front, where the features must be scaled before their BF16 rounding."""
    torch = torch_cuda
    rng = np.random.default_rng(13)
    nz, ny, nx = shape
    p = rng.standard_normal(shape).astype(np.float32)
    p[: nz // 3] = 0.0
    if mode == "sparse":
        blob = p[14:21, 20:27, 33:41].copy()
        p[:] = 0.0
        p[14:21, 20:27, 33:41] = blob
    elif mode == "wide":
        e2 = rng.uniform(-149.0, 10.0, shape)
        p = np.where(p != 0.0, np.sign(p) * np.exp2(e2), 0.0).astype(np.float32)
        assert (np.abs(p[p != 0]) < np.finfo(np.float32).tiny).any()
    q = rng.standard_normal(shape).astype(np.float32)
    v2 = rng.uniform(1500, 4500, shape).astype(np.float32) ** 2
    g = sb.Grid(nx, ny, nz, 10.0, 12.0, 9.0, 8e-4)
    w, X, t = net_and_rows(14, 4096)
    with sb.Mlp() as m:
        m.set_params(w)
        m.output_scale = 0.3
        m.set_kernel("tcgen05")
        P, V = dev(torch, p), dev(torch, v2)
        for trained in (False, True):
            if trained:  # parameters changed on the device: the fused step re-reads them
                loss = torch.zeros(1, dtype=torch.float32, device="cuda")
                m.train_step(dev(torch, X.view(np.int16)), dev(torch, t), 1e-2, loss)
            ref = dev(torch, q)
            sb.wave_step(P, ref, V, ref, g)
            m.correct(P, V, ref, g)
            got = dev(torch, q)
            m.learned_step(P, got, V, g)
            plain = dev(torch, q)
            sb.wave_step(P, plain, V, plain, g)
            assert not torch.equal(ref, plain)  # the correction is not zero
            assert torch.equal(got, ref), float((got - ref).abs().max())


def test_learned_step_needs_aligned_rows(torch_cuda):
    torch = torch_cuda
    g = sb.Grid(38, 20, 20)  # nx % 4 != 0
    z = torch.zeros(g.shape, device="cuda")
    with sb.Mlp() as m:
        with pytest.raises(sb.StencilError) as e:
            m.learned_step(z, z.clone(), z.clone(), g)
    assert e.value.status == sb.SB200_ERR_UNSUPPORTED


def test_correction_floor(torch_cuda):
    """Points whose star stays below the floor get no correction, in the
    standalone kernels and the fused step alike (bitwise), and the others are
    corrected as without a floor: a field ramped over five decades along x."""
    torch = torch_cuda
    rng = np.random.default_rng(17)
    shape = (28, 24, 96)
    nz, ny, nx = shape
    ramp = (10.0 ** np.linspace(-5, 0, nx)).astype(np.float32)
    p = rng.standard_normal(shape).astype(np.float32) * ramp
    q = rng.standard_normal(shape).astype(np.float32) * ramp
    v2 = rng.uniform(1500, 4500, shape).astype(np.float32) ** 2
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 8e-4)
    w, _, _ = net_and_rows(18, 1)
    P, V = dev(torch, p), dev(torch, v2)
    outs = {}
    with sb.Mlp() as m:
        m.set_params(w)
        m.output_scale = 0.3
        for floor in (0.0, 1e-2):
            m.min_scale = floor
            assert m.min_scale == np.float32(floor)
            for kern in ("tcgen05", "mma"):
                m.set_kernel(kern)
                ref = dev(torch, q)
                sb.wave_step(P, ref, V, ref, g)
                m.correct(P, V, ref, g)
                outs[(floor, kern)] = ref.cpu().numpy()
            got = dev(torch, q)
            m.learned_step(P, got, V, g)
            outs[(floor, "fused")] = got.cpu().numpy()
        with pytest.raises(sb.StencilError):
            m.min_scale = -1.0
    plain = dev(torch, q)
    sb.wave_step(P, plain, V, plain, g)
    plain = plain.cpu().numpy()
    for floor in (0.0, 1e-2):
        assert np.array_equal(outs[(floor, "fused")], outs[(floor, "tcgen05")])
    # star maxima: points below the floor are plain steps; the rest match no floor
    pad = np.pad(np.abs(p), 4)
    m_star = np.zeros(shape, np.float32)
    for axis in range(3):
        for r in range(-4, 5):
            m_star = np.maximum(m_star, np.roll(pad, r, axis)[4:-4, 4:-4, 4:-4])
    inner = np.zeros(shape, bool)
    inner[4:-4, 4:-4, 4:-4] = True
    fl = np.float32(1e-2)
    low, high = inner & (m_star < fl), inner & (m_star >= fl)
    assert low.sum() > 1000 and high.sum() > 1000
    for kern in ("tcgen05", "mma"):
        f, nf = outs[(1e-2, kern)], outs[(0.0, kern)]
        assert np.array_equal(f[low], plain[low])
        assert np.array_equal(f[high], nf[high])
        assert not np.array_equal(nf[low], plain[low])


@pytest.mark.parametrize("floor", [0.0, 2.0 ** -20])
def test_learned_step_flags_keep_the_bits(torch_cuda, floor):
    """Activity flags: over 14 steps of a sparse field with a source box added
    after every step, the flagged fused step (chunks far from any value at the
    floor take the plain path) gives the same bits as the unflagged one and as
    the acoustic step followed by the correction; the flags mark some chunks
    idle and some active."""
    torch = torch_cuda
    nz, ny, nx = 100, 64, 96
    rng = np.random.default_rng(31)
    p0 = np.zeros((nz, ny, nx), np.float32)
    p0[10:18, 8:14, 10:20] = rng.standard_normal((8, 6, 10))
    v2 = rng.uniform(1500, 4500, (nz, ny, nx)).astype(np.float32) ** 2
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 8e-4)
    w, _, _ = net_and_rows(15, 1)
    origin, dims = (60, 40, 70), (5, 4, 3)  # a source box far from the blob
    pat = torch.from_numpy(rng.uniform(0.5, 1.0, dims[::-1]).astype(np.float32)).cuda()
    box = (origin[0], origin[0] + dims[0], origin[1], origin[1] + dims[1], origin[2],
           origin[2] + dims[2])
    V = dev(torch, v2)
    with sb.Mlp() as m:
        m.set_params(w)
        m.output_scale = 0.3
        m.min_scale = floor
        m.set_kernel("tcgen05")
        n = m.flags_bytes(g)
        assert n > 0
        states = {k: [dev(torch, p0), dev(torch, p0)] for k in ("ref", "fused", "flags")}
        fl = [torch.full((n,), 255, dtype=torch.uint8, device="cuda"),
              torch.zeros(n, dtype=torch.uint8, device="cuda")]
        idle = active = 0
        for step in range(14):
            for k, (p, q) in states.items():
                if k == "ref":
                    sb.wave_step(p, q, V, q, g)
                    m.correct(p, V, q, g)
                elif k == "fused":
                    m.learned_step(p, q, V, g)
                else:
                    m.learned_step(p, q, V, g, flags=(fl[0], fl[1]), box=box)
                sb.add_box(q, g, origin, dims, pat, 0.25 * (step % 3 + 1))
                states[k] = [q, p]
            f = fl[1].cpu().numpy()
            idle += int((f == 0).sum())
            active += int((f != 0).sum())
            fl.reverse()
        torch.cuda.synchronize()
        for k in ("fused", "flags"):
            for a, b in zip(states[k], states["ref"]):
                assert torch.equal(a, b), (k, float((a - b).abs().max()))
        assert idle > 0 and active > 0, (idle, active)
        assert not torch.equal(states["ref"][0], dev(torch, p0))


def test_composed_flags_keep_the_bits(torch_cuda):
    """The composition pre-pass (r = p + c L p, p_prev += 2 c L p) followed by the
    fused step on r: with the flags of r composed from those of p
    (sb200_mlp_flags_compose) and the source box grown by the stencil radius, 14
    steps of a sparse field with a source box give the same bits as the same
    steps without flags, and some chunks take the plain path."""
    torch = torch_cuda
    nz, ny, nx = 100, 64, 96
    rng = np.random.default_rng(37)
    p0 = np.zeros((nz, ny, nx), np.float32)
    p0[10:18, 8:14, 10:20] = rng.standard_normal((8, 6, 10))
    v2 = rng.uniform(1500, 4500, (nz, ny, nx)).astype(np.float32) ** 2
    g = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 8e-4)
    w, _, _ = net_and_rows(15, 1)
    origin, dims = (60, 40, 70), (5, 4, 3)
    pat = torch.from_numpy(rng.uniform(0.5, 1.0, dims[::-1]).astype(np.float32)).cuda()
    box = (origin[0] - 4, origin[0] + dims[0] + 4, origin[1] - 4, origin[1] + dims[1] + 4,
           origin[2] - 4, origin[2] + dims[2] + 4)
    V = dev(torch, v2)
    with sb.Mlp() as m:
        m.set_params(w)
        m.output_scale = 0.3
        m.min_scale = 2.0 ** -20
        m.set_kernel("tcgen05")
        n = m.flags_bytes(g)
        states = {k: [dev(torch, p0), dev(torch, p0)] for k in ("plain", "flags")}
        r = {k: torch.zeros_like(states[k][0]) for k in states}
        fl = [torch.full((n,), 255, dtype=torch.uint8, device="cuda"),
              torch.zeros(n, dtype=torch.uint8, device="cuda"),
              torch.zeros(n, dtype=torch.uint8, device="cuda")]
        idle = 0
        for step in range(14):
            for k, (p, q) in states.items():
                sb.wave_prepass(p, q, V, r[k], g, 1.0 / 16.0)
                if k == "plain":
                    m.learned_step(r[k], q, V, g)
                else:
                    m.flags_compose(g, fl[0], fl[2])
                    idle += int((fl[2].cpu().numpy() == 0).sum())
                    m.learned_step(r[k], q, V, g, flags=(fl[2], fl[1]), box=box)
                sb.add_box(q, g, origin, dims, pat, 0.25 * (step % 3 + 1))
                states[k] = [q, p]
            fl[0], fl[1] = fl[1], fl[0]
        torch.cuda.synchronize()
        for a, b in zip(states["flags"], states["plain"]):
            assert torch.equal(a, b), float((a - b).abs().max())
        assert idle > 0
        assert sb.device_error() == 0
