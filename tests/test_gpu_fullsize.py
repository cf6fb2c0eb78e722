"""The hot path at the configurations' full sizes, checked through properties
that do not need a full-size oracle run: one step of the 1024^3 FP32 acoustic
grid (2^30 cells, byte offsets past 2^32) and of the 2048^3 FP16 grid (2^33
cells) at 4096 sampled interior points against a float64 restatement of the
stencil from the gathered stars (tolerance: FP32 rounding of the terms, plus
one FP16 ulp for the stored halves), linearity of the FP32 step under a
power-of-two scaling (bit for bit), two steps per sweep at 1024^3 against two
one-step launches (bit for bit), and one heat step of the 512^3 grid."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu
R = 4


def sample_points(torch, shape, n, seed):
    """Flat indices of n interior cells, the far corner among them."""
    nz, ny, nx = shape
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    z = torch.randint(R, nz - R, (n,), generator=gen, device="cuda")
    y = torch.randint(R, ny - R, (n,), generator=gen, device="cuda")
    x = torch.randint(R, nx - R, (n,), generator=gen, device="cuda")
    z[0], y[0], x[0] = nz - R - 1, ny - R - 1, nx - R - 1
    return (z * ny + y) * nx + x


def stars(torch, field, idx, shape):
    """(n, 25) float64: centre, then the +-r neighbours of x, y, z (r = 1..4)."""
    nz, ny, nx = shape
    flat = field.reshape(-1)
    cols = [flat[idx]]
    for stride in (1, nx, nx * ny):
        for r in range(1, R + 1):
            cols.append(flat[idx + r * stride])
            cols.append(flat[idx - r * stride])
    return torch.stack(cols, 1).double().cpu().numpy()


def lap_terms(st, wx, wy, wz, c0):
    """Laplacian (weights per axis, float64) and the sum of |terms|."""
    c = st[:, 0]
    lap = c0 * (wx + wy + wz) * c
    mag = np.abs(c0 * (wx + wy + wz) * c)
    k = 1
    for w in (wx, wy, wz):
        for r in range(1, R + 1):
            pair = st[:, k] + st[:, k + 1]
            lap = lap + w * oracle.fd_coefficients()[r] * pair
            mag = mag + w * abs(oracle.fd_coefficients()[r]) * (np.abs(st[:, k]) + np.abs(st[:, k + 1]))
            k += 2
    return lap, mag


def test_acoustic_1024_sampled_and_linear(torch_cuda):
    torch = torch_cuda
    n = 1024
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 8.5e-4)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(11)
    p = torch.randn(g.shape, generator=gen, device="cuda")
    q = torch.randn(g.shape, generator=gen, device="cuda")
    v = torch.rand(g.shape, generator=gen, device="cuda") * (4500.0 ** 2 - 1500.0 ** 2) + 1500.0 ** 2
    out = torch.zeros(g.shape, device="cuda")
    sb.wave_step(p, q, v, out, g)
    idx = sample_points(torch, g.shape, 4096, 12)
    st = stars(torch, p, idx, g.shape)
    qs = q.reshape(-1)[idx].double().cpu().numpy()
    vs = v.reshape(-1)[idx].double().cpu().numpy()
    got = out.reshape(-1)[idx].double().cpu().numpy()
    dt2, inv = float(np.float32(8.5e-4)) ** 2, 1.0 / 100.0
    lap, mag = lap_terms(st, inv, inv, inv, oracle.fd_coefficients()[0])
    ref = 2 * st[:, 0] - qs + dt2 * vs * lap
    tol = 4e-6 * (2 * np.abs(st[:, 0]) + np.abs(qs) + dt2 * vs * mag) + 1e-30
    assert np.all(np.abs(got - ref) <= tol), float(np.max(np.abs(got - ref) / tol))
    # halo cells are never written
    assert float(out[:R].abs().max()) == 0.0 and float(out[:, :, -R:].abs().max()) == 0.0
    # linearity: 2^k p, 2^k q give 2^k times the step, bit for bit
    out2 = torch.zeros_like(out)
    sb.wave_step(p * 4.0, q * 4.0, v, out2, g)
    assert torch.equal(out2, out * 4.0)


def test_two_step_1024_equals_two_one_step_launches(torch_cuda):
    """Two steps per sweep on the 1024^3 grid (byte offsets past 2^32, random
    halos): bit for bit two in-place one-step launches, the outputs' halos
    started as the walls they stand for (p_prev's for t+dt, p's for t+2dt)."""
    torch = torch_cuda
    n = 1024
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 8.5e-4)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(21)
    p = torch.randn(g.shape, generator=gen, device="cuda")
    q = torch.randn(g.shape, generator=gen, device="cuda")
    v = torch.rand(g.shape, generator=gen, device="cuda") * (4500.0 ** 2 - 1500.0 ** 2) + 1500.0 ** 2
    src = g.index(512, 500, 700)
    o1, o2 = q.clone(), p.clone()
    sb.wave_step2(p, q, v, o1, o2, g, src, 0.75, -0.5)
    a, b = q.clone(), p.clone()
    sb.wave_step(p, a, v, a, g, src, 0.75)
    sb.wave_step(a, b, v, b, g, src, -0.5)
    torch.cuda.synchronize()
    assert torch.equal(o1, a) and torch.equal(o2, b)


def test_fp16_2048_sampled(torch_cuda):
    torch = torch_cuda
    n = 2048
    g = sb.Grid(n, n, n, 10.0, 10.0, 10.0, 8.5e-4)
    free, _ = torch.cuda.mem_get_info()
    if free < 60e9:
        pytest.skip("needs ~52 GB of device memory")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(21)
    P = torch.empty(g.shape, dtype=torch.int16, device="cuda")
    Q = torch.empty_like(P)
    K = torch.empty_like(P)
    for z0 in range(0, n, 256):  # fill by slabs (no FP32 copy of the whole grid)
        sl = slice(z0, z0 + 256)
        shp = (256, n, n)
        P[sl] = (torch.randn(shp, generator=gen, device="cuda") * 512).half().view(torch.int16)
        Q[sl] = (torch.randn(shp, generator=gen, device="cuda") * 512).half().view(torch.int16)
        K[sl] = (torch.rand(shp, generator=gen, device="cuda") * 0.14 + 0.02).bfloat16().view(torch.int16)
    for f in (P, Q):  # zero walls
        f[:R] = 0
        f[-R:] = 0
        f[:, :R] = 0
        f[:, -R:] = 0
        f[:, :, :R] = 0
        f[:, :, -R:] = 0
    idx = sample_points(torch, g.shape, 4096, 22)

    def halves(t):
        return t.view(torch.float16)

    st = stars(torch, halves(P), idx, g.shape)
    qs = halves(Q).reshape(-1)[idx].double().cpu().numpy()
    ks = K.view(torch.bfloat16).reshape(-1)[idx].double().cpu().numpy()
    sb.wave_step_f16(P, Q, K, g, torch.tensor([512.0, 1.0], device="cuda"), 0)
    got = halves(Q).reshape(-1)[idx].double().cpu().numpy()
    lap, mag = lap_terms(st, 1.0, 1.0, 1.0, oracle.fd_coefficients()[0])
    ref = 2 * st[:, 0] - qs + ks * lap
    ulp = np.spacing(np.abs(ref).astype(np.float16)).astype(np.float64)
    tol = ulp + 64 * 2.0 ** -24 * (2 * np.abs(st[:, 0]) + np.abs(qs) + ks * mag)
    assert np.all(np.abs(got - ref) <= tol), float(np.max(np.abs(got - ref) / tol))


def test_heat_512_sampled(torch_cuda):
    """The heat configuration's grid (512^3, alpha dt / dx^2 = 0.05, U[0, 1)
    interior, zero walls): one step at sampled points against float64."""
    torch = torch_cuda
    n = 512
    g = sb.Grid(n, n, n, 1.0, 1.0, 1.0, 0.05)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(31)
    u = torch.rand(g.shape, generator=gen, device="cuda")
    u[:R] = 0
    u[-R:] = 0
    u[:, :R] = 0
    u[:, -R:] = 0
    u[:, :, :R] = 0
    u[:, :, -R:] = 0
    out = torch.zeros_like(u)
    sb.heat_step(u, out, g, 1.0)
    idx = sample_points(torch, g.shape, 4096, 32)
    st = stars(torch, u, idx, g.shape)
    got = out.reshape(-1)[idx].double().cpu().numpy()
    lap, mag = lap_terms(st, 1.0, 1.0, 1.0, oracle.fd_coefficients()[0])
    k = float(np.float32(0.05))
    ref = st[:, 0] + k * lap
    tol = 4e-6 * (np.abs(st[:, 0]) + k * mag) + 1e-30
    assert np.all(np.abs(got - ref) <= tol), float(np.max(np.abs(got - ref) / tol))
