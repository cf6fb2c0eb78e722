"""Generates tests/golden/* from the reference's own CPU path (oracle/_ref).

Run in a checkout where the reference sources are available (oracle/build.py
compiles them).  Every output is produced by the reference's code --
stencil::launch_naive (src/kernels/stencil_naive.cu:136-170, -ffp-contract=off
build, plus an FP64 build) and stencil::make_solver (src/solver/*.cpp) -- on
inputs defined here, so the fixtures pin the oracle restatement and the CUDA
path without the reference being present at test time.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from oracle import build as obuild  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    obuild.build_oracle()
    built = obuild.build_reference()
    if "f32_strict" not in built:
        raise SystemExit("reference sources not found: cannot generate golden fixtures")
    manifest = {}

    # 1. KernelTest.NaiveHaloCellsRemainZero inputs (tests/unit/test_kernels.cpp:202-215):
    #    24^3, dx=10, dt=1e-3, vel2=1, Gaussian sigma=3 as p and p_prev, one step.
    n = 24
    g = oracle.ref_init_gaussian((n, n, n), 0.5, 0.5, 0.5, 3.0)
    v = np.ones((n, n, n), np.float32)
    out = oracle.ref_wave_step(g, g, v, 10.0, 10.0, 10.0, 1e-3)
    np.savez_compressed(HERE / "wave_gauss24.npz", p=g, vel2=v, out=out,
                        dx=10.0, dt=1e-3)
    manifest["wave_gauss24"] = {"source": "stencil::launch_naive (CPU, -ffp-contract=off)",
                                "sha256_out": sha(out)}

    # 2. KernelCorrectness.NaiveMatchesCPUReference (test_kernel_correctness.cpp:78-108):
    #    Config 32^3, v=1500, dx=10, sigma=4, dt from Config::make_grid, one step of the
    #    reference solver (make_solver -> WavePropSolver::step).
    n = 32
    dt = oracle.ref().ref_make_grid_dt(10.0, 1500.0)
    g = oracle.ref_init_gaussian((n, n, n), 0.5, 0.5, 0.5, 4.0)
    out = oracle.ref_solver_run(0, n, 10.0, 1500.0, 1e-4, 4.0, 1)
    np.savez_compressed(HERE / "wave_solver32.npz", p=g, out=out, dx=10.0, dt=dt,
                        velocity=1500.0)
    manifest["wave_solver32"] = {"source": "stencil::make_solver wave/naive, 1 step",
                                 "dt": dt, "sha256_out": sha(out)}

    # 3. Heterogeneous velocity, Ricker source, 40 steps, non-cubic grid.
    rng = np.random.default_rng(20261203)
    shape = (28, 36, 44)  # (nz, ny, nx)
    vel = rng.uniform(1500.0, 3000.0, shape)
    vel2 = (vel * vel).astype(np.float32)
    cur = np.zeros(shape, np.float32)
    prev = np.zeros(shape, np.float32)
    nz, ny, nx = shape
    src = (nz // 2 * ny + ny // 2) * nx + nx // 2
    steps = 40
    w = oracle.ricker(15.0, 1.0 / 15.0, 1e-3, steps)
    c32, p32 = oracle.ref_wave_run(cur.copy(), prev.copy(), vel2, 10.0, 10.0, 10.0, 1e-3, steps,
                                   src, w)
    c64, p64 = oracle.ref_wave_run(cur.astype(np.float64), prev.astype(np.float64),
                                   vel2.astype(np.float64), 10.0, 10.0, 10.0, 1e-3, steps, src, w,
                                   variant="f64")
    np.savez_compressed(HERE / "wave_src_44x36x28.npz", vel2=vel2, src=src, wavelet=w,
                        cur=c32, prev=p32, cur64=c64, dx=10.0, dt=1e-3, steps=steps)
    manifest["wave_src_44x36x28"] = {"source": "stencil::launch_naive x40 + source rule",
                                     "sha256_cur": sha(c32), "sha256_prev": sha(p32)}

    # 4. Odd extents (interior 17 x 23 x 29; nx % 4 != 0), Gaussian, 6 steps.
    shape = (37, 31, 25)
    g = oracle.ref_init_gaussian(shape, 0.45, 0.5, 0.55, 3.0)
    vel2 = np.full(shape, 2000.0 ** 2, np.float32)
    c32, p32 = oracle.ref_wave_run(g.copy(), g.copy(), vel2, 10.0, 10.0, 10.0, 1e-3, 6)
    np.savez_compressed(HERE / "wave_odd_25x31x37.npz", p=g, vel2=vel2, cur=c32, prev=p32,
                        dx=10.0, dt=1e-3, steps=6)
    manifest["wave_odd_25x31x37"] = {"source": "stencil::launch_naive x6",
                                     "sha256_cur": sha(c32)}

    # 5. Heat through the reference solver (HeatDiffusionSolver, heat_diffusion.cpp:73-122):
    #    32^3, dx=1, velocity 500 (dt = 0.45*dx/v), diffusivity 1e-2, sigma 5, 10 steps.
    n = 32
    out = oracle.ref_solver_run(1, n, 1.0, 500.0, 1e-2, 5.0, 10)
    dt = oracle.ref().ref_make_grid_dt(1.0, 500.0)
    g = oracle.ref_init_gaussian((n, n, n), 0.5, 0.5, 0.5, 5.0)
    np.savez_compressed(HERE / "heat_solver32.npz", u0=g, out=out, dx=1.0, dt=dt,
                        alpha=1e-2, steps=10)
    manifest["heat_solver32"] = {"source": "stencil::make_solver heat/naive, 10 steps",
                                 "dt": dt, "sha256_out": sha(out)}

    # 6. Acoustic config: 128^3 (120^3 interior), dx=10 m, v=2000 m/s, dt=1 ms,
    #    15 Hz Ricker (t0 = 1/f) at the centre cell, p = p_prev = 0, 300 steps.
    n, steps = 128, 300
    shape = (n, n, n)
    vel2 = np.full(shape, 2000.0 ** 2, np.float32)
    src = (n // 2 * n + n // 2) * n + n // 2
    w = oracle.ricker(15.0, 1.0 / 15.0, 1e-3, steps)
    c32 = np.zeros(shape, np.float32)
    p32 = np.zeros(shape, np.float32)
    tr32 = np.zeros(steps, np.float32)
    # trace by stepping the reference one step at a time
    buf = [p32, c32, np.zeros(shape, np.float32)]
    ip, ic, inn = 0, 1, 2
    for s in range(steps):
        oracle.ref_wave_step(buf[ic], buf[ip], vel2, 10.0, 10.0, 10.0, 1e-3, out=buf[inn])
        k = np.float32(np.float32(1e-3) * np.float32(1e-3)) * vel2.flat[src]
        buf[inn].flat[src] = np.float32(buf[inn].flat[src] + np.float32(k * np.float32(w[s])))
        tr32[s] = buf[inn].flat[src]
        ip, ic, inn = ic, inn, ip
    fin32 = buf[ic].copy()
    c64, p64 = oracle.ref_wave_run(np.zeros(shape), np.zeros(shape), vel2.astype(np.float64),
                                   10.0, 10.0, 10.0, 1e-3, steps, src, w, variant="f64")
    np.savez_compressed(HERE / "acoustic128_300.npz", trace32=tr32,
                        mid32=fin32[n // 2], mid64=c64[n // 2], src=src, wavelet=w)
    manifest["acoustic128_300"] = {
        "source": "stencil::launch_naive x300 (f32 strict and f64) + source rule",
        "sha256_final32": sha(fin32),
        "rel_l2_f32_vs_f64": float(np.linalg.norm((fin32 - c64).ravel()) /
                                   np.linalg.norm(c64.ravel())),
    }

    (HERE / "manifest.json").write_text(json.dumps(manifest, indent=2) + "\n")
    print(json.dumps(manifest, indent=2))


if __name__ == "__main__":
    main()
