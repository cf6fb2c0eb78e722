"""Accuracy against the FP64 oracle on the precision configuration's accuracy
case: a 256^3 instance of the seeded layered model (dx 10 m, Courant 0.4 at
v_max, 15 Hz Ricker at the centre), 500 steps from rest, through the run handle
(CUDA-graph chunks) in FP32 and in FP16 storage (renormalised every 50 steps).
Bars: FP32 field and trace within 1e-4 of FP64; FP16 receiver trace within 1e-3
(the target); FP16 field within 3e-2 (16-bit storage of p carries ~2.4e-4
relative rounding per step, which the leapfrog accumulates: ~1.8e-2 here)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import stencil_solver_b200 as sb

pytestmark = pytest.mark.gpu


def test_fp32_and_fp16_against_fp64_256_500():
    n, steps, dx = 256, 500, 10.0
    vel2, vmax = sb.model_layered(n, n, n, 1234)
    dt = float(np.float32(0.4 * dx / vmax))
    g = sb.Grid(n, n, n, dx, dx, dx, dt)
    src = g.index(n // 2, n // 2, n // 2)
    w = sb.ricker(15.0, 1.0 / 15.0, dt, steps)
    z = np.zeros(g.shape, np.float32)
    got = {}
    for prec in (sb.PRECISION_F32, sb.PRECISION_F16):
        with sb.Run(g, precision=prec, src_index=src) as r:
            r.set_fields(z, z, vel2)
            r.set_wavelet(w)
            r.steps(steps)
            got[prec] = (r.field().astype(np.float64), r.trace(steps).astype(np.float64))
    cur = np.zeros(g.shape, np.float64)
    prev = np.zeros(g.shape, np.float64)
    ref, _, tr = oracle.wave_run(cur, prev, vel2.astype(np.float64), dx, dx, dx, dt, steps, src,
                                 w.astype(np.float64), trace=True)
    e32 = (oracle.rel_l2(got[sb.PRECISION_F32][0], ref), oracle.rel_l2(got[sb.PRECISION_F32][1], tr))
    e16 = (oracle.rel_l2(got[sb.PRECISION_F16][0], ref), oracle.rel_l2(got[sb.PRECISION_F16][1], tr))
    print("rel L2 vs FP64 (field, trace): fp32", e32, "fp16", e16)
    assert e32[0] <= 1e-4 and e32[1] <= 1e-4
    assert e16[1] <= 1e-3
    assert e16[0] <= 3e-2
