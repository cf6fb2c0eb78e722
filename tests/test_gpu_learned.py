"""The learned 2x-coarse path on small grids: the geometry and the source on the
two grids, pairs from the plain fine solver, training with the library's
kernels, and the ablation against the plain coarse solve on a velocity model
that was not trained on."""
from __future__ import annotations

import numpy as np
import pytest

import stencil_solver_b200 as sb
from stencil_solver_b200 import learned

pytestmark = pytest.mark.gpu

NC, H = 64, 10.0
DT = 0.4 * H / 4700.0  # Courant 0.4 at the models' top speed


@pytest.fixture(autouse=True)
def _clean(torch_cuda):
    yield
    torch_cuda.cuda.synchronize()
    assert sb.device_error() == 0


def test_geometry_and_source_agree_between_grids(torch_cuda):
    pb = learned.Problem(NC, H, DT, seed=1)
    fg = pb.fine
    assert fg.nx == 2 * NC - 8 and fg.dx == H / 2 and fg.dt == DT / 2
    # the far wall: coarse halo cell nc - 4 sits on the fine halo cell nf - 4
    assert 2 * (NC - 4) - 4 == fg.nx - 4
    wf, wc = pb.wavelet(True, 21), pb.wavelet(False, 10)
    # coarse sample m averages fine samples 2m - 1, 2m, 2m + 1 with weights 1, 2, 1
    avg = (wf[1:18:2].astype(np.float64) + 2 * wf[2:19:2] + wf[3:20:2]) / 4  # m = 1..9
    assert np.allclose(wc[1:10], avg, rtol=1e-5, atol=1e-7)
    # the two source patterns sample the same function: equal on shared cells
    (of, df, pf, af), (oc, dc, pc, ac) = pb.source(True), pb.source(False)
    assert af == ac
    pf, pc = pf.cpu().numpy(), pc.cpu().numpy()
    rc, rf = (dc[0] - 1) // 2, (df[0] - 1) // 2
    hits = 0
    for k in range(dc[0]):
        j = 2 * (oc[0] + k) - 4 - of[0]
        if 0 <= j < df[0]:
            assert np.isclose(pc[rc, rc, k], pf[rf, rf, j], rtol=1e-6)
            hits += 1
    assert hits >= dc[0] - 1


def test_learned_correction_beats_plain_coarse(torch_cuda):
    nc, c = 80, 40
    mk = lambda s, **kw: learned.Problem(nc, H, DT, seed=s, smooth_cells=1.5, **kw)  # noqa: E731
    train_pbs = [mk(s, src_c=(c - 4 + s % 8, c - 2 + s % 5, c - 3 + s % 7)) for s in range(1, 11)]
    ds = learned.make_pairs(train_pbs, fine_steps=320, samples_per_pair=4096, every=4)
    assert ds.n > 500_000
    with sb.Mlp(seed=3) as mlp:
        hist = learned.train(ds, mlp, epochs=10, batch=8192, lr=2e-3)
        assert hist[-1] < 0.2 * hist[0]
        errs = {k: learned.evaluate(mk(99), k, mlp) for k in (40, 120)}
    print("ablation", errs, "loss", hist[0], hist[-1])
    for k, e in errs.items():
        assert e["learned"] < 0.8 * e["plain"], (k, e)
