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


NC80, C80 = 80, 40


def mk80(s, **kw):
    return learned.Problem(NC80, H, DT, seed=s, smooth_cells=1.5, **kw)


@pytest.fixture(scope="module")
def trained(torch_cuda):
    """A network trained on 10 smoothed layered models (80^3 coarse / 152^3 fine)."""
    pbs = [mk80(s, src_c=(C80 - 4 + s % 8, C80 - 2 + s % 5, C80 - 3 + s % 7)) for s in range(1, 11)]
    ds = learned.make_pairs(pbs, fine_steps=320, samples_per_pair=4096, every=4)
    assert ds.n > 500_000
    mlp = sb.Mlp(seed=3)
    hist = learned.train(ds, mlp, epochs=10, batch=8192, lr=2e-3)
    del ds
    yield mlp, hist
    mlp.close()


def test_learned_correction_beats_plain_coarse(trained):
    mlp, hist = trained
    assert hist[-1] < 0.2 * hist[0]
    errs = {k: learned.evaluate(mk80(99), k, mlp) for k in (40, 120)}
    print("ablation", errs, "loss", hist[0], hist[-1])
    for k, e in errs.items():
        assert e["learned"] < 0.8 * e["plain"], (k, e)


def test_judged_solve_without_fallback_is_the_corrected_solve(trained):
    mlp, _ = trained
    pb = mk80(77)
    rep = learned.learned_solve(pb, 60, mlp, bound=1.0, check_every=20)
    assert rep.fallback_at is None and [c[0] for c in rep.checks] == [20, 40, 60]
    _, vc = pb.device_models()
    ref = learned.coarse_solve(pb, vc, 60, mlp)
    assert bool((rep.field == ref).all())


def test_judged_solve_falls_back_to_the_fine_solve(trained):
    mlp, _ = trained
    pb = mk80(78)
    rep = learned.learned_solve(pb, 40, mlp, bound=1e-12, check_every=10)
    assert rep.fallback_at == 10 and len(rep.checks) == 1 and rep.checks[0][1] > 1e-12
    _, ref = learned.time_fine_solve(pb, 80)
    assert bool((rep.field == ref).all())
