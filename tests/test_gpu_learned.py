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
    (of, df, pf, af), (oc, dc, pc, ac) = pb.source(True)[:4], pb.source(False)[:4]
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


def test_source_composition_pattern(torch_cuda):
    """The coarse source's composition pattern is v^2 lap(v^2 g): on a constant
    model, v^4 g (r^2 / sigma^4 - 3 / sigma^2) / h^2 to the 8th-order stencil's
    accuracy; the fine grid has none."""
    pb = learned.Problem(NC, H, DT, seed=3, model="constant")
    assert pb.source(True).comp_pattern is None
    s = pb.source(False)
    v2 = float(pb.device_models()[1][NC // 2, NC // 2, NC // 2])
    comp = s.comp_pattern.cpu().numpy().astype(np.float64)
    n = s.comp_dims[0]
    assert s.comp_dims == (n, n, n) and n == s.dims[0] + 8
    assert tuple(o + n // 2 for o in s.comp_origin) == tuple(pb.src_c)
    off = np.arange(n) - n // 2
    r2 = off[None, None, :] ** 2 + off[None, :, None] ** 2 + off[:, None, None] ** 2
    sig = pb.sigma_cells
    ref = v2 * v2 * np.exp(-r2 / (2 * sig * sig)) * (r2 / sig ** 4 - 3 / sig ** 2) / (H * H)
    assert np.max(np.abs(comp - ref)) <= 2e-3 * np.max(np.abs(ref))
    off_pb = learned.Problem(NC, H, DT, seed=3, model="constant", compose_source=False)
    assert off_pb.source(False).comp_pattern is None


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
    # rows inside the source region (the default) are the hardest: the last
    # epoch's loss ends near 0.22 of the first one's (0.15 without them)
    assert hist[-1] < 0.3 * hist[0]
    errs = {k: learned.evaluate(mk80(99), k, mlp) for k in (40, 120)}
    print("ablation", errs, "loss", hist[0], hist[-1])
    for k, e in errs.items():
        assert e["learned"] < 0.8 * e["plain"], (k, e)


def test_source_composition_lowers_the_early_corrected_error(trained):
    """Two fine steps compose to a coarse step plus h^4 L^2 p + h^4 L S: the
    network (trained with the composition term in the coarse source) supplies
    the state's part, the source term the rest.  While the source is on, the
    corrected solve is closer to the fine one with the term than without."""
    mlp, _ = trained
    errs = {comp: learned.evaluate(mk80(98, compose_source=comp), 30, mlp)["learned"]
            for comp in (False, True)}
    print("composition", errs)
    assert errs[True] < 0.8 * errs[False], errs


def test_judged_solve_without_fallback_is_the_corrected_solve(trained):
    mlp, _ = trained
    pb = mk80(77)
    rep = learned.learned_solve(pb, 60, mlp, bound=1.0, check_every=20, rival=False)
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


def test_composition_prepass_beats_the_plain_coarse_step(torch_cuda):
    """The coarse step with the two-step composition term (sb200_wave_prepass_f32:
    h^4 L^2 p, h = dt / 2) against the plain coarse step, both against the
    restricted plain fine solve of an unseen smoothed layered model."""
    errs = {comp: learned.evaluate(mk80(97, compose_state=comp), 120, None)["plain"]
            for comp in (False, True)}
    print("composition pre-pass", errs)
    assert errs[True] < 0.2 * errs[False], errs


def test_judge_switches_off_a_network_that_loses(trained):
    """The judge runs the proxy with and without the network: a network that
    gains stays on; one that loses is switched off at the first check and the
    solve carries on without it.  The network trained on the plain step's
    residual double-counts the L^2 term on a pre-passed step, so it loses there."""
    mlp, _ = trained
    rep = learned.learned_solve(mk80(76), 40, mlp, bound=1.0, check_every=20)
    assert rep.network_off_at is None and rep.checks[0][1] < rep.checks[0][2], rep.checks
    pbc = mk80(76, compose_state=True)
    rep = learned.learned_solve(pbc, 40, mlp, bound=1.0, check_every=20)
    assert rep.network_off_at == 20 and rep.fallback_at is None, rep.checks
    assert rep.checks[0][1] > rep.checks[0][2]
    assert rep.checks[1][2] is None  # no rival once the network is off
