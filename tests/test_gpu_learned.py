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
    wf, wc = pb.wavelet(True, 20), pb.wavelet(False, 10)
    assert np.allclose(wc, wf[::2], rtol=1e-6, atol=1e-7)
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
