"""The learned warm start on the 16-parameter grid-with-diodes deck (B200).

The network is trained on the GPU on plain-solver operating points; on
held-out points its guesses cut the mean Newton iterations against the
nominal warm start, every point converges (a lane that does not within k
iterations is solved again from the nominal start), and each lane solved
from its learned guess matches the oracle started from the same guess:
the same iteration count and x within 1e-9 relative or 1e-12 absolute.
"""

import numpy as np
import pytest

from espice_b200 import decks, lanes, learned
from oracle import oracle

pytestmark = pytest.mark.gpu


def test_learned_warm_start_cuts_newton_iterations():
    import torch
    assert torch.cuda.is_available()
    fr, slots, values, nominal = decks.grid_diodes_16(points=16384 + 1024)
    train, test = values[:16384], values[16384:]
    ctx = lanes.DcLanes(fr)
    ctx.set_lanes(slots, nominal[None, :])
    x_nom, _, st, _ = ctx.solve(x0=None)
    assert st[0] == lanes.LANE_CONVERGED
    x_nom = x_nom[0]
    ctx.set_lanes(slots, train)
    x_tr, _, st_tr, _ = ctx.solve(x0=x_nom)
    ok = st_tr == lanes.LANE_CONVERGED
    ws = learned.LearnedWarmStart(len(slots), fr.n, hidden=256, layers=3)
    loss = ws.fit(train[ok], x_tr[ok], epochs=60, batch=256, lr=2e-3)
    assert loss[-1] < 0.01 * loss[0]

    ctx.set_lanes(slots, test)
    _, it_plain, st_plain, _ = ctx.solve(x0=x_nom)
    fb = lanes.DcLanes(fr)
    d_x, it_learned, conv, n_fb = learned.solve(ctx, fb, ws, slots, test, x_nom, k=8)
    assert conv.all()
    assert (st_plain == lanes.LANE_CONVERGED).all()
    assert it_learned.mean() < 0.95 * it_plain.mean(), (it_learned.mean(), it_plain.mean())

    # lanes that converged from their guess, against the oracle from the same guess
    guess = ws.predict(torch.tensor(test, dtype=torch.float32, device="cuda"), len(test)).cpu().numpy()
    x = d_x.cpu().numpy()
    first = np.flatnonzero(it_learned <= 8)[:48]
    for i in first:
        xo, ito, cvo = oracle.dc_points(fr, slots, test[i:i + 1], warm=guess[i])
        assert cvo[0] and ito[0] == it_learned[i]
        close = np.abs(x[i] - xo[0]) <= 1e-12 + 1e-9 * np.maximum(np.abs(x[i]), np.abs(xo[0]))
        assert close.all()
    ws.close()
    fb.close()
    ctx.close()
