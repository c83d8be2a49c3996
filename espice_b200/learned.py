"""Learned warm start for independent DC sweep points.

A tanh MLP (include/espice_mlp.h) maps a lane's swept parameter values to its
unknowns. It is trained on the GPU, by the library's tensor-core kernels, on
operating points the plain FP64 lane solver produced; its prediction seeds
each lane's Newton solve. The plain solver judges every result with its own
gates, so a poor guess costs iterations, never accuracy: a lane that has not
converged within `k` iterations from the learned guess is solved again from
the nominal warm start (the reference's start for independent points,
src/analysis/sweep/lanes.zig:73-80).
"""

from __future__ import annotations

import numpy as np

from . import lanes, mlp


class LearnedWarmStart:
    def __init__(self, n_params, n_unknowns, hidden=256, layers=3, device=0, seed=1):
        self.net = mlp.Mlp(n_params, hidden, layers, n_unknowns, device=device, seed=seed)
        self.n_params, self.n = n_params, n_unknowns
        self._bufs = {}

    def buffers(self, n_points):
        """Device work buffers for a batch of n_points, kept across calls: the
        FP32 guesses, the FP64 unknowns, and the solver's status and
        iteration words (one [2][N] int32 tensor, read back in one copy)."""
        import torch
        b = self._bufs.get(n_points)
        if b is None:
            b = (torch.empty((n_points, self.n), dtype=torch.float32, device="cuda"),
                 torch.empty((n_points, self.n), dtype=torch.float64, device="cuda"),
                 torch.zeros((2, n_points), dtype=torch.int32, device="cuda"))
            self._bufs[n_points] = b
        return b

    def close(self):
        self.net.close()

    def fit(self, values, x, epochs=40, batch=256, lr=2e-3, lr_end=2e-5, seed=1):
        """Trains on (values [N][n_params], x [N][n]); returns the loss per epoch."""
        import torch
        values = np.asarray(values, np.float64)
        x = np.asarray(x, np.float64)
        sig_in = values.std(0)
        sig_out = x.std(0)
        self.net.set_scaling(values.mean(0), np.where(sig_in > 0, sig_in, 1.0), x.mean(0),
                             np.where(sig_out > 1e-12, sig_out, 1.0))
        dx = torch.tensor(values, dtype=torch.float32, device="cuda")
        dy = torch.tensor(x, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        n = (len(values) // batch) * batch
        return self.net.train(dx.data_ptr(), dy.data_ptr(), n, epochs=epochs, batch=batch, lr=lr, lr_end=lr_end,
                              seed=seed)

    def predict(self, d_values, n_points):
        """The guesses for device values [n_points][n_params] (float32), as a
        float64 device tensor [n_points][n]."""
        import torch
        out = torch.empty((n_points, self.n), dtype=torch.float32, device="cuda")
        self.net.predict(d_values.data_ptr(), n_points, out.data_ptr())
        return out.double()


def solve(ctx, fallback, ws, slots, values, x_nominal, k=8, opts=None, d_values=None, stats_out=None, cols=None):
    """Solves every lane of `ctx` (lanes already set to `values`) from the
    learned guess with at most `k` Newton iterations, then the lanes that did
    not converge again from `x_nominal` on `fallback` (a DcLanes of the same
    circuit). `d_values`: the values already on the device as float32 (as the
    lanes' records are), else they are uploaded. Returns (x [N][n] device
    tensor, iterations [N] (both passes), converged mask [N] host, number of
    fallback lanes). The returned x is the learned start's work buffer for
    this batch size: valid until its next solve of the same size. With
    stats_out a list, the solves' statistics (esl_stats dicts) are appended
    to it. With cols, `values` are the lanes' live parameter values
    (DcLanes.set_lanes with cols) and the fallback lanes take them the same
    way."""
    import torch
    opts = opts or lanes.newton_opts()
    N = values.shape[0]
    d_vals = d_values if d_values is not None else torch.tensor(values, dtype=torch.float32, device="cuda")
    guess, d_x, words = ws.buffers(N)
    ws.net.predict(d_vals.data_ptr(), N, guess.data_ptr())  # returns with its stream drained
    d_x.copy_(guess)
    capped = lanes.newton_opts(opts.reltol, opts.abstol, opts.vntol, opts.residual_tol, opts.gmin,
                               opts.max_iter, bool(opts.init_fix), iter_cap=k)
    torch.cuda.current_stream().synchronize()
    s = ctx.solve_device(d_x.data_ptr(), words[1].data_ptr(), words[0].data_ptr(), cold=False, opts=capped)
    if stats_out is not None:
        stats_out.append(s)
    host = words.cpu().numpy()
    st = host[0]
    it = host[1].astype(np.int64)
    failed = np.flatnonzero(st != lanes.LANE_CONVERGED)
    if len(failed):
        fallback.set_lanes(slots, values[failed], cols=cols)
        xf, itf, stf, sf = fallback.solve(x0=np.broadcast_to(x_nominal, (len(failed), len(x_nominal))), opts=opts)
        if stats_out is not None:
            stats_out.append(sf)
        d_x[torch.as_tensor(failed, device="cuda")] = torch.tensor(xf, device="cuda")
        it[failed] += itf
        st[failed] = stf
    return d_x, it, st == lanes.LANE_CONVERGED, len(failed)
