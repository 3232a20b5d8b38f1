"""Flooder, mirroring pyfastflow/graphflood/gf_fields.py:30-159."""
from __future__ import annotations

import numpy as np
import torch

from .. import constants as cte
from .. import _dev, _lib
from ..flow import fill_topo


class Flooder:
    def __init__(self, router, precipitation_rates=10e-3 / 3600, manning=0.033, edge_slope=1e-2, graphs=True):
        self.nx, self.ny, self.dx, self.rshp = router.nx, router.ny, router.dx, router.rshp
        self.router = router
        N = router.N
        self.h = torch.zeros(N, dtype=torch.float32, device=router.device)
        self.dh = torch.zeros(N, dtype=torch.float32, device=router.device)
        self._h0 = torch.zeros(N, dtype=torch.float32, device=router.device)
        self._dhmax = torch.zeros(1, dtype=torch.float32, device=router.device)
        self.precipitation_rates = precipitation_rates
        self.manning = manning
        self.edge_slope = edge_slope
        self.graphs = bool(graphs)  # replay the post-reroute part of an iteration from a CUDA graph
        self._graphs = {}
        cte.PREC = precipitation_rates  # gf_fields.py:106-108
        cte.MANNING = manning
        cte.EDGESW = edge_slope

    def _consts(self):
        f = lambda x: float(np.float32(x))  # noqa: E731  (Python folds in double, the kernel sees f32)
        return dict(dx=f(self.dx), dx2=f(self.dx ** 2), prec_dx2=f(self.precipitation_rates * self.dx * self.dx),
                    manning=f(self.manning), edgesw=f(self.edge_slope), dt=f(cte.DT_HYDRO))

    def _after_reroute(self, c, track_dh: bool):
        """Fill with delta (epsilon 1e-3), 5 diffusion sweeps, Manning update."""
        r = self.router
        st = _dev.stream()
        if track_dh:
            self._h0.copy_(self.h)
            self._dhmax.zero_()
        fill_topo.fill_z_add_delta(r.z, self.h, r.z_, r.receivers, r.receivers_, r.receivers__, epsilon=1e-3,
                                   workspace=r._ws_fill)
        wp, wn = r._ws_diff.get(_lib.load().pff_diffuse_workspace_bytes(r.N), r.device)
        _lib.call("pff_diffuse_q", r.z.data_ptr(), r.Q.data_ptr(), r.Q_.data_ptr(), 5, r.nx, r.ny, c["dx"],
                  c["prec_dx2"], r.mode, r._codes(), wp, wn, st)
        _lib.call("pff_graphflood_core", self.h.data_ptr(), r.z.data_ptr(), self.dh.data_ptr(),
                  r.receivers.data_ptr(), r.Q.data_ptr(), r.N, c["dx"], c["dx2"], c["manning"], c["edgesw"],
                  c["dt"], self._h0.data_ptr() if track_dh else None, self._dhmax.data_ptr() if track_dh else None,
                  st)

    def iteration(self, track_dh: bool = False):
        """One GraphFlood iteration (gf_fields.py:126-141): receivers, carve
        reroute, fill with delta (epsilon 1e-3), 5 diffusion sweeps, Manning update.
        The part after the reroute (about 30 launches on fixed buffers) is replayed
        from a CUDA graph captured on first use for these constants."""
        r = self.router
        c = self._consts()
        r.compute_receivers()
        r.reroute_flow()
        if not self.graphs:
            self._after_reroute(c, track_dh)
            return
        key = (track_dh,) + tuple(sorted(c.items()))
        g = self._graphs.get(key)
        if g is None:
            # workspaces exist before the capture, so the graph only reads and writes them
            r._ws_fill.get(_lib.load().pff_fill_workspace_bytes(r.N), r.device)
            r._ws_diff.get(_lib.load().pff_diffuse_workspace_bytes(r.N), r.device)
            g = torch.cuda.CUDAGraph()
            torch.cuda.current_stream().synchronize()
            try:
                with torch.cuda.graph(g):
                    self._after_reroute(c, track_dh)
            except Exception:  # capture not possible here: stay eager
                self.graphs = False
                torch.cuda.synchronize()
                self._after_reroute(c, track_dh)
                return
            self._graphs[key] = g
        g.replay()

    def run_graphflood(self, N=10):
        """N iterations (gf_fields.py:111-141)."""
        for _ in range(N):
            self.iteration()

    def run_to_residual(self, tol_ratio=1e-4, max_iter=20000, return_trace=False, stop="max"):
        """Iterate until the residual < tol_ratio * precipitation rate, or max_iter
        iterations.  stop="max": the residual is max|dh|/dt, the reference's
        criterion; stop="mean": mean|dh|/dt over the cells.  dh is the change of h
        over one whole iteration.  Returns (iterations, stop_reason, residual) with
        stop_reason "residual" or "max_iter" (and the per-iteration residuals if
        return_trace)."""
        if stop not in ("max", "mean"):
            raise ValueError(f"stop must be 'max' or 'mean', got {stop!r}")
        thr = tol_ratio * self.precipitation_rates
        trace = torch.zeros(max_iter, dtype=torch.float32, device=self.h.device)
        stats = torch.zeros(2, dtype=torch.float32, device=self.h.device)
        res = float("inf")
        N = self.router.N
        for it in range(1, max_iter + 1):
            if stop == "max":
                self.iteration(track_dh=True)
                src = self._dhmax
            else:
                self._h0.copy_(self.h)
                self.iteration()
                stats.zero_()
                _lib.call("pff_abs_diff_stats", self.h.data_ptr(), self._h0.data_ptr(), N, stats.data_ptr(),
                          _dev.stream())
                src = stats[1:2] / N
            trace[it - 1:it].copy_(src)  # on the device: no extra synchronisation
            # the reroute synchronises the host every iteration anyway: read the residual
            res = float(src.item()) / cte.DT_HYDRO
            if res < thr:
                break
        n = it
        out = (n, "residual" if res < thr else "max_iter", res)
        if return_trace:
            return out + ((trace[:n] / cte.DT_HYDRO).cpu().numpy(),)
        return out

    def set_h(self, val):
        if isinstance(val, torch.Tensor):
            self.h.copy_(val.reshape(-1).to(torch.float32))
        else:
            self.h.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(val, np.float32).ravel())))

    def get_h(self):
        return self.h.cpu().numpy().reshape(self.rshp)
