"""GraphFlood on a ragged batch of tiles in one persistent launch.

``RaggedFlooder`` runs, on every tile of a ``RaggedRouter``, the iterations of
``Flooder.run_graphflood`` (pyfastflow/graphflood/gf_fields.py:111-141): each
tile's CTA loops receivers -> carve reroute -> fill with delta -> 5 diffusion
sweeps -> Manning update until the tile's stop or the iteration cap, with no
host round trip.  h, Q and the router's z are updated in place, bit-identical
to a Flooder run on each tile alone.  Each tile has its own rainfall and
Manning coefficient.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _dev, _lib
from .. import constants as cte

STOP = {"max": 0, "mean": 1, None: -1}


class RaggedFlooder:
    def __init__(self, router, precipitation_rates=10e-3 / 3600, manning=0.033, edge_slope=1e-2):
        self.router = router
        n = router.ntiles
        self.P = np.broadcast_to(np.asarray(precipitation_rates, np.float64), (n,)).copy()
        self.n = np.broadcast_to(np.asarray(manning, np.float64), (n,)).copy()
        self.edge_slope = float(edge_slope)
        self.h = torch.zeros(router.total, dtype=torch.float32, device=router.device)
        self.iters = torch.zeros(n, dtype=torch.int32, device=router.device)
        self.residuals = torch.zeros(2 * n, dtype=torch.float32, device=router.device)

    def _consts(self, tol_ratio):
        f = np.float32
        c = np.empty((self.router.ntiles, 4), np.float32)
        for t in range(self.router.ntiles):
            dx = self.router.dx[t]
            # the same f32 constants as Flooder._consts; the stop threshold is on |dh| per iteration
            c[t] = (f(dx ** 2), f(self.P[t] * dx * dx), f(self.n[t]), f(tol_ratio * self.P[t] * cte.DT_HYDRO))
        return torch.from_numpy(c.ravel()).to(self.router.device)

    def run(self, niter, stop="max", tol_ratio=1e-4, trace=False, threads=1024, ctas_per_sm=1):
        """Up to `niter` iterations per tile; stop "max" ends a tile when
        max|dh|/dt < tol_ratio * P (the reference's residual), "mean" when
        mean|dh|/dt < tol_ratio * P, None never.  Returns (iterations per tile,
        last (max|dh|, mean|dh|) per tile[, trace niter x 2 per tile])."""
        r = self.router
        cst = self._consts(tol_ratio)
        tr = torch.zeros(r.ntiles * max(niter, 1) * 2, dtype=torch.float32, device=r.device) if trace else None
        _lib.call("pff_batch_graphflood", r.z.data_ptr(), r.codes.data_ptr() if r.codes is not None else None,
                  self.h.data_ptr(), r.Q.data_ptr(), cst.data_ptr(),
                  float(np.float32(self.edge_slope)), float(np.float32(cte.DT_HYDRO)), int(niter), STOP[stop],
                  self.iters.data_ptr(), self.residuals.data_ptr(), tr.data_ptr() if trace else None, r.total,
                  r.ntiles, threads, ctas_per_sm, r.ws.data_ptr(), r.ws_bytes, _dev.stream())
        r.check_status()
        it = self.iters.cpu().numpy()
        res = self.residuals.cpu().numpy().reshape(-1, 2)
        if trace:
            return it, res, tr.cpu().numpy().reshape(r.ntiles, max(niter, 1), 2)
        return it, res

    def get_h(self, t):
        r = self.router
        o = int(r.offset[t])
        return self.h[o:o + r.cells(t)].cpu().numpy().reshape(r.ny[t], r.nx[t])

    def set_h(self, arrays):
        self.h.copy_(torch.from_numpy(self.router.packed(arrays)))
