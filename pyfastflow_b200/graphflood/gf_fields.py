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

    def __del__(self):
        # the guarded graphs live in the library's registry until destroyed
        for gid in getattr(self, "_guards", {}).values():
            try:
                _lib.load().pff_guard_destroy(gid)
            except Exception:
                pass

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
        # the fill left the filled surface in both z and z_: the Manning update reads
        # its slopes from z_ and updates z in the same pass
        _lib.call("pff_graphflood_core_filled", self.h.data_ptr(), r.z.data_ptr(), r.z_.data_ptr(),
                  self.dh.data_ptr(), r.receivers.data_ptr(), r.Q.data_ptr(), r.N, c["dx"], c["dx2"], c["manning"],
                  c["edgesw"], c["dt"], self._h0.data_ptr() if track_dh else None,
                  self._dhmax.data_ptr() if track_dh else None, st)

    def iteration(self, track_dh: bool = False):
        """One GraphFlood iteration (gf_fields.py:126-141): receivers, carve
        reroute, fill with delta (epsilon 1e-3), 5 diffusion sweeps, Manning update.
        The part after the reroute (about 30 launches on fixed buffers) is replayed
        from a CUDA graph captured on first use for these constants."""
        self._route()
        self._update(track_dh)

    def _route(self):
        """Receivers and carve reroute on the current surface (gf_fields.py:128-131);
        the reroute synchronises the host once.  h, z and Q are not changed."""
        self.router.compute_receivers()
        self.router.reroute_flow()

    def _update(self, track_dh: bool):
        """Fill, diffusion and Manning update (gf_fields.py:134-141), replayed from a
        CUDA graph per set of constants (asynchronous)."""
        r = self.router
        # graphs keyed by the raw parameters: no f32 conversions on the per-iteration path
        key = (track_dh, self.dx, self.precipitation_rates, self.manning, self.edge_slope, cte.DT_HYDRO)
        g = self._graphs.get(key) if self.graphs else None
        if g is not None:
            g.replay()
            return
        c = self._consts()
        if not self.graphs:
            self._after_reroute(c, track_dh)
            return
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
        if self._pipeline(N) is None:
            for _ in range(N):
                self.iteration()

    def run_to_residual(self, tol_ratio=1e-4, max_iter=20000, return_trace=False, stop="max"):
        """Iterate until the residual < tol_ratio * precipitation rate, or max_iter
        iterations.  stop="max": the residual is max|dh|/dt, the reference's
        criterion; stop="mean": mean|dh|/dt over the cells.  dh is the change of h
        over one whole iteration.  Returns (iterations, stop_reason, residual) with
        stop_reason "residual" or "max_iter" (and the per-iteration residuals if
        return_trace).  On return h, z and Q are those of the last counted
        iteration; the router's receiver and lake fields route that final surface
        (the loop runs the next iteration's receivers and reroute before it reads a
        residual)."""
        if stop not in ("max", "mean"):
            raise ValueError(f"stop must be 'max' or 'mean', got {stop!r}")
        thr = tol_ratio * self.precipitation_rates
        trace = torch.zeros(max_iter, dtype=torch.float32, device=self.h.device)
        out = self._pipeline(max_iter, stop=stop, thr=thr, trace=trace)
        if out is None:
            out = self._residual_loop(max_iter, stop, thr, trace)
        n = out[0]
        if return_trace:
            return out + ((trace[:n] / cte.DT_HYDRO).cpu().numpy(),)
        return out

    # ---- the pipelined loop --------------------------------------------------------------
    def _post(self, c, stop, thr):
        """The part of an iteration after the reroute, and (stop given) its residual
        into self._res, and (thr given) the converged flag."""
        N = self.router.N
        if stop == "mean":
            self._h0.copy_(self.h)
        self._after_reroute(c, stop == "max")
        if stop == "mean":
            self._stats.zero_()
            _lib.call("pff_abs_diff_stats", self.h.data_ptr(), self._h0.data_ptr(), N, self._stats.data_ptr(),
                      _dev.stream())
            torch.div(self._stats[1:2], N, out=self._res)
        if thr is not None:
            _lib.call("pff_residual_flag", self._src(stop).data_ptr(), float(cte.DT_HYDRO), float(thr),
                      self._flag.data_ptr(), _dev.stream())

    def _src(self, stop):
        """The device scalar holding an iteration's residual (times dt)."""
        return self._dhmax if stop == "max" else self._res

    def _pipeline(self, n_iter, stop=None, thr=None, trace=None):
        """n_iter iterations (stop: also each residual into trace; thr: stop after the
        first iteration whose residual is below thr), with the host never idling the
        GPU: iteration k's post-reroute part is queued behind its reroute, as a graph
        that runs only if the reroute finished on the device (and, with thr, only if
        iteration k-1 did not converge), before the host waits for the reroute.  A
        reroute that stopped for the host's steps is finished on the host and its
        post-reroute part run then.  Returns (iterations, reason, residual), or None
        where the device-driven reroute or graphs are not available (the caller then
        runs the iterations one by one)."""
        r = self.router
        if not self.graphs or not torch.cuda.is_available() or self.h.device.type != "cuda":
            return None
        dev = self.h.device
        if not hasattr(self, "_side"):
            self._side = torch.cuda.Stream(device=dev)
            # the reroute's final state and each residual are written by kernels straight
            # into pinned host memory (unified addresses): no copy engine in the loop
            self._ctl = torch.zeros(9, dtype=torch.int32, pin_memory=True)
            self._flag = torch.zeros(1, dtype=torch.int32, device=dev)
            self._res = torch.zeros(1, dtype=torch.float32, device=dev)
            self._stats = torch.zeros(2, dtype=torch.float32, device=dev)
            self._res_host = torch.zeros(2, dtype=torch.float32, pin_memory=True)
            self._ev_route = [torch.cuda.Event(), torch.cuda.Event()]
            self._ev_post = [torch.cuda.Event(), torch.cuda.Event()]
            self._guards = {}
        caller = torch.cuda.current_stream(dev)
        self._side.wait_stream(caller)
        try:
            with torch.cuda.stream(self._side):
                return self._pipeline_on_side(n_iter, stop, thr, trace)
        finally:
            caller.wait_stream(self._side)

    def _guard_launch(self, stop, thr):
        import ctypes as C

        r = self.router
        key = (stop, thr, self.dx, self.precipitation_rates, self.manning, self.edge_slope, cte.DT_HYDRO)
        gid = self._guards.get(key)
        st = _dev.stream()
        if gid is None:
            c = self._consts()
            r._ws_fill.get(_lib.load().pff_fill_workspace_bytes(r.N), r.device)
            r._ws_diff.get(_lib.load().pff_diffuse_workspace_bytes(r.N), r.device)
            h = C.c_int()
            _lib.call("pff_guard_begin", self._ctl.data_ptr(), self._flag.data_ptr() if thr is not None else None,
                      st, C.byref(h))
            try:
                self._post(c, stop, thr)
            except BaseException:
                _lib.load().pff_guard_destroy(h.value)
                raise
            _lib.call("pff_guard_end", h.value, st)
            gid = self._guards[key] = h.value
        _lib.call("pff_guard_launch", gid, st)

    def _pipeline_on_side(self, n_iter, stop, thr, trace):
        r = self.router
        self._flag.zero_()
        res, n = float("inf"), 0
        for k in range(1, n_iter + 2):
            slot = k & 1
            if k <= n_iter:
                r.compute_receivers()
                if not r.reroute_flow_async(self._ctl):
                    if k == 1:
                        return None  # no device-driven reroute here: the plain loop
                    raise RuntimeError("the device-driven reroute became unavailable during a run")
                self._ev_route[slot].record()
                self._guard_launch(stop, thr)
                if stop is not None:
                    self._store_residual(trace, k, slot, stop)
                self._ev_post[slot].record()
            if k > 1 and stop is not None:  # the residual of iteration k - 1
                (self._ev_route[slot] if k <= n_iter else self._ev_post[slot ^ 1]).synchronize()
                res = float(self._res_host[slot ^ 1]) / cte.DT_HYDRO
                n = k - 1
                if thr is not None and res < thr:
                    # iteration k's post-reroute part was skipped on the device; its
                    # reroute is completed, so the router's fields route the final surface
                    if k <= n_iter:
                        r.reroute_flow_finish(self._ctl)
                    break
            if k > n_iter:
                break
            self._ev_route[slot].synchronize()
            state = r.reroute_flow_finish(self._ctl)
            if state not in (1, 2):  # finished on the host: the guarded part did not run
                self._post(self._consts(), stop, thr)
                if stop is not None:
                    self._store_residual(trace, k, slot, stop)
                self._ev_post[slot].record()
            n = k
        if stop is None:
            return (n, "iterations", float("nan"))
        reason = "residual" if thr is not None and res < thr else "max_iter"
        return (n, reason, res)

    def _store_residual(self, trace, k, slot, stop):
        """Iteration k's residual into trace[k - 1] and the pinned slot (one kernel)."""
        _lib.call("pff_value_store", self._src(stop).data_ptr(), trace[k - 1:k].data_ptr(),
                  self._res_host[slot:slot + 1].data_ptr(), _dev.stream())

    def _residual_loop(self, max_iter, stop, thr, trace):
        """run_to_residual one iteration at a time (no device-driven reroute here)."""
        dev = self.h.device
        stats = torch.zeros(2, dtype=torch.float32, device=dev)
        host = torch.zeros(1, dtype=torch.float32, pin_memory=dev.type == "cuda")
        done = torch.cuda.Event() if dev.type == "cuda" else None
        N = self.router.N
        res = float("inf")
        n = 0
        for it in range(1, max_iter + 2):
            if it <= max_iter:
                self._route()
            if it > 1:  # the residual of iteration it - 1
                if done is not None:
                    done.synchronize()
                res = float(host[0]) / cte.DT_HYDRO
                n = it - 1
                if res < thr or it > max_iter:
                    break
            if stop == "max":
                self._update(track_dh=True)
                src = self._dhmax
            else:
                self._h0.copy_(self.h)
                self._update(track_dh=False)
                stats.zero_()
                _lib.call("pff_abs_diff_stats", self.h.data_ptr(), self._h0.data_ptr(), N, stats.data_ptr(),
                          _dev.stream())
                src = stats[1:2] / N
            trace[it - 1:it].copy_(src)
            host.copy_(src, non_blocking=True)
            if done is not None:
                done.record()
        return (n, "residual" if res < thr else "max_iter", res)

    def set_h(self, val):
        if isinstance(val, torch.Tensor):
            self.h.copy_(val.reshape(-1).to(torch.float32))
        else:
            self.h.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(val, np.float32).ravel())))

    def get_h(self):
        return self.h.cpu().numpy().reshape(self.rshp)
