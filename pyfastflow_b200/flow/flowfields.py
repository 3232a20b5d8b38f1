"""FlowRouter, mirroring pyfastflow/flow/flowfields.py:26-319.

Holds the same fields as the reference (as torch CUDA tensors, same attribute
names) and drives the same pipeline: compute_receivers -> reroute_flow ->
accumulate_constant_Q.  The grid is a runtime argument of every kernel, so
several routers of different shapes can coexist (the reference allows one grid
per process).
"""
from __future__ import annotations

import numpy as np
import torch

from .. import constants as cte
from .. import _dev, _lib
from . import environment as env
from .f32_i32_struct import INVALID_KEY


class FlowRouter:
    def __init__(self, nx, ny, dx, boundary_mode="normal", boundaries=None, lakeflow=True,
                 stochastic_receivers=False, device="cuda"):
        if boundary_mode not in cte.BOUND_MODES:
            boundary_mode = "normal"  # the reference falls back to mode 0 (flowfields.py:169-175)
        self.nx, self.ny, self.dx = int(nx), int(ny), float(dx)
        self.rshp = (self.ny, self.nx)
        self.boundary_mode = boundary_mode
        self.mode = cte.BOUND_MODES[boundary_mode]
        self.lakeflow = lakeflow
        self.stochastic_receivers = bool(stochastic_receivers)
        self.device = _dev.resolve_device(device)
        N = self.nx * self.ny
        self.N = N
        f32, i32 = dict(dtype=torch.float32, device=self.device), dict(dtype=torch.int32, device=self.device)
        # core fields (flowfields.py:71-115)
        self.z = torch.zeros(N, **f32)
        self.Q = torch.zeros(N, **f32)
        self.Q_ = torch.zeros(N, **f32)
        self.gradient = torch.zeros(N, **f32)
        self.receivers = torch.zeros(N, **i32)
        self.src = torch.zeros(N, **i32)
        self.ndonors = torch.zeros(N, **i32)
        self.ndonors_ = torch.zeros(N, **i32)
        self.donors = torch.zeros(4 * N, **i32)
        self.donors_ = torch.zeros(4 * N, **i32)
        # exact drainage counts (new: the reference accumulates f32 only)
        self.counts = torch.zeros(N, dtype=torch.int32, device=self.device)
        self.codes = None
        if self.mode == 3:
            if boundaries is None:
                raise ValueError("custom boundary mode needs a boundaries array")
            self.codes = torch.from_numpy(np.ascontiguousarray(np.asarray(boundaries, np.uint8).ravel())).to(self.device)
            if self.codes.numel() != N:
                raise ValueError("boundaries must have nx*ny entries")
        self.boundaries = boundaries
        # lake fields (flowfields.py:119-159); basin arrays sized N+1
        if lakeflow:
            self.z_ = torch.zeros(N, **f32)
            self.z__ = torch.zeros(N, **f32)
            self.receivers_ = torch.zeros(N, **i32)
            self.receivers__ = torch.zeros(N, **i32)
            self.bid = torch.zeros(N, **i32)
            self.basin_saddlenode = torch.full((N + 1,), -1, **i32)
            self.outlet = torch.full((N + 1,), INVALID_KEY, dtype=torch.int64, device=self.device)
            self.basin_saddle = torch.full((N + 1,), INVALID_KEY, dtype=torch.int64, device=self.device)
            self.is_border = torch.zeros(N, dtype=torch.uint8, device=self.device)
            self.tag = torch.zeros(N, dtype=torch.uint8, device=self.device)
            self.tag_ = torch.zeros(N, dtype=torch.uint8, device=self.device)
            self.change = torch.zeros((), dtype=torch.uint8, device=self.device)
        self._ws_acc = _dev.Scratch()
        self._ws_tree = _dev.Scratch()
        self._ws_lake = _dev.Scratch()
        self._ws_fill = _dev.Scratch()
        self._ws_diff = _dev.Scratch()
        self.last_n_outer = 0
        # global configuration, as the reference writes it (flowfields.py:163-182)
        cte.NX, cte.NY, cte.DX = self.nx, self.ny, self.dx
        cte.RAND_RCV = self.stochastic_receivers  # flowfields.py:166
        cte.BOUND_MODE = self.mode
        if self.mode == 3:
            cte.boundaries = self.codes
        if not cte.INITIALISED:
            env.initialise()

    # ---- helpers --------------------------------------------------------------
    def _codes(self):
        return self.codes.data_ptr() if self.codes is not None else None

    def free(self):
        """Release the device fields (flowfields.py:186-200)."""
        for k in list(vars(self)):
            if isinstance(getattr(self, k), torch.Tensor):
                setattr(self, k, None)

    # ---- host I/O ---------------------------------------------------------------
    def set_z(self, z):
        """Upload elevations (flowfields.py:202-214); accepts numpy or torch."""
        if isinstance(z, torch.Tensor):
            self.z.copy_(z.reshape(-1).to(torch.float32))
        else:
            self.z.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(z).ravel().astype(np.float32))))

    def get_Q(self):
        return self.Q.cpu().numpy().reshape(self.rshp)

    def get_Z(self):
        return self.z.cpu().numpy().reshape(self.rshp)

    def get_receivers(self):
        return self.receivers.cpu().numpy().reshape(self.rshp)

    def get_counts(self):
        """Exact upstream cell counts (uint32) from the last accumulation."""
        return self.counts.cpu().numpy().view(np.uint32).reshape(self.rshp)

    # ---- pipeline -----------------------------------------------------------------
    def compute_receivers(self, seed=None):
        """flowfields.py:216-226 -> receivers.py:15-58; stochastic (receivers.py:46-47)
        if the router was made with stochastic_receivers=True (seed: the draw's seed,
        default a fresh one per call)."""
        if self.stochastic_receivers:
            from .receivers import next_seed

            _lib.call("pff_compute_receivers_stochastic", self.z.data_ptr(), self.receivers.data_ptr(),
                      self.gradient.data_ptr(), self.nx, self.ny, self.dx, self.mode, self._codes(),
                      next_seed() if seed is None else int(seed), _dev.stream())
            return
        _lib.call("pff_compute_receivers", self.z.data_ptr(), self.receivers.data_ptr(), self.gradient.data_ptr(),
                  self.nx, self.ny, self.dx, self.mode, self._codes(), _dev.stream())

    def reroute_flow(self, carve=True):
        """flowfields.py:228-252 -> lakeflow.py:466-538."""
        if not self.lakeflow:
            raise RuntimeError("Flow field not compiled for lakeflow")
        import ctypes as C

        n = self.N
        wp, wn = self._ws_lake.get(_lib.load().pff_reroute_workspace_bytes(n), self.device)
        nout = C.c_int()
        _lib.call("pff_reroute_flow", self.bid.data_ptr(), self.receivers.data_ptr(), self.receivers_.data_ptr(),
                  self.receivers__.data_ptr(), self.z.data_ptr(), self.z_.data_ptr(), self.is_border.data_ptr(),
                  self.outlet.data_ptr(), self.basin_saddle.data_ptr(), self.basin_saddlenode.data_ptr(),
                  self.tag.data_ptr(), self.tag_.data_ptr(), int(bool(carve)), self.nx, self.ny, self.mode,
                  self._codes(), wp, wn, C.byref(nout), _dev.stream())
        self.last_n_outer = nout.value

    def _reroute_args(self):
        n = self.N
        wp, wn = self._ws_lake.get(_lib.load().pff_reroute_workspace_bytes(n), self.device)
        return (self.bid.data_ptr(), self.receivers.data_ptr(), self.receivers_.data_ptr(),
                self.receivers__.data_ptr(), self.z.data_ptr(), self.z_.data_ptr(), self.is_border.data_ptr(),
                self.outlet.data_ptr(), self.basin_saddle.data_ptr(), self.basin_saddlenode.data_ptr(),
                self.tag.data_ptr(), self.tag_.data_ptr(), self.nx, self.ny, self.mode, self._codes(), wp, wn)

    def reroute_flow_async(self, ctl: torch.Tensor) -> bool:
        """Launch the carve reroute's device-driven loop without waiting for it; its
        final state (9 int32) lands in `ctl` (a device tensor).  False where that
        loop is not available (graphs switched off): call reroute_flow instead.
        Complete with reroute_flow_finish once a host copy of `ctl` is readable."""
        if not self.lakeflow:
            raise RuntimeError("Flow field not compiled for lakeflow")
        lib = _lib.load()
        _lib._sync_device()
        rc = lib.pff_reroute_flow_async(*self._reroute_args(), ctl.data_ptr(), _dev.stream())
        if rc == 5:  # PFF_ERR_UNAVAILABLE
            return False
        if rc != 0:
            raise _lib.PFFError(f"pff_reroute_flow_async failed with status {rc}: "
                                f"{lib.pff_last_error_string().decode(errors='replace')}")
        return True

    def reroute_flow_finish(self, ctl_host) -> int:
        """The host's part of an asynchronous reroute, from a host copy of its state
        (pinned int32 tensor of 9): nothing if the loop finished on the device, the
        reference's steps on the host if it stopped for them.  Returns the reroute's
        state word (1 no pits, 2 done on the device, 3-4 finished on the host)."""
        import ctypes as C

        nout = C.c_int()
        _lib.call("pff_reroute_flow_finish", *self._reroute_args(), ctl_host.data_ptr(), C.byref(nout),
                  _dev.stream())
        self.last_n_outer = nout.value
        return int(ctl_host[3])

    def _accumulate(self, counts: bool = True, exact_order: bool = False, value=None):
        """Upstream sums of the seeds (Q, or `value` per cell) into Q and counts.

        Default: the tile-hierarchy accumulation (pff_accumulate_tree) -- exact
        integer sums, Q rounded once to f32, exact counts.  exact_order=True, and
        receivers the tree path reports it cannot take (a receiver cycle), use the
        rake-and-compress rounds with the reference's f32 summation order
        (pff_accumulate_grid), bit-identical to the reference's Q."""
        lib = _lib.load()
        if not exact_order:
            import ctypes as C

            local = 1
            for _ in range(2):
                wp, wn = self._ws_tree.get(lib.pff_accumulate_tree_workspace_bytes(self.nx, self.ny, local),
                                           self.device)
                seeds = None if value is not None else self.Q.data_ptr()
                _lib.call("pff_accumulate_tree", self.receivers.data_ptr(), seeds,
                          float(value) if value is not None else 0.0, self.Q.data_ptr(),
                          self.counts.data_ptr() if counts else None, self.nx, self.ny, local, wp, wn,
                          _dev.stream())
                st = C.c_int()
                _lib.call("pff_accumulate_tree_status", self.nx, self.ny, local, wp, wn, C.byref(st), _dev.stream())
                if st.value == 0:
                    return
                if st.value & 1:
                    raise _lib.PFFError("accumulate: a receiver index is out of range")
                if st.value == 8 and local == 1:
                    local = 0  # receivers that are not D4 neighbours (jump rerouting): general form
                    continue
                break
            # a receiver cycle (or a tile with more than 256 outside receivers): the
            # reference's own rounds, which define a result there
            if value is not None:
                self.Q.fill_(float(value))
        wp, wn = self._ws_acc.get(lib.pff_accumulate_workspace_bytes(self.N), self.device)
        _lib.call("pff_accumulate_grid", self.receivers.data_ptr(), self.Q.data_ptr(),
                  self.counts.data_ptr() if counts else None, self.nx, self.ny, self.mode, self._codes(), self.N,
                  wp, wn, _dev.stream())

    def accumulate_constant_Q(self, value, area=True, counts=True, exact_order=False):
        """flowfields.py:254-292: Q = value*dx^2 (area) or value per cell,
        accumulated upstream; the exact uint32 upstream cell counts land in
        ``counts``.  Q is the exact upstream sum rounded once to f32 (the
        reference's f32 sums carry their own rounding); exact_order=True gives the
        reference's f32 summation order bit for bit instead."""
        v = value * (self.dx * self.dx if area else 1.0)
        if exact_order:
            self.Q.fill_(v)
            self._accumulate(counts, exact_order=True)
        else:
            self._accumulate(counts, value=float(np.float32(v)))

    def route_many(self, dems, weights=None, out_Q=None, out_counts=None, carve=True):
        """Route a sequence of DEMs of this grid: for each k, z = dems[k] ->
        compute_receivers -> reroute_flow(carve) -> accumulate (weights[k] per cell,
        or 1 per cell with area False) -> out_Q[k], out_counts[k].

        dems, weights, out_Q, out_counts are host tensors (pinned for overlap) of N
        elements each (counts as int32 bits of the uint32 values).  The host-to-device
        copy of DEM k+1 and the device-to-host copy of the results of DEM k-1 run on
        two copy streams while DEM k is routed, so a long sequence costs about the
        routing time when the copies are shorter.  No reference counterpart (the
        reference routes one DEM per call).  Returns when every copy has landed."""
        n = len(dems)
        if n == 0:
            return
        dev = self.device
        main = torch.cuda.current_stream(dev)
        if getattr(self, "_rm", None) is None:  # double buffers and copy streams, kept for later calls
            N = self.N
            self._rm = dict(h2d=torch.cuda.Stream(dev), d2h=torch.cuda.Stream(dev),
                            zb=[torch.empty(N, dtype=torch.float32, device=dev) for _ in range(2)],
                            wb=[torch.empty(N, dtype=torch.float32, device=dev) for _ in range(2)],
                            qb=[torch.empty(N, dtype=torch.float32, device=dev) for _ in range(2)],
                            cb=[torch.empty(N, dtype=torch.int32, device=dev) for _ in range(2)])
        rm = self._rm
        h2d, d2h = rm["h2d"], rm["d2h"]
        zb, qb, cb = rm["zb"], rm["qb"], rm["cb"]
        wb = rm["wb"] if weights is not None else None
        h2d.wait_stream(main)  # the buffers' previous users (an earlier call) are done
        d2h.wait_stream(main)
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_used = [torch.cuda.Event() for _ in range(2)]
        ev_out = [torch.cuda.Event() for _ in range(2)]
        ev_drained = [torch.cuda.Event() for _ in range(2)]
        start = torch.cuda.Event()
        start.record(main)

        def load(k):
            b = k & 1
            h2d.wait_event(start)
            if k >= 2:
                h2d.wait_event(ev_used[b])  # DEM k-2 has left this buffer
            with torch.cuda.stream(h2d):
                zb[b].copy_(dems[k].reshape(-1), non_blocking=True)
                if wb is not None:
                    wb[b].copy_(weights[k].reshape(-1), non_blocking=True)
            ev_in[b].record(h2d)

        load(0)
        for k in range(n):
            b = k & 1
            if k + 1 < n:
                load(k + 1)
            main.wait_event(ev_in[b])
            self.z.copy_(zb[b])
            if wb is not None:
                self.Q.copy_(wb[b])
            else:
                self.Q.fill_(1.0)
            ev_used[b].record(main)
            self.compute_receivers()
            if self.lakeflow:
                self.reroute_flow(carve)
            self._accumulate(True)
            if k >= 2:
                main.wait_event(ev_drained[b])  # results of DEM k-2 have left this buffer
            qb[b].copy_(self.Q)
            cb[b].copy_(self.counts)
            ev_out[b].record(main)
            d2h.wait_event(ev_out[b])
            with torch.cuda.stream(d2h):
                if out_Q is not None:
                    out_Q[k].reshape(-1).copy_(qb[b], non_blocking=True)
                if out_counts is not None:
                    out_counts[k].reshape(-1).copy_(cb[b], non_blocking=True)
            ev_drained[b].record(d2h)
        main.wait_stream(d2h)
        main.wait_stream(h2d)

    def accumulate_weighted_Q(self, weights, counts=True, exact_order=False):
        """Upstream sum of per-cell weights (e.g. precipitation-weighted
        discharge), the path scripts run by filling Q before rcv2donor
        (examples/exemple_raw_1.py:135-150).  Exact sum rounded once to f32, or
        the reference's f32 summation order with exact_order=True."""
        if isinstance(weights, torch.Tensor):
            self.Q.copy_(weights.reshape(-1).to(torch.float32))
        else:
            self.Q.copy_(torch.from_numpy(np.ascontiguousarray(np.asarray(weights, np.float32).ravel())))
        self._accumulate(counts, exact_order=exact_order)
