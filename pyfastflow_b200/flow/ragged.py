"""Ragged batches: many independent DEM tiles routed in one persistent launch.

The reference routes one grid per process (its grid size is a module global,
pyfastflow/constants.py).  ``RaggedRouter`` holds many tiles of their own shape,
cell size and boundary mode (0 normal, 1 periodic E-W, 2 periodic N-S, 3 custom
codes) packed back to back, and runs for every tile the chain a ``FlowRouter``
user runs tile by tile:

    compute_receivers()                 (flow/receivers.py:16-58)
    reroute_flow(carve=True)            (flow/lakeflow.py:466-538)
    accumulate_constant_Q / weighted    (flow/flowfields.py:254-292)

Results are bit-identical to those per-tile calls.  One launch covers the whole
batch; ``route(graph=True)`` replays it from a captured CUDA graph, and ``tune()``
picks the CTA size and residency by timing the candidates on the batch itself.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from .. import _dev, _lib
from ..constants import BOUND_MODES

# (threads per CTA, CTAs per SM) candidates of the autotuner
TUNE_CANDIDATES = ((1024, 1), (512, 1), (512, 2), (256, 2), (256, 4), (256, 5))
_tuned: dict = {}  # batch signature -> (threads, ctas_per_sm)


def partition_tiles(cells, world: int):
    """Split tiles over `world` ranks, largest first onto the least loaded rank
    (longest-processing-time bin packing; ties go to the lower rank).  Tiles are
    independent, so the ranks need no collective on the data path.  Returns one
    ascending list of tile indices per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cells = [int(c) for c in cells]
    order = sorted(range(len(cells)), key=lambda t: (-cells[t], t))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for t in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(t)
        load[r] += cells[t]
    return [sorted(p) for p in parts]


def _mode_code(m) -> int:
    if isinstance(m, str):
        m = BOUND_MODES[m]
    m = int(m)
    if m not in (0, 1, 2, 3):
        raise ValueError(f"boundary modes are 0-3 (normal, periodic_EW, periodic_NS, custom), got {m}")
    return m


class RaggedRouter:
    """A packed batch of tiles; ``shapes`` is a list of (ny, nx).  Custom-mode tiles
    ("custom" / 3) take their uint8 boundary codes (ny, nx) from ``codes``, a list
    with None for the other tiles (pyfastflow/constants.py:56-83 codes)."""

    def __init__(self, shapes, dx, modes, codes=None, device=None):
        self.ntiles = len(shapes)
        if self.ntiles == 0:
            raise ValueError("empty batch")
        self.device = _dev.resolve_device(device or "cuda")
        self.ny = np.array([int(s[0]) for s in shapes], np.int32)
        self.nx = np.array([int(s[1]) for s in shapes], np.int32)
        dxs = np.broadcast_to(np.asarray(dx, np.float64), (self.ntiles,))
        self.dx = [float(d) for d in dxs]
        ms = [modes] * self.ntiles if isinstance(modes, (str, int)) else list(modes)
        self.mode = np.array([_mode_code(m) for m in ms], np.int32)
        self.offset = np.zeros(self.ntiles, np.int64)
        self.order = np.zeros(self.ntiles, np.int32)
        lib = _lib.load()
        dx32 = np.asarray(self.dx, np.float32)
        args = (self.nx.ctypes.data, self.ny.ctypes.data, self.mode.ctypes.data, dx32.ctypes.data, self.ntiles,
                self.offset.ctypes.data, self.order.ctypes.data)
        total = lib.pff_batch_plan(*args, None, 0, None)
        if total < 0:
            raise _lib.PFFError(f"pff_batch_plan failed with status {-total}: "
                                f"{lib.pff_last_error_string().decode(errors='replace')}")
        self.total = int(total)
        self.ws_bytes = int(lib.pff_batch_workspace_bytes(self.total, self.ntiles))
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=self.device)
        _lib._sync_device()
        total = lib.pff_batch_plan(*args, self.ws.data_ptr(), self.ws_bytes, _dev.stream())
        if total != self.total:
            raise _lib.PFFError(f"pff_batch_plan failed with status {-total}: "
                                f"{lib.pff_last_error_string().decode(errors='replace')}")
        self.codes = None
        if (self.mode == 3).any():
            if codes is None or len(codes) != self.ntiles:
                raise ValueError("custom-mode tiles need a codes list (one entry per tile, None where unused)")
            packed = np.zeros(self.total, np.uint8)
            for t in range(self.ntiles):
                if self.mode[t] != 3:
                    continue
                c = np.asarray(codes[t], np.uint8)
                if c.size != self.cells(t):
                    raise ValueError(f"tile {t}: {c.size} codes for {self.cells(t)} cells")
                o = int(self.offset[t])
                packed[o:o + c.size] = c.ravel()
            self.codes = torch.from_numpy(packed).to(self.device)
        T = lambda dt: torch.zeros(self.total, dtype=dt, device=self.device)  # noqa: E731
        self.z = T(torch.float32)
        self.receivers = T(torch.int32)
        self.gradient = T(torch.float32)
        self.Q = T(torch.float32)
        self.seed = T(torch.float32)
        self.counts = T(torch.int32)  # uint32 bits
        self.threads, self.ctas_per_sm = _tuned.get(self.signature(), (1024, 1))
        self._graph = None
        self._graph_cfg = None

    # ---- layout -------------------------------------------------------------------------
    def signature(self):
        return (tuple(self.nx.tolist()), tuple(self.ny.tolist()), tuple(self.mode.tolist()))

    def cells(self, t: int) -> int:
        return int(self.nx[t]) * int(self.ny[t])

    def _slice(self, a: torch.Tensor, t: int) -> torch.Tensor:
        o = int(self.offset[t])
        return a[o:o + self.cells(t)]

    def packed(self, arrays) -> np.ndarray:
        """Concatenate per-tile (ny, nx) arrays in tile order into one float32 vector."""
        if len(arrays) != self.ntiles:
            raise ValueError(f"{len(arrays)} arrays for {self.ntiles} tiles")
        out = np.empty(self.total, np.float32)
        for t, a in enumerate(arrays):
            a = np.asarray(a, np.float32)
            if a.shape != (self.ny[t], self.nx[t]):
                raise ValueError(f"tile {t}: shape {a.shape}, expected ({self.ny[t]}, {self.nx[t]})")
            o = int(self.offset[t])
            out[o:o + a.size] = a.ravel()
        return out

    def set_z(self, dems):
        """dems: list of (ny, nx) arrays, or one packed float32 vector/tensor."""
        if isinstance(dems, torch.Tensor):
            self.z.copy_(dems.reshape(-1).to(torch.float32))
        elif isinstance(dems, np.ndarray) and dems.ndim == 1:
            self.z.copy_(torch.from_numpy(np.ascontiguousarray(dems, np.float32)))
        else:
            self.z.copy_(torch.from_numpy(self.packed(dems)))

    # ---- seeds --------------------------------------------------------------------------
    def seed_constant(self, value: float = 1.0, area: bool = True):
        """Per tile: Q = value*dx^2 (area) or value, as FlowRouter.accumulate_constant_Q."""
        for t in range(self.ntiles):
            v = value * (self.dx[t] * self.dx[t] if area else 1.0)
            self._slice(self.seed, t).fill_(v)

    def seed_weights(self, weights):
        """Per-cell weights: list of (ny, nx) arrays or one packed vector/tensor."""
        if isinstance(weights, torch.Tensor):
            self.seed.copy_(weights.reshape(-1).to(torch.float32))
        elif isinstance(weights, np.ndarray) and weights.ndim == 1:
            self.seed.copy_(torch.from_numpy(np.ascontiguousarray(weights, np.float32)))
        else:
            self.seed.copy_(torch.from_numpy(self.packed(weights)))

    # ---- routing ------------------------------------------------------------------------
    def _launch(self, threads: int, ctas: int):
        self.Q.copy_(self.seed)
        _lib.call("pff_batch_route", self.z.data_ptr(), self.codes.data_ptr() if self.codes is not None else None,
                  self.receivers.data_ptr(), self.gradient.data_ptr(),
                  self.Q.data_ptr(), self.counts.data_ptr(), self.total, self.ntiles, threads, ctas,
                  self.ws.data_ptr(), self.ws_bytes, _dev.stream())

    def route(self, graph: bool = False, check: bool = True):
        """receivers -> reroute(carve) -> accumulate for every tile, one launch.

        graph=True captures the launch (with the seed copy) in a CUDA graph on the
        first call and replays it afterwards.  check=True reads the status word
        (one host synchronisation) and raises on an error bit."""
        if graph:
            cfg = (self.threads, self.ctas_per_sm)
            if self._graph is None or self._graph_cfg != cfg:
                self._launch(*cfg)  # warm-up outside capture
                torch.cuda.synchronize(self.device)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._launch(*cfg)
                self._graph, self._graph_cfg = g, cfg
            self._graph.replay()
        else:
            self._launch(self.threads, self.ctas_per_sm)
        if check:
            self.check_status()

    def check_status(self):
        st = C.c_int(0)
        _lib.call("pff_batch_status", self.total, self.ntiles, self.ws.data_ptr(), self.ws_bytes, C.byref(st),
                  _dev.stream())
        if st.value:
            raise _lib.PFFError(f"ragged routing status {st.value} (1: bad tile mode, 8: receiver cycle with "
                                "mixed serial labels, 16: carve did not converge)")

    def tune(self, candidates=TUNE_CANDIDATES, reps: int = 2) -> tuple[int, int]:
        """Time each (threads, CTAs per SM) candidate on this batch, keep the fastest."""
        best, best_ms = None, float("inf")
        for th, ct in candidates:
            self._launch(th, ct)  # warm-up
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                self._launch(th, ct)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1) / reps
            if ms < best_ms:
                best, best_ms = (th, ct), ms
        self.threads, self.ctas_per_sm = best
        _tuned[self.signature()] = best
        self.tune_ms = best_ms
        return best

    # ---- results ------------------------------------------------------------------------
    def get_receivers(self, t: int) -> np.ndarray:
        return self._slice(self.receivers, t).cpu().numpy().reshape(self.ny[t], self.nx[t])

    def get_gradient(self, t: int) -> np.ndarray:
        return self._slice(self.gradient, t).cpu().numpy().reshape(self.ny[t], self.nx[t])

    def get_Q(self, t: int) -> np.ndarray:
        return self._slice(self.Q, t).cpu().numpy().reshape(self.ny[t], self.nx[t])

    def get_counts(self, t: int) -> np.ndarray:
        return self._slice(self.counts, t).cpu().numpy().view(np.uint32).reshape(self.ny[t], self.nx[t])
