"""Benchmark: Mcells/s of receivers -> carve reroute -> accumulate on one DEM.

Workload (default): 4096 x 4096 float32 DEM from the seeded spectral generator
(relief 0-1500 m, 2000 Gaussian pits), periodic east-west with outlets on the
north and south rows, carve rerouting on, accumulation of exact uint32 counts and
lognormal(0, 0.5) precipitation-weighted discharge in one pass.

A step = FlowRouter.compute_receivers -> reroute_flow -> accumulate_weighted_Q
on the resident DEM.  value = cells x steps / device time (CUDA events, L2
flushed between steps).  e2e = the same chain through the public API with the
DEM and weights copied from pinned host memory and Q + counts copied back, every
step, inside the timed region.

--impl reference times the CPU restatement of the reference algorithm (the
reference itself is Python on Taichi, which is not installable here) on the
same full workload with all host threads, one chain per step.

roofline: the kernel with the largest event time per step among the probed
kernels (library-side CUDA events around each launch, in a separate pass with
the reroute loop driven from the host so that its kernels launch one by one).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcells/s route+reroute+accumulate"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# algorithmic bytes per cell (z in, rcv+gradient out | rcv+z in, rcv+bid out | rcv+w in, Q+counts out)
ALG_BYTES = {"receivers": 12, "reroute": 16, "accumulate": 16}
# Probed kernels: algorithmic bytes per cell of a launch over the whole grid
# (None: the launch covers a varying list of tiles), and DRAM read + write bytes
# of one 4096^2 launch from an ncu capture of this workload (None: not captured).
KERNELS = {
    "k_receivers": (12, 152.3e6),           # z in; receivers + gradient out
    "k_tile_terminal<grid>": (8, None),     # receivers in; tile terminals out
    "k_tile_terminal<list>": (None, None),  # the tiles a carve changed
    "k_saddle_p12_strip": (13, None),       # labels + z in; is_border + z' out (the border lists are extra)
    "k_tree_tile<up>": (8, 251.0e6),        # receivers + seeds in
    "k_tree_tile<down>": (16, 323.0e6),     # receivers + seeds in; Q + counts out
}


def peak_hbm():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(n, seed=2):
    from pyfastflow_b200 import synthetic

    cache = os.path.join(tempfile.gettempdir(), f"pff_routing_lakes_{n}_{seed}.npz")
    if os.path.exists(cache):
        d = np.load(cache)
        return d["z"], d["w"]
    w = synthetic.routing_lakes(n, seed=seed)
    wt = synthetic.lognormal_weights(n * n, seed + 100)
    try:
        np.savez(cache, z=w["z"], w=wt)
    except OSError:
        pass
    return w["z"], wt


class Clocks:
    """SM clock and clock-event reasons sampled through NVML while the
    timed region runs (read-only queries, every 5 ms); nvidia-smi every 200 ms when NVML is
    not importable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []  # (sm_mhz, max_mhz, reason names)
        self.proc = None
        self.stop = threading.Event()
        self.t = None
        self.error = None

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:  # the same device as torch's, also under CUDA_VISIBLE_DEVICES
            uuid = str(torch.cuda.get_device_properties(self.idx).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.idx)

    def _poll(self, nv, h):
        try:
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self.stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((float(sm), float(mx), [k for k, b in self.REASONS.items() if bits & b]))
                self.stop.wait(0.002)
        except Exception as e:  # reported in the summary
            self.error = f"{type(e).__name__}: {e}"

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.t = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.t.start()
            # the region starts once the sampler has its first row (at most 0.5 s):
            # a short region must not end before the thread is scheduled
            t0 = time.perf_counter()
            while not self.rows and self.error is None and time.perf_counter() - t0 < 0.5:
                time.sleep(0.001)
            return self
        except Exception as e:
            self.error = f"{type(e).__name__}: {e}"
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            if len(r) >= 9 and r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                self.rows.append((float(r[1]), float(r[2]), [names[k] for k in range(4) if r[5 + k] == "Active"]))

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.t:
            self.t.join(timeout=5)

    def summary(self):
        if not self.rows:
            out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
            if self.error:
                out["error"] = self.error
            return out
        out = {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
               "reasons": sorted({x for r in self.rows for x in r[2]}), "samples": len(self.rows),
               "source": "nvml" if self.proc is None else "nvidia-smi"}
        if self.error:  # a query that failed part-way: the samples cover only part of the region
            out["error"] = self.error
        return out


def run_cpu_reference(z, w, n, threads):
    """The CPU restatement of the reference chain (oracle) on one DEM; returns seconds."""
    from oracle import oracle as O

    g = O.Grid(n, n, 1)
    t0 = time.perf_counter()
    rcv, _ = O.compute_receivers(z, g, 30.0)
    r2, _, _, _, _ = O.reroute_flow(rcv, z, g, carve=True)
    O.accumulate(r2, w, with_counts=True)
    return time.perf_counter() - t0


def cpu_setup(threads):
    from oracle import oracle as O

    O.build()
    return O.set_threads(threads)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="routing", choices=["routing", "graphflood", "ragged", "conv", "warmstart"])
    ap.add_argument("--tau", type=float, default=30.0, help="warmstart: stop when mean|dh|/dt < tau * P")
    ap.add_argument("--train-tiles", type=int, default=512)
    ap.add_argument("--train-iters", type=int, default=30000)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--eval-tiles", type=int, default=64)
    ap.add_argument("--eval-size", type=int, default=512)
    ap.add_argument("--eval-scenarios", type=int, default=4)
    ap.add_argument("--tiles", type=int, default=512)
    ap.add_argument("--no-per-tile", action="store_true", help="ragged: skip the per-tile comparison arm")
    ap.add_argument("--no-tune", action="store_true", help="ragged: fixed 1024 threads x 1 CTA per SM")
    ap.add_argument("--per-layer", action="store_true", help="conv: also time every layer on both kernels")
    ap.add_argument("--max-iter", type=int, default=20000)
    ap.add_argument("--fp64-size", type=int, default=256)
    ap.add_argument("--fp64-iters", type=int, default=200)
    args = ap.parse_args()
    if args.workload == "ragged":
        return ragged_main(args)
    if args.workload == "conv":
        return conv_main(args)
    if args.workload == "warmstart":
        return warmstart_main(args)
    if args.workload == "graphflood":
        return graphflood_main(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    n = args.size
    cfg = {"workload": f"routing_lakes {n}x{n} f32 DEM, relief 0-1500 m, 2000 pits per 4096^2, periodic EW, "
                       "carve reroute, uint32 counts + lognormal(0,0.5) weighted Q",
           "cells": n * n, "dx": 30.0, "boundary": "periodic_EW", "l2": "flushed between steps (256 MiB write)"}

    if args.impl == "reference":
        if rank != 0:
            return
        # the CPU restatement of the reference chain on the whole workload: the same
        # n x n DEM and weights the GPU arm routes, one full chain per step
        used = cpu_setup(os.cpu_count() or 1)
        z, w = workload(n)
        for _ in range(args.warmup):
            run_cpu_reference(z, w, n, used)
        ts = [run_cpu_reference(z, w, n, used) for _ in range(args.steps)]
        tot = sum(ts)
        v = n * n * args.steps / tot / 1e6
        sample = f"the full {n}x{n} workload (same DEM and weights as the GPU arm), one chain per step"
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "Mcells/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / args.steps * 1e3,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": v, "unit": "Mcells/s", "cores": used, "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": v, "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return

    import torch

    import pyfastflow_b200 as pf
    from pyfastflow_b200 import _lib

    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    lib = _lib.load()

    z, w = workload(n)
    router = pf.flow.FlowRouter(n, n, 30.0, boundary_mode="periodic_EW", device=dev)
    router.set_z(z)
    wd = torch.from_numpy(w).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        router.compute_receivers()
        router.reroute_flow()
        router.accumulate_weighted_Q(wd)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- device-timed value ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    l0 = lib.pff_launch_count()
    with Clocks(torch.cuda.current_device()) as clk:
        barrier()
        for s in range(args.steps):
            flush.fill_(s & 0xFF)
            ev[s][0].record()
            step()
            ev[s][1].record()
        barrier()
    launches = (lib.pff_launch_count() - l0) // args.steps
    ms = sum(a.elapsed_time(b) for a, b in ev)
    t_dev = torch.tensor([ms], device=dev)
    if world > 1:
        torch.distributed.all_reduce(t_dev, op=torch.distributed.ReduceOp.MAX)
    ms = float(t_dev.item())
    value = world * n * n * args.steps / (ms * 1e-3) / 1e6

    # ---- per-stage times (separate pass) -> roofline of the dominant stage ----
    stages = {"receivers": [], "reroute": [], "accumulate": []}
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record()
        router.compute_receivers()
        e[1].record()
        router.reroute_flow()
        e[2].record()
        router.accumulate_weighted_Q(wd)
        e[3].record()
        torch.cuda.synchronize()
        for k, name in enumerate(stages):
            stages[name].append(e[k].elapsed_time(e[k + 1]))
    st_ms = {k: sum(v) / len(v) for k, v in stages.items()}
    pk, pk_kind = peak_hbm()

    # ---- per-kernel event times (separate pass, probes armed) -> roofline ----
    import ctypes

    prev_graphs = lib.pff_reroute_use_graphs(0)
    lib.pff_probe_enable(1)
    for s in range(args.steps):
        flush.fill_(s & 0xFF)
        step()
    torch.cuda.synchronize()
    kernels = {}
    for name, (bpc, traffic) in KERNELS.items():
        tot, nl = ctypes.c_double(), ctypes.c_int()
        if lib.pff_probe_read(name.encode(), ctypes.byref(tot), ctypes.byref(nl)) != 0 or nl.value == 0:
            continue
        per = tot.value / nl.value
        k = {"ms_per_launch": per, "launches_per_step": nl.value / args.steps, "ms_per_step": tot.value / args.steps}
        if bpc is not None:
            k["alg_bytes_per_launch"] = bpc * n * n
            k["achieved_gbs"] = bpc * n * n / (per * 1e-3) / 1e9
            k["frac"] = k["achieved_gbs"] / pk
            k["traffic"] = traffic * (n * n) / 16777216.0 if traffic else None
        kernels[name] = k
    lib.pff_probe_enable(0)
    lib.pff_reroute_use_graphs(prev_graphs)
    timed = [k for k in kernels if "alg_bytes_per_launch" in kernels[k]]
    dom = max(timed, key=lambda k: kernels[k]["ms_per_step"])
    kd = kernels[dom]
    roofline = {"bound": "hbm", "kernel": dom, "achieved": kd["achieved_gbs"], "peak": pk, "unit": "GB/s",
                "frac": kd["frac"], "peak_source": pk_kind, "traffic": kd["traffic"],
                "alg_bytes_per_launch": kd["alg_bytes_per_launch"], "ms_per_launch": kd["ms_per_launch"],
                "traffic_note": "DRAM read + write of one launch of this workload from an ncu capture",
                "kernels": kernels, "stage_ms": st_ms}
    # the stencil kernel (receivers), 12 algorithmic bytes per cell
    kr = kernels.get("k_receivers")
    roofline_stencil = None
    if kr:
        roofline_stencil = {"bound": "hbm", "kernel": "k_receivers", "achieved": kr["achieved_gbs"], "peak": pk,
                            "unit": "GB/s", "frac": kr["frac"], "peak_source": pk_kind,
                            "alg_bytes_per_launch": kr["alg_bytes_per_launch"], "ms_per_launch": kr["ms_per_launch"],
                            "traffic": kr["traffic"],
                            "traffic_note": "DRAM read+write of one 4096^2 launch from an ncu capture (71.3 + 81.0 MB), "
                                            "scaled by cells"}

    # ---- e2e through the public API with host buffers ----
    zh = torch.from_numpy(z.ravel()).pin_memory()
    wh = torch.from_numpy(w).pin_memory()
    qh = torch.empty(n * n, dtype=torch.float32).pin_memory()
    ch = torch.empty(n * n, dtype=torch.int32).pin_memory()
    e2e_steps = max(2, args.steps)  # as many DEMs as timed steps: the first copy in and the last copy out do not overlap
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # one DEM per step through FlowRouter.route_many: every step copies its DEM and
    # weights in and its Q and counts out; the copies of neighbouring steps overlap
    # the routing on two copy streams
    qhs = [qh] * e2e_steps
    chs = [ch] * e2e_steps
    router.route_many([zh] * 2, [wh] * 2, qhs[:2], chs[:2])  # untimed: creates the copy streams and buffers
    torch.cuda.synchronize()
    barrier()
    e0.record()
    router.route_many([zh] * e2e_steps, [wh] * e2e_steps, qhs, chs)
    e1.record()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    t_e = torch.tensor([e2e_ms], device=dev)
    if world > 1:
        torch.distributed.all_reduce(t_e, op=torch.distributed.ReduceOp.MAX)
    e2e_v = world * n * n * e2e_steps / (float(t_e.item()) * 1e-3) / 1e6

    # the host link alone: the same per-step copies (DEM and weights in, Q and counts out, on two
    # copy streams at once) without the routing, the bound the end-to-end figure can reach
    cs_in, cs_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    zd_c, wd_c = torch.empty(n * n, dtype=torch.float32, device=dev), torch.empty(n * n, dtype=torch.float32, device=dev)
    qd_c, cd_c = torch.empty(n * n, dtype=torch.float32, device=dev), torch.empty(n * n, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record()
    cs_in.wait_event(c0)
    cs_out.wait_event(c0)
    for _ in range(e2e_steps):
        with torch.cuda.stream(cs_in):
            zd_c.copy_(zh, non_blocking=True)
            wd_c.copy_(wh, non_blocking=True)
        with torch.cuda.stream(cs_out):
            qh.copy_(qd_c, non_blocking=True)
            ch.copy_(cd_c, non_blocking=True)
    torch.cuda.current_stream().wait_stream(cs_in)
    torch.cuda.current_stream().wait_stream(cs_out)
    c1.record()
    torch.cuda.synchronize()
    copy_ms = c0.elapsed_time(c1) / e2e_steps
    del zd_c, wd_c, qd_c, cd_c

    out = {"metric": METRIC, "value": value, "unit": "Mcells/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded spectral DEM + Gaussian pits)",
           "config": dict(cfg, parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                          n_outer_reroute=router.last_n_outer),
           "roofline": roofline, "roofline_stencil": roofline_stencil, "clocks": clk.summary(),
           "gpu_launches": int(launches),
           "e2e": {"value": e2e_v, "unit": "Mcells/s", "h2d_bytes_per_step": 8 * n * n,
                   "d2h_bytes_per_step": 8 * n * n, "steps": e2e_steps,
                   "api": "FlowRouter.route_many (copies of neighbouring steps overlap the routing)",
                   "copies_alone_ms_per_step": copy_ms,
                   "copies_alone_mcells": n * n / (copy_ms * 1e-3) / 1e6}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # bounded: one run of the whole chain on the same DEM and weights (about 15 s
        # on 16 host cores), no warm-up (the restatement is compiled C: nothing to JIT)
        used = cpu_setup(os.cpu_count() or 1)
        t = run_cpu_reference(z, w, n, used)
        out["cpu_baseline"] = {"value": n * n / t / 1e6, "unit": "Mcells/s", "cores": used, "kind": "port",
                               "sample": f"one run of the full {n}x{n} chain on the GPU arm's DEM and weights"}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()


RG_METRIC = "Mcells/s ragged route+reroute+accumulate"


def ragged_main(args):
    """The ragged batch: --tiles tiles (sides log-uniform in [128, 1024], nx and ny
    drawn independently, 0-200 pits, modes normal / periodic EW, dx 30 m), routed in
    one persistent launch replayed from a CUDA graph, against the same chain run tile
    by tile through FlowRouter (per-tile launches).  Both arms compute exact counts
    and Q = dx^2 seeds; the batch is checked bit-for-bit against the per-tile arm."""
    import torch

    import pyfastflow_b200 as pf
    from pyfastflow_b200 import _lib, synthetic

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:  # each rank routes its own share of the tiles; no collective on the data path
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    lib = _lib.load()
    all_tiles = synthetic.ragged_tiles(ntiles=args.tiles, seed=4)
    parts = pf.flow.ragged.partition_tiles([t["nx"] * t["ny"] for t in all_tiles], world)
    tiles = [all_tiles[k] for k in parts[rank]]
    total_all = sum(t["nx"] * t["ny"] for t in all_tiles)
    shapes = [(t["ny"], t["nx"]) for t in tiles]
    rr = pf.flow.RaggedRouter(shapes, 30.0, [t["mode"] for t in tiles])
    zp = rr.packed([t["z"] for t in tiles])
    rr.set_z(zp)
    rr.seed_constant(1.0, area=True)
    total = rr.total
    best = (rr.threads, rr.ctas_per_sm) if args.no_tune else rr.tune()
    for _ in range(args.warmup):
        rr.route(graph=True, check=False)
    rr.check_status()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps)]
    l0 = lib.pff_launch_count()
    with Clocks(0) as clk:
        for k in range(args.steps):
            ev[2 * k].record()
            rr.route(graph=True, check=False)
            ev[2 * k + 1].record()
        torch.cuda.synchronize()
    # each replay runs the captured graph: the seed copy plus 2 kernels (queue reset, batch route)
    launches = 2 * args.steps + (lib.pff_launch_count() - l0)
    ms = [ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(args.steps)]
    ms_step = sum(ms) / len(ms)
    rr.check_status()
    if world > 1:  # the job takes as long as its slowest rank
        t = torch.tensor([ms_step], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_step = float(t.item())
    value = total_all / (ms_step * 1e-3) / 1e6

    # e2e: packed DEM from pinned host memory in, receivers + Q + counts back, every step
    zh = torch.from_numpy(zp).pin_memory()
    rh = torch.empty(total, dtype=torch.int32).pin_memory()
    qh = torch.empty(total, dtype=torch.float32).pin_memory()
    ch = torch.empty(total, dtype=torch.int32).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        rr.z.copy_(zh, non_blocking=True)
        rr.route(graph=True, check=False)
        rh.copy_(rr.receivers, non_blocking=True)
        qh.copy_(rr.Q, non_blocking=True)
        ch.copy_(rr.counts, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps

    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    if args.no_per_tile or world > 1:
        if rank == 0:
            print(json.dumps({"metric": RG_METRIC, "value": value, "unit": "Mcells/s", "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                              "higher_is_better": True, "scaling": "strong",
                              "config": {"tiles": args.tiles, "total_cells": total_all,
                                         "sharding": "LPT bin packing of whole tiles over ranks"},
                              "e2e": {"value": total_all / (e2e_ms * 1e-3) / 1e6, "unit": "Mcells/s"},
                              "per_tile_launches": None, "gpu_launches": launches}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    # per-tile launches: the same chain through FlowRouter, one tile at a time
    routers = []
    for t in tiles:
        fr = pf.flow.FlowRouter(t["nx"], t["ny"], 30.0, boundary_mode=t["mode"])
        fr.set_z(t["z"])
        routers.append(fr)

    def per_tile():
        for fr in routers:
            fr.compute_receivers()
            fr.reroute_flow()
            fr.accumulate_constant_Q(1.0, area=True, exact_order=True)  # the batch's summation order

    per_tile()
    torch.cuda.synchronize()
    e0.record()
    t0 = time.perf_counter()
    per_tile()
    e1.record()
    torch.cuda.synchronize()
    pt_ms = e0.elapsed_time(e1)
    pt_wall = time.perf_counter() - t0
    exact = True
    for k, fr in enumerate(routers):
        o, n = int(rr.offset[k]), rr.cells(k)
        exact &= bool(torch.equal(rr.receivers[o:o + n], fr.receivers))
        exact &= bool(torch.equal(rr.counts[o:o + n], fr.counts))
        exact &= bool(torch.equal(rr.Q[o:o + n].view(torch.int32), fr.Q.view(torch.int32)))
    sides = np.array([[t["nx"], t["ny"]] for t in tiles])
    hbm, src = peak_hbm()
    alg = 36.0 * total  # receivers 12 + reroute 16 + accumulate 8 B per cell
    out = {"metric": RG_METRIC, "value": value, "unit": "Mcells/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+i32", "data": "synthetic (seeded spectral DEMs + Gaussian pits)",
           "config": {"workload": f"ragged batch of {args.tiles} tiles, sides log-uniform [128,1024] (nx, ny "
                                  "independent), 0-200 pits, modes normal/periodic_EW, dx 30 m",
                      "total_cells": total, "largest_tile": int((sides[:, 0] * sides[:, 1]).max()),
                      "l2": "working set ~100 B/cell >> L2, no flush needed",
                      "tuned": {"threads": best[0], "ctas_per_sm": best[1]}, "graph": True},
           "e2e": {"value": total / (e2e_ms * 1e-3) / 1e6, "unit": "Mcells/s", "h2d_bytes_per_step": 4 * total,
                   "d2h_bytes_per_step": 12 * total},
           "per_tile_launches": {"value": total / (pt_ms * 1e-3) / 1e6, "unit": "Mcells/s", "device_s": pt_ms / 1e3,
                                 "wall_s": pt_wall, "speedup_of_batch": pt_ms / ms_step},
           "bit_exact_vs_per_tile": exact,
           "roofline": {"bound": "hbm", "achieved": alg / (ms_step * 1e-3) / 1e9, "peak": hbm,
                        "unit": "GB/s", "frac": alg / (ms_step * 1e-3) / 1e9 / hbm, "traffic": None,
                        "peak_source": src},
           "gpu_launches": launches, "clocks": clk.summary()}
    print(json.dumps(out))


CONV_METRIC = "TFLOP/s U-Net training step (BF16 conv fwd + dgrad + wgrad)"


def conv_main(args):
    """The warm-start U-Net's training step on a batch of 16 tiles of 128 x 128:
    forward, loss, backward (data and weight gradients of every 3x3 convolution),
    Adam.  FLOPs counted for the convolutions only: 2 * Cin * Cout * 9 per pixel
    forward, twice that backward (the head's data gradient included)."""
    import torch

    from pyfastflow_b200 import _lib
    from pyfastflow_b200.warmstart import LAYERS, UNet

    torch.cuda.set_device(0)
    lib = _lib.load()
    B, H, W = 16, 128, 128
    net = UNet(seed=0)
    g = torch.Generator().manual_seed(0)
    x = (torch.randn(B * H * W * 8, generator=g) * 0.5).to(torch.bfloat16).cuda()
    tgt = torch.randn(B * H * W, generator=g).cuda()
    flops = 0
    for name, _, _, _, _, cin, cout, _, lev in LAYERS:
        px = B * (H >> lev) * (W >> lev)
        f = 2.0 * cin * cout * 9 * px
        flops += f + (f if name != "enc0a" else 0) + f  # fwd, dgrad, wgrad

    def step():
        net.forward(x, B, H, W)
        loss, dp = net.loss_grad(tgt)
        net.backward(dp)
        net.adam_step(lr=1e-4)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    l0 = lib.pff_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    tf = flops / (ms * 1e-3) / 1e12
    try:
        with open(PEAKS) as f:
            pk = json.load(f)
        peak, src = float(pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))), "measured"
    except Exception:
        peak, src = 1400.0, "fallback"
    layers = None
    if args.per_layer:
        layers = conv_per_layer(B, H, W)
    print(json.dumps({"metric": CONV_METRIC, "value": tf, "per_layer": layers, "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "dtype": "bf16",
                      "data": "synthetic", "config": {"workload": f"U-Net step, batch {B} x {H} x {W}",
                                                      "conv_gflop_per_step": flops / 1e9},
                      "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                                   "frac": tf / peak, "traffic": None, "peak_source": src},
                      "gpu_launches": (lib.pff_launch_count() - l0), "clocks": clk.summary()}))


WS_METRIC = "graphflood s-to-residual, warm vs plain"


def warmstart_main(args):
    """Learned warm start for GraphFlood.

    1. Training data: --train-tiles 128 x 128 tiles (P ~ U(5e-6, 5e-5) m/s, n ~ U(0.02,
       0.06), dx 10 m), the plain iteration run --train-iters times from h = 0 on all
       tiles at once (RaggedFlooder); features after the first iteration.
    2. Training: the U-Net, --epochs epochs of Adam, on the BF16 tensor-core kernels.
    3. Held-out tiles (batched): cold vs warm (network) vs warm (kinematic depth, no
       network): iterations until mean|dh|/dt < tau * P, from per-iteration traces.
    4. Held-out --eval-size scenarios, one grid at a time through the public Flooder:
       device seconds until mean|dh|/dt < tau * P (at most 30000 iterations), cold
       vs warm, the warm time including the plain iteration, the routing of the
       filled surface and the network's inference.
    The reference's own stop (max|dh|/dt < 1e-4 P) is never reached by this update
    scheme (the first fill pours every depression's volume into h and the
    Manning step drains it over tens of thousands of iterations, and max|dh| stays
    above 1e-4 P from the fill's churn), so tau applies to the mean."""
    import torch

    import pyfastflow_b200 as pf
    from pyfastflow_b200 import _lib
    from pyfastflow_b200.warmstart import UNet, make_dataset, scenario_tiles, train, warm_start_batch, \
        warm_start_flooder

    torch.cuda.set_device(0)
    lib = _lib.load()
    t_start = time.perf_counter()
    logs = []

    def log(m):
        logs.append(f"{time.perf_counter() - t_start:7.1f}s {m}")
        print(logs[-1], file=sys.stderr, flush=True)

    side = 128
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    x, tgt, wgt = make_dataset(args.train_tiles, side, args.train_iters, seed=10, log=log)
    e1.record()
    torch.cuda.synchronize()
    data_s = e0.elapsed_time(e1) / 1e3
    net = UNet(seed=0)
    net.set_head_bias(float(tgt.mean()))
    e0.record()
    hist = train(net, x, tgt, side, weight=wgt, epochs=args.epochs, log=log)
    e1.record()
    torch.cuda.synchronize()
    train_s = e0.elapsed_time(e1) / 1e3
    log(f"data {data_s:.1f} s, training {train_s:.1f} s, loss {hist[0]:.3f} -> {hist[-1]:.3f}")

    # 3. held-out tiles, batched: iterations to the stop from traces
    NEV, CAP = args.eval_tiles, 30000
    etiles, eP, en = scenario_tiles(NEV, side, seed=99)
    rr = pf.flow.RaggedRouter([t.shape for t in etiles], 10.0, "normal")
    taus = [1000.0, 300.0, 100.0, 30.0, 10.0]
    first = {}
    for arm in ("cold", "warm_net", "warm_kinematic"):
        rr.set_z(etiles)
        fl = pf.graphflood.RaggedFlooder(rr, precipitation_rates=eP, manning=en)
        rr.Q.zero_()
        extra = 0
        if arm != "cold":
            warm_start_batch(fl, net, "net" if arm == "warm_net" else "kinematic")
            extra = 1
        _, _, tr = fl.run(CAP - extra, stop=None, trace=True)
        r = tr[:, :, 1] / (5e-3 * eP[:, None])
        first[arm] = {tau: [int(np.argmax(r[k] < tau)) + 1 + extra if (r[k] < tau).any() else None
                            for k in range(NEV)] for tau in taus}
        log(f"batched eval {arm} done")
    table = {}
    for tau in taus:
        row = {}
        for arm in first:
            v = [q for q in first[arm][tau] if q is not None]
            row[arm] = {"reached": len(v), "median_iterations": float(np.median(v)) if v else None}
        both = [(c, w) for c, w in zip(first["cold"][tau], first["warm_net"][tau]) if c is not None and w is not None]
        row["median_iteration_ratio_warm_net_over_cold"] = float(np.median([w / c for c, w in both])) if both else None
        table[str(tau)] = row

    # 4. single-grid scenarios, wall clock through the public API
    S = args.eval_size
    stiles, sP, sn = scenario_tiles(args.eval_scenarios, S, seed=77)
    scen = []
    for k in range(args.eval_scenarios):
        router = pf.flow.FlowRouter(S, S, 10.0)
        res = {}
        hs = {}
        for arm in ("cold", "warm"):
            router.set_z(stiles[k])
            router.Q.zero_()
            fl = pf.graphflood.Flooder(router, precipitation_rates=float(sP[k]), manning=float(sn[k]),
                                       edge_slope=1e-2)
            torch.cuda.synchronize()
            e0.record()
            extra = 0
            if arm == "warm":
                warm_start_flooder(fl, net)
                extra = 1
            it, why, resid = fl.run_to_residual(tol_ratio=args.tau, max_iter=CAP - extra, stop="mean")
            e1.record()
            torch.cuda.synchronize()
            res[arm] = {"seconds": e0.elapsed_time(e1) / 1e3, "iterations": it + extra, "stop": why,
                        "residual_over_P": resid / float(sP[k])}
            hs[arm] = fl.h.clone()
        d = (hs["warm"] - hs["cold"]).abs()
        res["final_h_warm_vs_cold"] = {"mean_abs_m": float(d.nanmean()),
                                       "rel_l1": float(d.nansum() / hs["cold"].abs().nansum()),
                                       "max_abs_m": float(d.nan_to_num(0).max())}
        res["P"], res["n"] = float(sP[k]), float(sn[k])
        scen.append(res)
        log(f"scenario {k}: cold {res['cold']['seconds']:.2f} s / {res['cold']['iterations']} it, "
            f"warm {res['warm']['seconds']:.2f} s / {res['warm']['iterations']} it")
    ratios = [r["warm"]["seconds"] / r["cold"]["seconds"] for r in scen]
    cold_s = float(np.median([r["cold"]["seconds"] for r in scen]))
    warm_s = float(np.median([r["warm"]["seconds"] for r in scen]))
    out = {"metric": WS_METRIC, "value": warm_s, "unit": "s", "n_gpus": 1, "steps": args.eval_scenarios,
           "warmup": 0, "ms_per_step": warm_s * 1e3, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 solver, bf16 network", "data": "synthetic (seeded spectral DEMs + pits)",
           "config": {"workload": f"graphflood {S}x{S} scenarios, dx 10 m, P ~ U(5e-6,5e-5), n ~ U(0.02,0.06); "
                                  f"stop mean|dh|/dt < {args.tau} P or 30000 iterations",
                      "train_tiles": args.train_tiles, "train_iters": args.train_iters, "epochs": args.epochs},
           "cold_seconds_median": cold_s, "warm_over_cold_median": float(np.median(ratios)),
           "warm_over_cold_per_scenario": ratios, "scenarios": scen,
           "batched_heldout_128": {"tiles": NEV, "cap": CAP, "iterations_to_mean_residual": table},
           "training": {"data_seconds": data_s, "train_seconds": train_s, "loss_first": hist[0],
                        "loss_last": hist[-1]},
           "log": logs}
    print(json.dumps(out))


def conv_per_layer(B, H, W, reps=10):
    """Forward time of every U-Net layer shape on the mma.sync kernel and (where it
    applies) the tcgen05 kernel, and the weight gradient, L2 flushed between runs."""
    import torch

    from pyfastflow_b200 import _dev, _lib
    from pyfastflow_b200.warmstart import LAYERS

    lib = _lib.load()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def timeit(fn):
        for _ in range(3):
            fn()
        ts = []
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts)) * 1e3

    out = {}
    for name, _, _, _, _, cin, cout, _, lev in LAYERS:
        h, w = H >> lev, W >> lev
        P = B * h * w
        x = (torch.randn(P * cin) * 0.5).to(torch.bfloat16).cuda()
        wt = (torch.randn(cout * 9 * cin) * 0.05).to(torch.bfloat16).cuda()
        y = torch.empty(P * cout, dtype=torch.bfloat16, device="cuda")
        fl = 2.0 * cin * cout * 9 * P
        row = {"shape": f"{B}x{h}x{w} {cin}->{cout}"}
        for path, key in ((1, "mma_sync_us"), (2, "tcgen05_us")):
            lib.pff_conv_set_path(path)
            try:
                row[key] = timeit(lambda: _lib.call("pff_conv3x3_fwd", x.data_ptr(), cin, 0, wt.data_ptr(), None,
                                                    y.data_ptr(), cout, 0, B, h, w, cin, cout, 1, 0, _dev.stream()))
                row[key.replace("_us", "_tflops")] = fl / row[key] / 1e6
            except _lib.PFFError:
                row[key] = None
        lib.pff_conv_set_path(0)
        dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device="cuda")
        row["wgrad_us"] = timeit(lambda: _lib.call("pff_conv3x3_wgrad", x.data_ptr(), cin, 0, y.data_ptr(), cout, 0,
                                                   dw.data_ptr(), B, h, w, cin, cout, _dev.stream()))
        out[name] = row
    return out


GF_METRIC = "graphflood s-to-residual"


def graphflood_main(args):
    """GraphFlood on the 2048 x 2048 DEM (dx 10 m, P 1e-5 m/s, n 0.033, h0 = 0,
    DT_HYDRO 5e-3): seconds until max|dh|/dt < 1e-4 * P or --max-iter iterations."""
    import torch

    import pyfastflow_b200 as pf
    from pyfastflow_b200 import _lib, synthetic

    n = args.size if args.size != 4096 else 2048
    torch.cuda.set_device(0)
    lib = _lib.load()
    w = synthetic.graphflood_plain(n)
    z = w["z"]
    P = 1e-5
    router = pf.flow.FlowRouter(n, n, 10.0)
    fl = pf.graphflood.Flooder(router, precipitation_rates=P, manning=0.033, edge_slope=1e-2)

    def reset():
        router.set_z(z)
        router.Q.zero_()
        fl.h.zero_()

    reset()
    for _ in range(args.warmup):
        fl.iteration()
    torch.cuda.synchronize()
    reset()
    torch.cuda.synchronize()
    l0 = lib.pff_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(0) as clk:
        t0 = time.perf_counter()
        e0.record()
        iters, reason, res, trace = fl.run_to_residual(tol_ratio=1e-4, max_iter=args.max_iter, return_trace=True)
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    dev_s = e0.elapsed_time(e1) / 1e3
    launches = (lib.pff_launch_count() - l0) / max(iters, 1)
    h = fl.get_h()
    tr = [float(x) for x in trace]
    out = {"metric": GF_METRIC, "value": dev_s, "unit": "s", "n_gpus": 1, "steps": 1, "warmup": args.warmup,
           "ms_per_step": dev_s * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic (seeded spectral DEM + Gaussian pits)",
           "config": {"workload": f"graphflood_plain {n}x{n}, dx 10 m, P 1e-5 m/s, n 0.033, h0 0, dt 5e-3, "
                                  "stop max|dh|/dt < 1e-4 P or max_iter", "max_iter": args.max_iter},
           "iterations": iters, "stop": reason, "final_residual": res,
           "ms_per_iteration": dev_s * 1e3 / max(iters, 1), "wall_s": wall, "gpu_launches_per_iteration": launches,
           "residual_trace": {str(k): tr[k - 1] for k in (1, 10, 100, 1000, 5000, 10000, 20000) if k <= len(tr)},
           "h_stats": {"max": float(np.nanmax(h)), "mean": float(np.nanmean(h)), "nan": int(np.isnan(h).sum()),
                       "wet_cells_1cm": int((h > 0.01).sum())},
           "clocks": clk.summary()}
    out["kernels"] = graphflood_kernel_probe(router, fl, reset, n, iters=min(20, args.max_iter))
    if args.fp64_iters > 0:
        out["fp64_check"] = graphflood_fp64_check(args.fp64_size, args.fp64_iters)
    print(json.dumps(out))


# Probed kernels of a GraphFlood iteration: algorithmic bytes per cell of one launch
# over the whole grid (None: the launch covers a varying list of tiles).
GF_KERNELS = {
    "k_receivers": 12,            # zh in; receivers + gradient out
    "k_tile_terminal<grid>": 8,   # receivers in; tile terminals out
    "k_tile_terminal<list>": None,
    "k_relabel_jump_block": None,  # one CTA: the basin chains of a short pit list
    "k_fill_round_packed": 16,    # one 8-byte {pointer, z} record in and out per round (the gather at the pointer is extra)
    "k_fill_round_late": 16,      # the same rounds from the tenth on (a round after a settled one returns at once)
    "k_diffuse_fused": 12,        # zh + Q in; Q after all sweeps out
    "k_core_fused": 28,           # receivers, filled z, h, Q in; dh, h, zh out
}


def graphflood_kernel_probe(router, fl, reset, n, iters):
    """Per-kernel device times of `iters` GraphFlood iterations from the library's
    event probes, run eagerly (no graphs: probes skip captured launches), with the
    achieved algorithmic GB/s against the measured HBM copy bandwidth."""
    import ctypes

    import torch

    from pyfastflow_b200 import _lib

    lib = _lib.load()
    pk, pk_kind = peak_hbm()
    reset()
    torch.cuda.synchronize()
    prev_graphs, prev_fl = lib.pff_reroute_use_graphs(0), fl.graphs
    fl.graphs = False
    lib.pff_probe_enable(1)
    for _ in range(iters):
        fl.iteration()
    torch.cuda.synchronize()
    res = {"iterations": iters, "peak": pk, "peak_source": pk_kind, "unit": "GB/s"}
    for name, bpc in GF_KERNELS.items():
        tot, nl = ctypes.c_double(), ctypes.c_int()
        if lib.pff_probe_read(name.encode(), ctypes.byref(tot), ctypes.byref(nl)) != 0 or nl.value == 0:
            continue
        per = tot.value / nl.value
        k = {"ms_per_launch": per, "launches_per_iteration": nl.value / iters, "ms_per_iteration": tot.value / iters}
        if bpc is not None:
            k["alg_bytes_per_launch"] = bpc * n * n
            k["achieved_gbs"] = bpc * n * n / (per * 1e-3) / 1e9
            k["frac"] = k["achieved_gbs"] / pk
        res[name] = k
    lib.pff_probe_enable(0)
    lib.pff_reroute_use_graphs(prev_graphs)
    fl.graphs = prev_fl
    return res


def graphflood_fp64_check(n, iters):
    """The same GraphFlood update run on an n x n DEM of the same generator for
    `iters` iterations: GPU f32 vs the CPU restatement in f32 (must match bit for
    bit) and in f64 (error reported)."""
    import torch

    import pyfastflow_b200 as pf
    from oracle import oracle as O
    from pyfastflow_b200 import synthetic

    O.build()
    z = synthetic.graphflood_plain(n)["z"]
    P = 1e-5
    router = pf.flow.FlowRouter(n, n, 10.0)
    router.set_z(z)
    fl = pf.graphflood.Flooder(router, precipitation_rates=P, manning=0.033, edge_slope=1e-2)
    fl.run_graphflood(iters)
    torch.cuda.synchronize()
    h32, Q32 = fl.get_h().ravel().astype(np.float64), router.get_Q().ravel().astype(np.float64)
    g = O.Grid(n, n, 0)
    zo, ho, Qo = z.ravel().copy(), np.zeros(n * n, np.float32), np.zeros(n * n, np.float32)
    O.graphflood_run(zo, ho, Qo, g, 10.0, P, niter=iters)
    z6, h6, Q6 = z.ravel().astype(np.float64), np.zeros(n * n), np.zeros(n * n)
    O.graphflood_run(z6, h6, Q6, g, 10.0, P, niter=iters, f64=True)
    wet = h6 > 1e-3
    rel_h = np.abs(h32 - h6)[wet] / h6[wet]
    rel_q = np.abs(Q32 - Q6) / np.maximum(np.abs(Q6), 1e-30)
    return {"grid": f"{n}x{n}", "iterations": iters,
            "gpu_vs_cpu_f32_bit_exact": bool(np.array_equal(fl.get_h().ravel().view(np.uint32), ho.view(np.uint32))
                                             and np.array_equal(router.get_Q().ravel().view(np.uint32),
                                                                Qo.view(np.uint32))),
            "h_abs_err_vs_f64": {"max": float(np.abs(h32 - h6).max()), "mean": float(np.abs(h32 - h6).mean())},
            "h_rel_err_vs_f64_wet": {"max": float(rel_h.max()) if rel_h.size else None,
                                     "mean": float(rel_h.mean()) if rel_h.size else None,
                                     "wet_cells_over_1mm": int(wet.sum())},
            "Q_rel_err_vs_f64": {"max": float(rel_q.max()), "mean": float(rel_q.mean())}}


if __name__ == "__main__":
    main()
