"""Generate tests/golden/graphflood_2048_50.json: the CPU oracle's GraphFlood on the
2048 x 2048 benchmark DEM (pyfastflow_b200.synthetic.graphflood_plain: dx 10 m,
P 1e-5 m/s, Manning 0.033, h0 = 0), 50 iterations (each with receivers, carve
rerouting, fill, 5 diffusion sweeps and the Manning update):

- SHA-256 of the f32 bit patterns of h, zh and Q (NaNs canonicalised), which the
  GPU test compares with the CUDA path's;
- the same 50 iterations in f64 (the same update, oracle f64 build) and the f32
  run's error against it.

Run from the repository root: python tests/golden/make_graphflood_2048_fixture.py
(about ten minutes on 8 cores)."""
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from pyfastflow_b200 import synthetic  # noqa: E402

N_SIDE, ITERS = 2048, 50


def canon_bits(a):
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).copy()
    b[np.isnan(a)] = 0x7FC00000
    return b


def sha(a):
    return hashlib.sha256(canon_bits(a).tobytes()).hexdigest()


def main():
    O.build()
    O.set_threads(os.cpu_count() or 1)
    z = synthetic.graphflood_plain(N_SIDE)["z"].ravel()
    g = O.Grid(N_SIDE, N_SIDE, 0)
    t0 = time.time()
    zh, h, Q = z.astype(np.float32).copy(), np.zeros(z.size, np.float32), np.zeros(z.size, np.float32)
    tr32 = O.graphflood_run(zh, h, Q, g, 10.0, 1e-5, niter=ITERS)
    t32 = time.time() - t0
    zh64, h64, Q64 = z.astype(np.float64).copy(), np.zeros(z.size), np.zeros(z.size)
    O.graphflood_run(zh64, h64, Q64, g, 10.0, 1e-5, niter=ITERS, f64=True)
    wet = h64 > 1e-3
    flow = Q64 > 0

    def rel(a, b, m):
        r = np.abs(a[m].astype(np.float64) - b[m]) / np.abs(b[m])
        return float(r.max()) if r.size else 0.0, float(r.mean()) if r.size else 0.0

    def pct(a, b, m):
        r = np.abs(a[m].astype(np.float64) - b[m]) / np.abs(b[m])
        return {"p50": float(np.percentile(r, 50)), "p90": float(np.percentile(r, 90)),
                "p99": float(np.percentile(r, 99))}

    hr, hm = rel(h, h64, wet)
    qr, qm = rel(Q, Q64, flow)
    same_rcv = float(np.mean(O.compute_receivers(zh, g, 10.0)[0] == O.compute_receivers(zh64, g, 10.0, f64=True)[0]))
    out = {
        "dem": f"synthetic.graphflood_plain({N_SIDE})", "dx": 10.0, "precipitation": 1e-5, "manning": 0.033,
        "iterations": ITERS, "sha256": {"h": sha(h), "zh": sha(zh), "Q": sha(Q)},
        "nan": {"h": int(np.isnan(h).sum()), "Q": int(np.isnan(Q).sum())},
        "max_dh_last": float(tr32[-1]),
        "fp64": {"h_wet_cells": int(wet.sum()), "h_max_rel": hr, "h_mean_rel": hm,
                 "h_max_abs": float(np.nanmax(np.abs(h - h64))),
                 "h_rel_percentiles": pct(h, h64, wet),
                 "Q_cells": int(flow.sum()), "Q_max_rel": qr, "Q_mean_rel": qm,
                 "Q_rel_percentiles": pct(Q, Q64, flow),
                 "water_volume_rel": float(abs(np.float64(h.astype(np.float64).sum()) - h64.sum()) / h64.sum()),
                 "same_receivers_fraction": same_rcv,
                 "note": "relative error of the f32 run against the f64 run of the same update, over cells with "
                         "h64 > 1 mm (h) and Q64 > 0 (Q); the two runs route on their own surfaces, so a rounding "
                         "difference that flips a receiver on a flat moves water to another path: the tails are "
                         "routing decisions, the medians and the total volume the arithmetic"},
        "oracle_seconds_f32": round(t32, 1),
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "graphflood_2048_50.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
