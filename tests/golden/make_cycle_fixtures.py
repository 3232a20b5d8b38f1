"""Generate tests/golden/cycle_crops.npz: water-surface crops on which carving
closes a cycle of basins (three pits whose saddles tie), so the receivers hold a
cycle that the reference resolves (or not) in later outer iterations.

Recipe: the 512 x 512 GraphFlood workload (pyfastflow_b200.synthetic.graphflood_plain,
dx 10 m, P 1e-5 m/s, n 0.033) advanced 446 iterations by the CPU oracle; zh is then
cropped around row 314, column 462 with half-widths 8 and 16.

Run from the repository root:  python tests/golden/make_cycle_fixtures.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from pyfastflow_b200 import synthetic  # noqa: E402


def main():
    n, iters = 512, 446
    z = synthetic.graphflood_plain(n)["z"]
    g = O.Grid(n, n, 0)
    zh, h, Q = z.ravel().copy(), np.zeros(n * n, np.float32), np.zeros(n * n, np.float32)
    O.graphflood_run(zh, h, Q, g, 10.0, 1e-5, niter=iters)
    zh = zh.reshape(n, n)
    r0, c0 = 314, 462
    out = {}
    for half in (8, 16):
        out[f"crop{2 * half}"] = zh[r0 - half:r0 + half, c0 - half:c0 + half].copy()
    np.savez(os.path.join(os.path.dirname(os.path.abspath(__file__)), "cycle_crops.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
