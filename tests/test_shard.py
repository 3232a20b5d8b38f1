"""Multi-rank ragged batches: tiles are independent, so ranks take disjoint shares
(largest-first bin packing) and need no collective on the data path.  Checked here
with 2 CPU ranks over gloo: the shares cover the batch exactly once, are balanced,
and routing each share (with the oracle, the CPU stand-in for a rank's GPU) and
gathering the whole per-tile arrays gives the single-process results.  A GPU test
routes the same kind of shares through RaggedRouter, the product's sharded path."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from pyfastflow_b200 import synthetic
from pyfastflow_b200.flow.ragged import partition_tiles


def test_partition_lpt_properties():
    rng = np.random.default_rng(0)
    cells = rng.integers(100, 100000, 97).tolist()
    for world in (1, 2, 3, 8):
        parts = partition_tiles(cells, world)
        flat = sorted(t for p in parts for t in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[t] for t in p) for p in parts]
        # LPT: no rank exceeds the mean by more than the largest tile
        assert max(loads) <= sum(cells) / world + max(cells)
    assert partition_tiles([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    from oracle import oracle as orc

    tiles = synthetic.ragged_tiles(ntiles=7, seed=3, side_min=16, side_max=48, max_pits=4)
    parts = partition_tiles([t["nx"] * t["ny"] for t in tiles], world)
    mine = {}
    for k in parts[rank]:
        t = tiles[k]
        g = orc.Grid(t["nx"], t["ny"], {"normal": 0, "periodic_EW": 1}[t["mode"]])
        rcv, _ = orc.compute_receivers(t["z"], g, t["dx"])
        r, _, _, _, _ = orc.reroute_flow(rcv, t["z"], g)
        Q, cnt = orc.accumulate(r, 1.0)
        mine[k] = (r, Q.view(np.uint32), cnt)  # whole per-tile arrays
    gathered = [None] * world
    dist.all_gather_object(gathered, (parts[rank], mine))  # results only; no data-path collective
    if rank == 0:
        out.put(gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_cover_the_batch(orc):
    ctx = mp.get_context("spawn")
    out = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = out.get()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    shares = [set(g[0]) for g in gathered]
    assert shares[0].isdisjoint(shares[1]) and shares[0] | shares[1] == set(range(7))
    results = {}
    for _, m in gathered:
        results.update(m)
    # the same tiles routed in one process
    tiles = synthetic.ragged_tiles(ntiles=7, seed=3, side_min=16, side_max=48, max_pits=4)
    for k, t in enumerate(tiles):
        g = orc.Grid(t["nx"], t["ny"], {"normal": 0, "periodic_EW": 1}[t["mode"]])
        rcv, _ = orc.compute_receivers(t["z"], g, t["dx"])
        r, _, _, _, _ = orc.reroute_flow(rcv, t["z"], g)
        Q, cnt = orc.accumulate(r, 1.0)
        rk, qk, ck = results[k]
        assert np.array_equal(rk, r) and np.array_equal(qk, Q.view(np.uint32)) and np.array_equal(ck, cnt)


@pytest.mark.gpu
def test_sharded_shares_through_raggedrouter(orc, cuda):
    """The product's sharded path on one GPU: each of two largest-first shares is
    routed by its own RaggedRouter (what each rank runs), and every tile equals the
    unsharded batch and the oracle, bit for bit."""
    import pyfastflow_b200 as pf

    tiles = synthetic.ragged_tiles(ntiles=10, seed=5, side_min=64, side_max=300, max_pits=40)
    parts = partition_tiles([t["nx"] * t["ny"] for t in tiles], 2)
    assert all(parts) and sorted(parts[0] + parts[1]) == list(range(10))

    def route(sel):
        rr = pf.flow.RaggedRouter([(tiles[k]["ny"], tiles[k]["nx"]) for k in sel], 30.0,
                                  [tiles[k]["mode"] for k in sel])
        rr.set_z([tiles[k]["z"] for k in sel])
        rr.seed_constant(1.0, area=True)
        rr.route(graph=True)
        cuda.cuda.synchronize()
        return {k: (rr.get_receivers(j).ravel(), rr.get_Q(j).ravel().view(np.uint32), rr.get_counts(j).ravel())
                for j, k in enumerate(sel)}

    whole = route(list(range(10)))
    shards = {}
    for p in parts:
        shards.update(route(p))
    for k, t in enumerate(tiles):
        g = orc.Grid(t["nx"], t["ny"], {"normal": 0, "periodic_EW": 1}[t["mode"]])
        rcv, _ = orc.compute_receivers(t["z"], g, t["dx"])
        r, _, _, _, _ = orc.reroute_flow(rcv, t["z"], g)
        Q, cnt = orc.accumulate(r, np.float32(900.0))
        for got in (whole[k], shards[k]):
            assert np.array_equal(got[0], r) and np.array_equal(got[1], Q.view(np.uint32))
            assert np.array_equal(got[2], cnt)
