"""Ragged batch: many tiles of their own shape, dx and boundary mode, routed in one
persistent launch.  Every tile must be bit-identical to the reference chain run on
that tile alone (receivers -> reroute_flow(carve) -> accumulate), checked against
the oracle.  Tiles include the receiver-cycle crops (tests/golden/cycle_crops.npz),
which exercise the serial cycle labelling and the largest-index reversal."""
import ctypes as C
import os

import numpy as np
import pytest

from pyfastflow_b200 import synthetic

HERE = os.path.dirname(os.path.abspath(__file__))
MODES = {"normal": 0, "periodic_EW": 1, "periodic_NS": 2}


def small_batch():
    tiles = synthetic.ragged_tiles(ntiles=12, seed=11, side_min=24, side_max=160, max_pits=30, dx=30.0)
    tiles[3]["mode"] = "periodic_NS"  # all three batched modes
    c = np.load(os.path.join(HERE, "golden", "cycle_crops.npz"))
    for name in ("crop16", "crop32"):
        z = c[name]
        tiles.append(dict(z=z, nx=z.shape[1], ny=z.shape[0], dx=10.0, mode="normal"))
    return tiles


def oracle_chain(orc, t, seed):
    g = orc.Grid(t["nx"], t["ny"], MODES[t["mode"]])
    rcv, grad = orc.compute_receivers(t["z"], g, t["dx"])
    r, _, _, _, _ = orc.reroute_flow(rcv, t["z"], g, carve=True)
    Q, cnt = orc.accumulate(r, seed)
    return grad, r, Q, cnt


def bits(a):
    """f32 bit patterns, every NaN mapped to one pattern (positions compared, payloads not)."""
    a = np.ascontiguousarray(a, np.float32).ravel()
    b = a.view(np.uint32).copy()
    b[np.isnan(a)] = 0x7FC00000
    return b


def _plan(lib, nx, ny, mode, dx, ws=None, wsb=0):
    n = len(nx)
    nx, ny, mode = (np.asarray(v, np.int32) for v in (nx, ny, mode))
    dx = np.asarray(dx, np.float32)
    off = np.zeros(n, np.int64)
    order = np.zeros(n, np.int32)
    tot = lib.pff_batch_plan(nx.ctypes.data, ny.ctypes.data, mode.ctypes.data, dx.ctypes.data, n, off.ctypes.data,
                             order.ctypes.data, ws, wsb, None)
    return tot, off, order


def test_plan_offsets_and_errors():
    """Host-side plan (size query): offsets, and argument errors as negated codes."""
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    tot, off, _ = _plan(lib, [5, 7, 3], [4, 2, 9], [0, 1, 2], [1.0, 2.0, 3.0])
    assert tot == 20 + 14 + 27
    assert off.tolist() == [0, 20, 34]
    assert lib.pff_batch_workspace_bytes(tot, 3) > 100 * tot
    tot, _, _ = _plan(lib, [5, 7], [4, 2], [0, 3], [1.0, 1.0])  # custom codes are batched too
    assert tot == 34
    tot, _, _ = _plan(lib, [5, 7], [4, 2], [0, 4], [1.0, 1.0])
    assert tot == -1 and b"mode 4" in lib.pff_last_error_string()
    tot, _, _ = _plan(lib, [1, 7], [4, 2], [0, 0], [1.0, 1.0])
    assert tot == -1
    tot, _, _ = _plan(lib, [4, 7], [4, 2], [0, 0], [1.0, 0.0])  # dx must be positive
    assert tot == -1
    small = C.create_string_buffer(64)
    tot, _, _ = _plan(lib, [5], [4], [0], [1.0], C.addressof(small), 64)
    assert tot == -4  # PFF_ERR_WORKSPACE


def test_ragged_generator_shapes():
    tiles = synthetic.ragged_tiles(ntiles=40, seed=4, side_min=128, side_max=1024, max_pits=5)
    sides = np.array([[t["nx"], t["ny"]] for t in tiles])
    assert sides.min() >= 128 and sides.max() <= 1024
    assert len({t["mode"] for t in tiles}) == 2
    assert (sides[:, 0] != sides[:, 1]).any()


@pytest.mark.gpu
def test_ragged_bit_exact_vs_oracle(orc, cuda):
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = small_batch()
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], [t["dx"] for t in tiles],
                              [t["mode"] for t in tiles])
    rr.set_z([t["z"] for t in tiles])
    rr.seed_constant(1.0, area=True)
    rr.route()
    torch.cuda.synchronize()
    for k, t in enumerate(tiles):
        seed = np.float32(1.0 * t["dx"] * t["dx"])
        grad, r, Q, cnt = oracle_chain(orc, t, seed)
        assert np.array_equal(rr.get_receivers(k).ravel(), r), f"tile {k} receivers"
        assert np.array_equal(bits(rr.get_gradient(k)), bits(grad)), f"tile {k} gradient"
        assert np.array_equal(rr.get_counts(k).ravel(), cnt), f"tile {k} counts"
        assert np.array_equal(bits(rr.get_Q(k)), bits(Q)), f"tile {k} Q"
    # the crops really took the cycle path: their rerouted receivers match the oracle,
    # which keeps a cycle in crop16
    k16 = len(tiles) - 2
    assert orc.count_cycle_nodes(rr.get_receivers(k16).ravel()) == 4


@pytest.mark.gpu
def test_ragged_weighted_graph_and_tuner(orc, cuda):
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = small_batch()[:8]
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], [t["dx"] for t in tiles],
                              [t["mode"] for t in tiles])
    rr.set_z([t["z"] for t in tiles])
    w = [synthetic.lognormal_weights(t["nx"] * t["ny"], 50 + k).reshape(t["ny"], t["nx"])
         for k, t in enumerate(tiles)]
    rr.seed_weights(w)
    best = rr.tune(reps=1)
    assert best in pf.flow.ragged.TUNE_CANDIDATES
    rr.route(graph=True)
    rr.Q.zero_()
    rr.receivers.zero_()
    rr.route(graph=True)  # replay of the captured launch recomputes everything
    torch.cuda.synchronize()
    for k, t in enumerate(tiles):
        _, r, Q, cnt = oracle_chain(orc, t, w[k].ravel())
        assert np.array_equal(rr.get_receivers(k).ravel(), r)
        assert np.array_equal(rr.get_counts(k).ravel(), cnt)
        assert np.array_equal(bits(rr.get_Q(k)), bits(Q))


@pytest.mark.gpu
def test_ragged_matches_flowrouter(cuda):
    """The batch equals the single-grid FlowRouter path run tile by tile."""
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = synthetic.ragged_tiles(ntiles=6, seed=21, side_min=100, side_max=400, max_pits=80)
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], 30.0, [t["mode"] for t in tiles])
    rr.set_z([t["z"] for t in tiles])
    rr.seed_constant(1.0, area=True)
    rr.route()
    for k, t in enumerate(tiles):
        fr = pf.flow.FlowRouter(t["nx"], t["ny"], 30.0, boundary_mode=t["mode"])
        fr.set_z(t["z"])
        fr.compute_receivers()
        fr.reroute_flow()
        fr.accumulate_constant_Q(1.0, area=True, exact_order=True)  # the batch keeps the reference's order
        torch.cuda.synchronize()
        assert np.array_equal(rr.get_receivers(k).ravel(), fr.get_receivers().ravel())
        assert np.array_equal(rr.get_counts(k), fr.get_counts())
        assert np.array_equal(bits(rr.get_Q(k)), bits(fr.get_Q()))


@pytest.mark.gpu
def test_ragged_graphflood_bit_exact_vs_oracle(orc, cuda):
    """GraphFlood on every tile in one launch equals the reference iteration
    (oracle, f32) run on each tile alone, with per-tile rainfall and Manning n."""
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = synthetic.ragged_tiles(ntiles=6, seed=31, side_min=24, side_max=72, max_pits=8, dx=10.0)
    tiles[2]["mode"] = "periodic_NS"
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], 10.0, [t["mode"] for t in tiles])
    rr.set_z([t["z"] for t in tiles])
    P = [1e-5 * (1 + k) for k in range(len(tiles))]
    n = [0.02 + 0.008 * k for k in range(len(tiles))]
    fl = pf.graphflood.RaggedFlooder(rr, precipitation_rates=P, manning=n)
    niter = 40
    it, res, tr = fl.run(niter, stop=None, trace=True)
    torch.cuda.synchronize()
    assert (it == niter).all()
    for k, t in enumerate(tiles):
        g = orc.Grid(t["nx"], t["ny"], MODES[t["mode"]])
        zh = t["z"].ravel().copy()
        h = np.zeros_like(zh)
        Q = np.zeros_like(zh)
        otr = orc.graphflood_run(zh, h, Q, g, 10.0, P[k], manning=n[k], niter=niter)
        o, N = int(rr.offset[k]), rr.cells(k)
        assert np.array_equal(bits(fl.get_h(k)), bits(h)), f"tile {k} h"
        assert np.array_equal(bits(rr.z[o:o + N].cpu().numpy()), bits(zh)), f"tile {k} z"
        assert np.array_equal(bits(rr.Q[o:o + N].cpu().numpy()), bits(Q)), f"tile {k} Q"
        assert np.array_equal(bits(tr[k, :, 0]), bits(otr)), f"tile {k} residual trace"


@pytest.mark.gpu
def test_ragged_graphflood_stops_per_tile(cuda):
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = synthetic.ragged_tiles(ntiles=4, seed=32, side_min=24, side_max=48, max_pits=3, dx=10.0)
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], 10.0, [t["mode"] for t in tiles])
    rr.set_z([t["z"] for t in tiles])
    fl = pf.graphflood.RaggedFlooder(rr, precipitation_rates=1e-5)
    it, res, tr = fl.run(300, stop="mean", tol_ratio=1e4, trace=True)
    for k in range(len(tiles)):
        n = int(it[k])
        assert 1 <= n <= 300
        if n < 300:  # stopped on its own criterion, at the first iteration below the threshold
            thr = np.float32(1e4 * 1e-5 * 5e-3)
            assert tr[k, n - 1, 1] < thr and (tr[k, :n - 1, 1] >= thr).all()
        assert bits(res[k, 0]) == bits(tr[k, n - 1, 0])  # (a tile whose h went NaN never stops early)


def custom_codes(nx, ny, seed):
    """Boundary codes of a custom-mode tile: outlets (3) on the south row and a few
    interior outlet cells, nodata (0) holes, periodic (9) west/east columns, inlets (7),
    normal (1) elsewhere (pyfastflow/constants.py:56-83)."""
    rng = np.random.default_rng(seed)
    c = np.ones((ny, nx), np.uint8)
    c[-1, :] = 3
    c[:, 0] = 9
    c[:, -1] = 9
    c[-1, 0] = c[-1, -1] = 3
    c[rng.integers(1, ny - 1, 4), rng.integers(1, nx - 1, 4)] = 0
    c[rng.integers(1, ny - 1, 2), rng.integers(1, nx - 1, 2)] = 3
    c[0, rng.integers(1, nx - 1, 3)] = 7
    return c


@pytest.mark.gpu
def test_ragged_custom_codes_bit_exact(orc, cuda):
    """Custom-mode tiles (codes 0/1/3/7/9) mixed with the other modes, routed and
    flooded in one launch each, equal the oracle tile by tile."""
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = synthetic.ragged_tiles(ntiles=6, seed=41, side_min=24, side_max=96, max_pits=10, dx=10.0)
    codes = [None] * len(tiles)
    for k in (1, 3, 4):
        tiles[k]["mode"] = "custom"
        codes[k] = custom_codes(tiles[k]["nx"], tiles[k]["ny"], 100 + k)
    modes = [t["mode"] for t in tiles]
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], 10.0, modes, codes=codes)
    rr.set_z([t["z"] for t in tiles])
    rr.seed_constant(1.0, area=True)
    rr.route()
    torch.cuda.synchronize()
    code_of = {"normal": 0, "periodic_EW": 1, "periodic_NS": 2, "custom": 3}
    for k, t in enumerate(tiles):
        g = orc.Grid(t["nx"], t["ny"], code_of[t["mode"]], codes[k].ravel() if codes[k] is not None else None)
        rcv, grad = orc.compute_receivers(t["z"], g, t["dx"])
        r, _, _, _, _ = orc.reroute_flow(rcv, t["z"], g, carve=True)
        Q, cnt = orc.accumulate(r, np.float32(t["dx"] * t["dx"]))
        assert np.array_equal(rr.get_receivers(k).ravel(), r), f"tile {k} receivers"
        assert np.array_equal(rr.get_counts(k).ravel(), cnt), f"tile {k} counts"
        assert np.array_equal(bits(rr.get_Q(k)), bits(Q)), f"tile {k} Q"
    # GraphFlood on the same batch
    rr.set_z([t["z"] for t in tiles])
    rr.Q.zero_()
    fl = pf.graphflood.RaggedFlooder(rr, precipitation_rates=2e-5, manning=0.04)
    fl.run(25, stop=None)
    torch.cuda.synchronize()
    for k, t in enumerate(tiles):
        g = orc.Grid(t["nx"], t["ny"], code_of[t["mode"]], codes[k].ravel() if codes[k] is not None else None)
        zh = t["z"].ravel().copy()
        h = np.zeros_like(zh)
        Q = np.zeros_like(zh)
        orc.graphflood_run(zh, h, Q, g, 10.0, 2e-5, manning=0.04, niter=25)
        assert np.array_equal(bits(fl.get_h(k)), bits(h)), f"tile {k} h"
        assert np.array_equal(bits(rr.Q[int(rr.offset[k]):int(rr.offset[k]) + rr.cells(k)].cpu().numpy()), bits(Q))


@pytest.mark.gpu
def test_ragged_config4_slice_bit_exact(orc, cuda):
    """The first 48 tiles of the benchmark's ragged batch (512 tiles, sides
    log-uniform in [128, 1024], 0-200 pits, normal / periodic east-west, seed 4)
    routed in one launch, bit-exact per tile against the oracle."""
    torch = cuda
    import pyfastflow_b200 as pf

    tiles = synthetic.ragged_tiles(ntiles=48, seed=4)
    sides = np.array([[t["nx"], t["ny"]] for t in tiles])
    assert sides.min() >= 128 and sides.max() <= 1024 and len({t["mode"] for t in tiles}) == 2
    rr = pf.flow.RaggedRouter([(t["ny"], t["nx"]) for t in tiles], 30.0, [t["mode"] for t in tiles])
    rr.set_z([t["z"] for t in tiles])
    rr.seed_constant(1.0, area=True)
    rr.route(graph=True)
    torch.cuda.synchronize()
    seed = np.float32(900.0)
    for k, t in enumerate(tiles):
        _, r, Q, cnt = oracle_chain(orc, t, seed)
        assert np.array_equal(rr.get_receivers(k).ravel(), r), f"tile {k} receivers"
        assert np.array_equal(rr.get_counts(k).ravel(), cnt), f"tile {k} counts"
        assert np.array_equal(bits(rr.get_Q(k)), bits(Q)), f"tile {k} Q"
