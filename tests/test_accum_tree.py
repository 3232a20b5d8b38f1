"""Hierarchical tile accumulation (pff_accumulate_tree) through the C ABI.

Counts are bit-exact against the oracle's rake-and-compress counts and an
independent Kahn topological count; Q is the exact upstream sum rounded once to
f32, so it is checked against an f64 topological sum (to f32 rounding) and
against the oracle's f32 rake-and-compress sums within the tolerance that bounds
their rounding (1e-5 mean, 1e-4 max relative)."""
import ctypes as C

import numpy as np
import pytest

from pyfastflow_b200 import synthetic

pytestmark = pytest.mark.gpu


def exact_f64(rcv, seed):
    """Upstream sums in f64, in topological order (leaves first)."""
    rcv = np.asarray(rcv, np.int64)
    N = rcv.size
    indeg = np.bincount(rcv[rcv != np.arange(N)], minlength=N)
    q = np.asarray(seed, np.float64).copy()
    front = np.nonzero(indeg == 0)[0]
    while front.size:
        r = rcv[front]
        mv = r != front
        src, dst = front[mv], r[mv]
        np.add.at(q, dst, q[src])
        np.subtract.at(indeg, dst, 1)
        nxt = np.unique(dst)
        front = nxt[indeg[nxt] == 0]
    return q


def run_tree(torch, rcv, nx, ny, weights=None, value=1.0, local=1, repeat_equal=True):
    from pyfastflow_b200 import _dev, _lib

    lib = _lib.load()
    N = nx * ny
    r = torch.from_numpy(np.ascontiguousarray(rcv, np.int32)).cuda()
    Q = torch.empty(N, dtype=torch.float32, device="cuda")
    cnt = torch.empty(N, dtype=torch.int32, device="cuda")
    wd = torch.from_numpy(np.ascontiguousarray(weights, np.float32)).cuda() if weights is not None else None
    nb = lib.pff_accumulate_tree_workspace_bytes(nx, ny, local)
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    st = _dev.stream()
    out = []
    for _ in range(2):  # twice on the same workspace: results must not depend on its previous contents
        rc = lib.pff_accumulate_tree(r.data_ptr(), wd.data_ptr() if wd is not None else None, value, Q.data_ptr(),
                                     cnt.data_ptr(), nx, ny, local, ws.data_ptr(), nb, st)
        assert rc == 0, lib.pff_last_error_string()
        status = C.c_int()
        assert lib.pff_accumulate_tree_status(nx, ny, local, ws.data_ptr(), nb, C.byref(status), st) == 0
        out.append((Q.cpu().numpy().copy(), cnt.cpu().numpy().view(np.uint32).copy(), status.value))
    if repeat_equal:  # (a call whose status reports a problem promises nothing)
        assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
        assert np.array_equal(out[0][1], out[1][1]) and out[0][2] == out[1][2]
    return out[1]


def check(orc, rcv, Q, cnt, seed):
    want_c = orc.topo_accumulate(rcv)
    assert np.array_equal(cnt, want_c)
    ex = exact_f64(rcv, seed)
    assert np.array_equal(Q, ex.astype(np.float32)) or np.max(np.abs(Q - ex) / np.abs(ex)) < 2 ** -23
    Qo, co = orc.accumulate(rcv, np.asarray(seed, np.float32))
    assert np.array_equal(cnt, co)
    rel = np.abs(Q.astype(np.float64) - Qo) / np.abs(Qo)
    assert rel.mean() < 1e-5 and rel.max() < 1e-4, (rel.mean(), rel.max())


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("shape", [(211, 173), (64, 64), (1000, 37), (9, 7), (33, 300)])
def test_tree_matches_oracle_rerouted(orc, cuda, mode, shape):
    nx, ny = shape
    from test_gpu_parity import random_codes

    codes = random_codes(nx, ny, 3) if mode == 3 else None
    g = orc.Grid(nx, ny, mode, codes)
    z = synthetic.spectral_dem(nx, ny, 5 + mode, relief=300.0, npits=max(1, nx * ny // 3000), pit_scale=0.1)
    rcv, _ = orc.compute_receivers(z, g, 10.0)
    rcv, _, _, _, _ = orc.reroute_flow(rcv, z, g)
    w = np.random.default_rng(1).lognormal(0, 0.5, nx * ny).astype(np.float32)
    Q, cnt, status = run_tree(cuda, rcv, nx, ny, weights=w)
    assert status == 0
    check(orc, rcv, Q, cnt, w)
    # constant seed (drainage area): Q = count * dx^2, rounded once
    Qa, ca, st2 = run_tree(cuda, rcv, nx, ny, value=900.0)
    assert st2 == 0 and np.array_equal(ca, cnt)
    assert np.array_equal(Qa, (cnt.astype(np.float64) * 900.0).astype(np.float32))


def test_tree_raw_receivers_many_roots(orc, cuda):
    """Unrerouted receivers (every pit a root), plain 512^2 routing config."""
    cfg = synthetic.routing_plain_512()
    g = orc.Grid(512, 512, 0)
    rcv, _ = orc.compute_receivers(cfg["z"], g, 30.0)
    Q, cnt, status = run_tree(cuda, rcv, 512, 512, value=900.0)
    assert status == 0
    assert np.array_equal(cnt, orc.topo_accumulate(rcv))
    assert np.array_equal(Q, (cnt.astype(np.float64) * 900.0).astype(np.float32))


def test_tree_jump_rerouting_more_than_four_donors(orc, cuda):
    """Jump rerouting (lakeflow.py:285-304) sends pits straight to their outlet
    nodes, so receivers stop being D4 neighbours and a node can gain more than 4
    donors, which overflows the reference's 4-slot donor array
    (downstream_propag.py:90-96).  The tree accumulation takes any in-degree
    (local = 0): counts equal the exact topological counts.  On top of a real
    jump-rerouted DEM, 16 donorless cells are sent to one node (the shape of
    many pits jumping to one outlet node), giving that node 16+ donors."""
    nx, ny = 300, 260
    g = orc.Grid(nx, ny, 0)
    z = synthetic.spectral_dem(nx, ny, 9, relief=200.0, npits=400, pit_scale=0.15)
    rcv, _ = orc.compute_receivers(z, g, 10.0)
    _, rj, _, _, _ = orc.reroute_flow(rcv, z, g, carve=False)  # the reference leaves the result in rec_
    rng = np.random.default_rng(3)
    idx = np.arange(rj.size)
    jumps = np.abs(idx // nx - rj // nx) + np.abs(idx % nx - rj % nx) > 1
    assert jumps.any()  # the jump rerouting made non-neighbour receivers
    indeg = np.bincount(rj[rj != idx], minlength=rj.size)
    target = int(rj[np.nonzero(jumps)[0][0]])  # an outlet node some pit jumped to
    leaves = np.nonzero((indeg == 0) & (rj != idx))[0]
    leaves = leaves[np.abs(leaves - target) > 2 * nx]
    rj = rj.copy()
    rj[rng.choice(leaves, 16, replace=False)] = target  # donorless cells: no cycle can form
    indeg = np.bincount(rj[rj != idx], minlength=rj.size)
    assert indeg.max() > 4  # the case the reference's donor slots cannot hold
    w = np.random.default_rng(2).lognormal(0, 0.5, nx * ny).astype(np.float32)
    Q, cnt, status = run_tree(cuda, rj, nx, ny, weights=w, local=0)
    assert status == 0
    assert np.array_equal(cnt, orc.topo_accumulate(rj))
    ex = exact_f64(rj, w)
    assert np.max(np.abs(Q - ex) / np.abs(ex)) < 2 ** -23
    # with local = 1 the non-neighbour receivers are reported, not silently mis-summed
    _, _, st1 = run_tree(cuda, rj, nx, ny, weights=w, local=1, repeat_equal=False)
    assert st1 & 8


def test_tree_reports_cycle_and_bad_receiver(orc, cuda):
    nx, ny = 100, 90
    N = nx * ny
    rcv = np.arange(N, dtype=np.int32)
    rcv[5] = 6
    rcv[6] = 106
    rcv[106] = 105
    rcv[105] = 5  # a 4-cell cycle
    _, _, status = run_tree(cuda, rcv, nx, ny, value=1.0, repeat_equal=False)
    assert status & 2
    rcv2 = np.arange(N, dtype=np.int32)
    rcv2[7] = N + 5
    _, cnt, status2 = run_tree(cuda, rcv2, nx, ny, value=1.0, repeat_equal=False)
    assert status2 & 1
