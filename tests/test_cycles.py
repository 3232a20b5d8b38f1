"""Receiver cycles: carving can close a cycle of basins whose saddles tie (the
reference removes only 2-cycles, flow/lakeflow.py:255-281), so the rerouted
receivers hold a cycle.  The reference's serial labelling and last-writer
reversal resolve it (or not) in later outer iterations; the kernels must do
exactly the same.  Inputs: tests/golden/cycle_crops.npz (see make_cycle_fixtures.py)."""
import os

import numpy as np
import pytest

from pyfastflow_b200 import synthetic

HERE = os.path.dirname(os.path.abspath(__file__))


def crops():
    return np.load(os.path.join(HERE, "golden", "cycle_crops.npz"))


def first_carve(orc, rec, z, g):
    """One carve of the reference on `rec` (lakeflow.py:405-438), serial order."""
    N = g.N
    bid = orc.basin_labels(rec, g)
    st = orc.saddlesort(bid, z, g)
    inv = orc.pack_float_index(1e8, 42)
    sn = st.basin_saddlenode[:N]
    tag = np.zeros(N, bool)
    for x in sn[sn >= 0]:
        while True:
            tag[x] = True
            if rec[x] == x:
                break
            x = rec[x]
    new = rec.copy()
    for i in range(N):  # serial reversal: the last (largest) writer wins
        r = rec[i]
        if tag[r] and tag[i] and i != r:
            new[r] = i
    for b in np.nonzero(st.outlet[:N] != inv)[0]:
        new[sn[b]] = orc.unpack_float_index(int(st.outlet[b]))[1]
    return new


def test_oracle_cycle_cases(orc):
    c = crops()
    z32 = c["crop32"]
    g = orc.Grid(32, 32, 0)
    rcv, _ = orc.compute_receivers(z32, g, 10.0)
    assert orc.count_cycle_nodes(first_carve(orc, rcv, z32, g)) == 4  # a 3-basin cycle after the first carve
    r2, _, _, nd, nout = orc.reroute_flow(rcv, z32, g)
    assert orc.count_cycle_nodes(r2) == 0  # resolved by the later outer iterations
    z16 = c["crop16"]
    g16 = orc.Grid(16, 16, 0)
    r16, _ = orc.compute_receivers(z16, g16, 10.0)
    r16b, _, _, _, _ = orc.reroute_flow(r16, z16, g16)
    assert orc.count_cycle_nodes(r16b) == 4  # the outer loop ends with the cycle in place


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["crop16", "crop32"])
def test_gpu_reroute_with_cycles(orc, cuda, name):
    torch = cuda
    from pyfastflow_b200 import constants as cte
    from pyfastflow_b200 import flow

    z = crops()[name]
    n = z.shape[0]
    g = orc.Grid(n, n, 0)
    cte.NX, cte.NY, cte.DX, cte.BOUND_MODE, cte.boundaries = n, n, 10.0, 0, None
    rcv, _ = orc.compute_receivers(z, g, 10.0)
    r_o, r_o_, st, nd, nout = orc.reroute_flow(rcv, z, g)
    N = n * n
    T = lambda k, dt: torch.zeros(k, dtype=dt, device="cuda")  # noqa: E731
    rec = torch.from_numpy(rcv).cuda()
    rec_, rec__, bid = T(N, torch.int32), T(N, torch.int32), T(N, torch.int32)
    zp, isb = T(N, torch.float32), T(N, torch.uint8)
    out, sad, sn = T(N + 1, torch.int64), T(N + 1, torch.int64), T(N + 1, torch.int32)
    tag, tag_ = T(N, torch.uint8), T(N, torch.uint8)
    n_outer = flow.reroute_flow(bid, rec, rec_, rec__, torch.from_numpy(z.ravel()).cuda(), zp, isb, out, sad, sn, tag,
                                tag_, None, carve=True)
    assert n_outer == nout
    assert np.array_equal(rec.cpu().numpy(), r_o)
    assert np.array_equal(rec_.cpu().numpy(), r_o_)
    assert np.array_equal(sad.cpu().numpy()[:N], st.basin_saddle[:N])
    assert np.array_equal(out.cpu().numpy()[:N], st.outlet[:N])
    assert np.array_equal(sn.cpu().numpy()[:N], st.basin_saddlenode[:N])
    assert np.array_equal(tag.cpu().numpy(), st.tag)
    assert np.array_equal(zp.cpu().numpy().view(np.uint32), st.z_prime.view(np.uint32))
    # accumulation on (possibly cyclic) receivers: the same bounded rake-and-compress rounds
    from pyfastflow_b200 import _dev, _lib

    w = synthetic.lognormal_weights(N, 3)
    Qd = torch.from_numpy(w.copy()).cuda()
    cd = torch.zeros(N, dtype=torch.int32, device="cuda")
    ws = _dev.Scratch()
    wp, wn = ws.get(_lib.load().pff_accumulate_workspace_bytes(N))
    _lib.call("pff_accumulate_grid", rec.data_ptr(), Qd.data_ptr(), cd.data_ptr(), n, n, 0, None, N, wp, wn,
              _dev.stream())
    Qo, co = orc.accumulate(r_o, w)
    assert np.array_equal(cd.cpu().numpy().view(np.uint32), co)
    assert np.array_equal(Qd.cpu().numpy().view(np.uint32), Qo.view(np.uint32))


@pytest.mark.gpu
def test_graphflood_512_long_run_bit_exact(orc, cuda):
    """512 x 512 GraphFlood, 460 iterations: past the first carve that closes a
    receiver cycle (iteration 447), GPU and oracle stay bit-identical."""
    torch = cuda
    import pyfastflow_b200 as pf

    n, iters = 512, 460
    z = synthetic.graphflood_plain(n)["z"]
    router = pf.flow.FlowRouter(n, n, 10.0)
    router.set_z(z)
    fl = pf.graphflood.Flooder(router, precipitation_rates=1e-5, manning=0.033, edge_slope=1e-2)
    fl.run_graphflood(iters)
    torch.cuda.synchronize()
    g = orc.Grid(n, n, 0)
    zh, h, Q = z.ravel().copy(), np.zeros(n * n, np.float32), np.zeros(n * n, np.float32)
    orc.graphflood_run(zh, h, Q, g, 10.0, 1e-5, niter=iters)

    def bits(a):
        a = np.asarray(a, np.float32)
        b = a.view(np.uint32).copy()
        b[np.isnan(a)] = 0x7FC00000
        return b

    assert np.array_equal(bits(fl.get_h().ravel()), bits(h))
    assert np.array_equal(bits(router.get_Z().ravel()), bits(zh))
    assert np.array_equal(bits(router.get_Q().ravel()), bits(Q))
