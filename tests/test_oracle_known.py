"""Known-answer tests of the CPU oracle on hand-derived grids.

The reference ships no golden vectors for receivers, basins, rerouting or
accumulation, so these cases are derived by hand from the reference's rules
(pyfastflow/flow/neighbourer_flat.py, receivers.py, lakeflow.py,
downstream_propag.py) and pin the oracle before it is used as the checker."""
import numpy as np
import pytest

# 4 x 3 grid:  0 1 2 3 / 4 5 6 7 / 8 9 10 11
NB_EXPECT = {
    0: {0: [-1, -1, 1, 4], 5: [1, 4, 6, 9], 7: [3, 6, -1, 11], 11: [7, 10, -1, -1], 1: [-1, 0, 2, 5]},
    1: {0: [-1, 3, 1, 4], 5: [1, 4, 6, 9], 7: [3, 6, 4, 11], 11: [7, 10, 8, -1], 1: [-1, 0, 2, 5]},
    2: {0: [8, -1, 1, 4], 5: [1, 4, 6, 9], 7: [3, 6, -1, 11], 11: [7, 10, -1, 3], 1: [9, 0, 2, 5]},
}
LEAVE_EXPECT = {
    0: {0, 1, 2, 3, 4, 7, 8, 9, 10, 11},
    1: {0, 1, 2, 3, 8, 9, 10, 11},
    2: {0, 3, 4, 7, 8, 11},
}


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_neighbours_modes(orc, mode):
    g = orc.Grid(4, 3, mode)
    nb, lv = orc.neighbour_table(g)
    for i, exp in NB_EXPECT[mode].items():
        assert list(nb[i]) == exp, (mode, i)
    assert set(np.nonzero(lv)[0]) == LEAVE_EXPECT[mode]


def test_neighbours_custom(orc):
    codes = np.ones(12, np.uint8)
    codes[5] = 0   # nodata
    codes[11] = 3  # outlet
    codes[4] = 9   # periodic (left edge: wraps east-west)
    g = orc.Grid(4, 3, 3, codes)
    nb, lv = orc.neighbour_table(g)
    assert list(nb[4]) == [0, 7, -1, 8]      # right neighbour 5 is nodata
    assert list(nb[6]) == [2, -1, 7, 10]     # left neighbour 5 is nodata
    assert list(nb[7]) == [3, 6, -1, 11]     # code 1 on the right edge: no wrap
    assert list(nb[5]) == [-1, -1, -1, -1]   # nodata cell has no links
    assert set(np.nonzero(lv)[0]) == {11}


def test_receivers_ties_first_direction(orc):
    # centre 10, top 9, left 9, right 8, bottom 8: drops 1,1,2,2 -> right (k=2) wins the tie
    z = np.full((3, 3), 20, np.float32)
    z[1, 1], z[0, 1], z[1, 0], z[1, 2], z[2, 1] = 10, 9, 9, 8, 8
    g = orc.Grid(3, 3, 0)
    rcv, grad = orc.compute_receivers(z, g, 1.0)
    assert rcv[4] == 5 and grad[4] == np.float32(2.0)
    # on a flat every cell drains to itself with gradient 0
    rf, gf = orc.compute_receivers(np.full((3, 3), 7, np.float32), g, 1.0)
    assert np.array_equal(rf, np.arange(9)) and not gf.any()


def test_receivers_division_ties(orc):
    # Two drops da > db (adjacent floats) whose quotients by dx round to the same
    # f32: the strict '>' keeps the earlier direction.  This holds only with an
    # IEEE division; a multiply by 1/dx can break the tie the other way.
    dx = np.float32(3.0)
    da = np.float32(1.5) + np.arange(1, 4096, dtype=np.float32) * np.float32(2 ** -23)
    db = np.nextafter(da, np.float32(0))
    tie = (da / dx == db / dx)
    assert tie.any()
    da, db = da[tie][0], db[tie][0]
    z = np.full((3, 3), 50, np.float32)
    z[1, 1] = 0.0
    z[0, 1] = -db  # k=0 (top): smaller drop
    z[2, 1] = -da  # k=3 (bottom): larger drop, equal after division
    g = orc.Grid(3, 3, 0)
    rcv, grad = orc.compute_receivers(z, g, float(dx))
    assert rcv[4] == 1 and grad[4] == db / dx


def _single_pit():
    z = np.array([[9, 9, 9, 9, 9],
                  [9, 5, 4, 5, 9],
                  [9, 4, 1, 3, 2],
                  [9, 5, 4, 5, 9],
                  [9, 9, 9, 9, 9]], np.float32)
    return z


def test_single_pit_reroute(orc):
    z = _single_pit()
    g = orc.Grid(5, 5, 0)
    rcv, _ = orc.compute_receivers(z, g, 1.0)
    exp = {6: 7, 7: 12, 8: 13, 11: 12, 12: 12, 13: 12, 16: 11, 17: 12, 18: 13, 1: 6, 9: 14, 19: 14, 14: 14, 0: 0}
    for i, r in exp.items():
        assert rcv[i] == r, (i, rcv[i], r)
    assert orc.depression_counter(rcv, g) == 1
    bid = orc.basin_labels(rcv, g)
    assert bid[12] == 13 and bid[1] == 13 and bid[23] == 13 and bid[9] == 0 and bid[0] == 0
    r2, _, st, nd, nout = orc.reroute_flow(rcv, z, g, carve=True)
    assert nd == 1 and nout == 1
    assert orc.unpack_float_index(int(st.basin_saddle[13])) == (np.float32(3.0), 0)
    assert st.basin_saddlenode[13] == 13
    assert orc.unpack_float_index(int(st.outlet[13])) == (np.float32(2.0), 14)
    changed = {i: (rcv[i], r2[i]) for i in range(25) if rcv[i] != r2[i]}
    assert changed == {12: (12, 13), 13: (12, 14)}
    cnt = orc.topo_accumulate(r2)
    assert cnt[14] == 21 and cnt[13] == 18
    Q, c2 = orc.accumulate(r2, 1.0)
    assert np.array_equal(c2, cnt) and np.array_equal(Q, cnt.astype(np.float32))


def test_two_cycle_and_merge(orc):
    # 7 x 3 grid, high rim: three pits (cells 8, 10, 12); basins 9 and 11 point at
    # each other (2-cycle) and pass 5 invalidates the larger id (11)
    z = np.full((3, 7), 100, np.float32)
    z[1, 1:6] = [1, 5, 3, 6, 2]
    g = orc.Grid(7, 3, 0)
    rcv, _ = orc.compute_receivers(z, g, 1.0)
    assert [rcv[i] for i in (8, 9, 10, 11, 12)] == [8, 8, 10, 12, 12]
    bid = orc.basin_labels(rcv, g)
    assert bid[9] == 9 and bid[3] == 11 and bid[13] == 13 and bid[6] == 0
    st = orc.saddlesort(bid, z, g)
    assert orc.unpack_float_index(int(st.basin_saddle[9])) == (np.float32(5), 11)
    assert orc.unpack_float_index(int(st.basin_saddle[13])) == (np.float32(6), 11)
    assert st.basin_saddlenode[9] == 9 and st.basin_saddlenode[13] == 11
    assert st.basin_saddlenode[11] == -1  # invalidated by the 2-cycle pass
    assert st.outlet[11] == orc.pack_float_index(1e8, 42)
    assert orc.unpack_float_index(int(st.outlet[9])) == (np.float32(3), 10)
    r2, _, st2, nd, nout = orc.reroute_flow(rcv, z, g, carve=True)
    assert nd == 3 and nout == 3
    assert [r2[i] for i in (8, 9, 10, 11, 12)] == [9, 10, 10, 10, 11]
    assert orc.depression_counter(r2, g) == 1  # closed domain: one pit remains
    assert orc.topo_accumulate(r2)[10] == 17


@pytest.mark.parametrize("n", [1023, 4096])
def test_chain_accumulation(orc, n):
    rcv = np.arange(-1, n - 1, dtype=np.int32)
    rcv[0] = 0
    Q, cnt = orc.accumulate(rcv, 1.0)
    assert np.array_equal(cnt, np.arange(n, 0, -1, dtype=np.uint32))
    assert np.array_equal(Q, cnt.astype(np.float32))


def test_random_forest_counts_match_topological(orc):
    rng = np.random.default_rng(5)
    for mode in (0, 1, 2):
        z = rng.integers(0, 40, (37, 53)).astype(np.float32)  # many ties and flats
        g = orc.Grid(53, 37, mode)
        rcv, _ = orc.compute_receivers(z, g, 2.0)
        r2, _, _, _, _ = orc.reroute_flow(rcv, z, g, carve=True)
        assert orc.count_cycle_nodes(r2) == 0
        Q, cnt = orc.accumulate(r2, 1.0)
        assert np.array_equal(cnt, orc.topo_accumulate(r2))


def test_weighted_accumulation_close_to_exact(orc):
    rng = np.random.default_rng(9)
    z = rng.random((64, 64)).astype(np.float32)
    g = orc.Grid(64, 64, 0)
    rcv, _ = orc.compute_receivers(z, g, 1.0)
    w = rng.lognormal(0, 0.5, 64 * 64).astype(np.float32)
    Q, _ = orc.accumulate(rcv, w)
    # exact sums by topological order in float64
    exact = w.astype(np.float64).copy()
    indeg = np.zeros(rcv.size, np.int64)
    for i, r in enumerate(rcv):
        if r != i:
            indeg[r] += 1
    q = [i for i in range(rcv.size) if indeg[i] == 0]
    while q:
        i = q.pop()
        r = rcv[i]
        if r == i:
            continue
        exact[r] += exact[i]
        indeg[r] -= 1
        if indeg[r] == 0:
            q.append(r)
    rel = np.abs(Q - exact) / exact
    assert rel.max() < 1e-5
