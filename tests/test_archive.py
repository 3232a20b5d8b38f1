"""Legacy downstream tree algorithms (archive/fastflow/kernels): the oracle on
hand-derived cases, and the sm_100a kernels bit for bit against the oracle on
rerouted DEM receivers (and on forests whose nodes have more than 4 donors)."""
import numpy as np
import pytest

from pyfastflow_b200 import synthetic


def chain():
    # 3 -> 2 -> 1 -> 0 (root)
    return np.array([0, 0, 1, 2], np.int32)


def test_oracle_tree_accum_down_chain(orc):
    rcv, W, p = orc.tree_accum_down(chain(), np.array([0, .5, .5, .5], np.float32), np.ones(4, np.float32))
    # x = p + W * x[rcv]: 1, 1.5, 1.75, 1.875 (exact in binary)
    assert p.tolist() == [1.0, 1.5, 1.75, 1.875]
    assert rcv.tolist() == [0, 0, 0, 0]


def test_oracle_tree_max_down_excludes_root(orc):
    _, p = orc.tree_max_down(chain(), np.array([5, 1, 3, 2], np.float32))
    # the maximum over each path below the cell, the final root's value excluded
    assert p.tolist() == [5.0, 1.0, 3.0, 3.0]


def test_oracle_erode_deposit_boundary_and_solve(orc):
    # boundary cells keep their (deposited-free) elevation and weight 0
    z = np.array([10, 11, 12, 13], np.float32)
    bound = np.array([1, 0, 0, 0], np.uint8)
    drain = np.array([4, 3, 2, 1], np.float32)
    Qs = np.zeros(4, np.float32)
    z2, pe, We = orc.erode_deposit(z, bound, chain(), drain, Qs, 1.0, 1.0, 0.5, 0.0, 0.0, 1.0, 0.5)
    assert pe[0] == 10.0 and We[0] == 0.0
    # the solve is x = z/(1+K) + K/(1+K) * x[rcv] (implicit erosion), step by step
    K = np.float32(1.0) * (np.float32(0.5) * np.float32(np.sqrt(np.float64(3.0))))
    x1 = np.float32(np.float32(11) / (1 + K)) + np.float32(K / (1 + K)) * np.float32(10)
    assert abs(pe[1] - x1) < 1e-5


def dem_forest(orc, nx, ny, seed, mode=0):
    g = orc.Grid(nx, ny, mode)
    z = synthetic.spectral_dem(nx, ny, seed, relief=300.0, npits=max(1, nx * ny // 2000), pit_scale=0.1)
    rcv, _ = orc.compute_receivers(z, g, 10.0)
    r2, _, _, _, _ = orc.reroute_flow(rcv, z, g)
    return z.ravel(), r2


@pytest.mark.gpu
def test_tree_accum_and_max_down_bit_exact(orc, cuda):
    torch = cuda
    import pyfastflow_b200 as pf

    for shape in [(211, 173), (64, 64), (17, 3)]:
        nx, ny = shape
        z, rcv = dem_forest(orc, nx, ny, 3)
        rng = np.random.default_rng(5)
        W = (rng.random(rcv.size) * 0.9).astype(np.float32)
        W[rcv == np.arange(rcv.size)] = 0.0
        p = rng.lognormal(0, 0.5, rcv.size).astype(np.float32)
        r_o, W_o, p_o = orc.tree_accum_down(rcv, W, p)
        rd, Wd, pd = (torch.from_numpy(a.copy()).cuda() for a in (rcv, W, p))
        pf.archive.tree_accum_downward(rd, Wd, pd)
        assert np.array_equal(pd.cpu().numpy().view(np.uint32), p_o.view(np.uint32))
        assert np.array_equal(Wd.cpu().numpy().view(np.uint32), W_o.view(np.uint32))
        assert np.array_equal(rd.cpu().numpy(), r_o)
        r_m, p_m = orc.tree_max_down(rcv, z)
        rd, pd = (torch.from_numpy(a.copy()).cuda() for a in (rcv, z.astype(np.float32)))
        pf.archive.tree_max_downward(rd, pd)
        assert np.array_equal(pd.cpu().numpy().view(np.uint32), p_m.view(np.uint32))
        assert np.array_equal(rd.cpu().numpy(), r_m)


@pytest.mark.gpu
def test_tree_accum_down_many_donors(orc, cuda):
    """A forest with nodes of 5-40 donors (the jump-rerouting shape) and a long chain."""
    torch = cuda
    import pyfastflow_b200 as pf

    rng = np.random.default_rng(8)
    N = 20000
    rcv = np.arange(N, dtype=np.int32)
    for i in range(1, N):
        rcv[i] = int(rng.integers(max(0, i - 60), i)) if rng.random() < 0.97 else i
    rcv[5000:5100] = np.arange(4999, 5099)  # a chain
    W = (rng.random(N) * 0.5).astype(np.float32)
    W[rcv == np.arange(N)] = 0.0
    p = rng.random(N).astype(np.float32)
    assert np.bincount(rcv[rcv != np.arange(N)]).max() > 4
    _, _, p_o = orc.tree_accum_down(rcv, W, p)
    rd, Wd, pd = (torch.from_numpy(a.copy()).cuda() for a in (rcv, W, p))
    pf.archive.tree_accum_downward(rd, Wd, pd)
    assert np.array_equal(pd.cpu().numpy().view(np.uint32), p_o.view(np.uint32))


@pytest.mark.gpu
def test_erode_deposit_bit_exact(orc, cuda):
    torch = cuda
    import pyfastflow_b200 as pf

    nx, ny = 160, 120
    z, rcv = dem_forest(orc, nx, ny, 11)
    N = nx * ny
    cnt = orc.topo_accumulate(rcv).astype(np.float32) * np.float32(100.0)
    bound = np.zeros((ny, nx), np.uint8)
    bound[0, :] = bound[-1, :] = bound[:, 0] = bound[:, -1] = 1
    bound = bound.ravel()
    Qs = np.random.default_rng(3).random(N).astype(np.float32) * 0.01
    args = (1e3, 10.0, 2e-5, 1e-6, 3e-6, 5.0, 0.45)
    z_o, pe_o, We_o = orc.erode_deposit(z, bound, rcv, cnt, Qs, *args)
    zd, bd, rd, dd, qd = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (z.copy(), bound, rcv.copy(),
                                                                                    cnt, Qs))
    pe = pf.archive.erode_deposit(zd, bd, rd, dd, qd, *args)
    assert np.array_equal(zd.cpu().numpy().view(np.uint32), z_o.view(np.uint32))
    assert np.array_equal(pe.cpu().numpy().view(np.uint32), pe_o.view(np.uint32))
