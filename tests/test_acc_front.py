"""The accumulation's tile front (the first rounds of the rake-and-compress run
per spatial tile in shared memory) against the oracle and against the plain
round-by-round path: f32 discharge and uint32 counts bit for bit, for boundary
modes 0-2, grid shapes smaller than, equal to and straddling the tile, receivers
from DEMs with ties and carve rerouting, a boustrophedon chain through every cell,
and non-neighbour receivers (the front hands over to the scatter path)."""
import numpy as np
import pytest

from pyfastflow_b200 import synthetic

DEFAULT = 3  # the library's default number of front rounds


def test_front_switch_host_checks():
    from pyfastflow_b200 import _lib

    lib = _lib.load()
    assert lib.pff_accumulate_set_front(4) != 0
    assert lib.pff_accumulate_set_front(-1) != 0
    for r in (0, 1, 2, 3):
        assert lib.pff_accumulate_set_front(r) == 0
    lib.pff_accumulate_set_front(DEFAULT)


def boustrophedon(nx, ny):
    """Receivers of one path through every cell, row by row, alternating direction;
    the last cell is the only root."""
    order = np.arange(nx * ny).reshape(ny, nx)
    order[1::2] = order[1::2, ::-1]
    path = order.ravel()
    rcv = np.empty(nx * ny, np.int32)
    rcv[path[:-1]] = path[1:]
    rcv[path[-1]] = path[-1]
    return rcv


def _run(torch, rcv, w, nx, ny, mode, front):
    from pyfastflow_b200 import _dev, _lib

    lib = _lib.load()
    N = nx * ny
    Qd = torch.from_numpy(w.copy()).cuda()
    cd = torch.zeros(N, dtype=torch.int32, device="cuda")
    ws = torch.empty(lib.pff_accumulate_workspace_bytes(N), dtype=torch.uint8, device="cuda")
    assert lib.pff_accumulate_set_front(front) == 0
    rd = torch.from_numpy(rcv).cuda()  # held until the kernels have run
    try:
        _lib.call("pff_accumulate_grid", rd.data_ptr(), Qd.data_ptr(), cd.data_ptr(), nx,
                  ny, mode, None, N, ws.data_ptr(), ws.numel(), _dev.stream())
    finally:
        lib.pff_accumulate_set_front(DEFAULT)
    return Qd.cpu().numpy(), cd.cpu().numpy().view(np.uint32)


SHAPES = [(3, 3), (5, 300), (300, 5), (64, 24), (64, 16), (130, 49), (257, 131)]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("nx,ny", SHAPES)
def test_front_matches_oracle(orc, cuda, mode, nx, ny):
    torch = cuda
    N = nx * ny
    rng = np.random.default_rng(nx * 1000 + ny + mode)
    g = orc.Grid(nx, ny, mode)
    cases = []
    z = rng.integers(0, 12, (ny, nx)).astype(np.float32)  # ties, flats and many pits
    r0, _ = orc.compute_receivers(z, g, 10.0)
    cases.append(r0)
    cases.append(orc.reroute_flow(r0, z, g, carve=True)[0])
    if nx >= 8 and ny >= 8:
        zs = synthetic.spectral_dem(nx, ny, 7, relief=200.0, npits=max(1, N // 500), pit_scale=0.05)
        rs, _ = orc.compute_receivers(zs, g, 10.0)
        cases.append(orc.reroute_flow(rs, zs, g, carve=True)[0])
    cases.append(boustrophedon(nx, ny))
    for rcv in cases:
        w = rng.lognormal(0, 0.5, N).astype(np.float32)
        Qo, co = orc.accumulate(rcv, w)
        for front in (0, 1, 2, 3):
            Q, c = _run(torch, rcv, w, nx, ny, mode, front)
            assert np.array_equal(c, co), f"counts, front {front}"
            assert np.array_equal(Q.view(np.uint32), Qo.view(np.uint32)), f"Q, front {front}"


@pytest.mark.gpu
@pytest.mark.parametrize("front", [1, 2, 3])
def test_front_hands_over_nonlocal_receivers(orc, cuda, front):
    """A forest whose links are not grid neighbours: the front flags it and the
    scatter path computes everything, bit-exact."""
    torch = cuda
    rng = np.random.default_rng(5)
    nx, ny = 150, 120
    N = nx * ny
    rcv = np.arange(N, dtype=np.int32)
    nchild = np.zeros(N, np.int32)
    for i in range(1, N):
        if rng.random() < 0.03:
            continue
        p = int(rng.integers(max(0, i - 5000), i))
        if nchild[p] < 4:
            rcv[i] = p
            nchild[p] += 1
    w = rng.lognormal(0, 0.5, N).astype(np.float32)
    Qo, co = orc.accumulate(rcv, w)
    Q, c = _run(torch, rcv, w, nx, ny, 1, front)
    assert np.array_equal(c, co)
    assert np.array_equal(Q.view(np.uint32), Qo.view(np.uint32))
