"""Parity of the sm_100a kernels (through the C ABI) with the CPU oracle.

Bar: bit-exact for receivers, gradients, basin labels, saddle/outlet keys,
rerouted receivers, drainage counts, the f32 rake-and-compress discharge and
the GraphFlood update (fill, diffusion, Manning): the kernels perform the
oracle's IEEE operations in the oracle's order."""
import numpy as np
import pytest

from pyfastflow_b200 import synthetic

pytestmark = pytest.mark.gpu

MODES = [0, 1, 2, 3]


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def fbits(a):
    """f32 bit patterns with NaNs canonicalised (positions compared, payloads not)."""
    a = np.asarray(a, np.float32)
    b = a.view(np.uint32).copy()
    b[np.isnan(a)] = 0x7FC00000
    return b


def random_codes(nx, ny, seed):
    rng = np.random.default_rng(seed)
    c = np.ones((ny, nx), np.uint8)
    c[rng.random((ny, nx)) < 0.03] = 0   # nodata holes
    c[rng.random((ny, nx)) < 0.01] = 3   # interior outlets
    c[rng.random((ny, nx)) < 0.01] = 7   # inlets (behave as normal cells)
    edge = np.zeros((ny, nx), bool)
    edge[0, :] = edge[-1, :] = edge[:, 0] = edge[:, -1] = True
    pick = rng.choice([1, 3, 9, 0], size=(ny, nx), p=[0.3, 0.4, 0.25, 0.05])
    c[edge] = pick[edge]
    return c.ravel()


def make_case(kind, nx, ny, seed):
    rng = np.random.default_rng(seed)
    if kind == "int":
        z = rng.integers(0, 30, (ny, nx)).astype(np.float32)  # ties and flats
    elif kind == "spectral":
        z = synthetic.spectral_dem(nx, ny, seed, relief=300.0, npits=max(1, nx * ny // 2000), pit_scale=0.1)
    else:
        z = (rng.random((ny, nx)) * 100).astype(np.float32)
    return z


class Grid:
    def __init__(self, orc, torch, nx, ny, mode, seed=0):
        self.nx, self.ny, self.mode, self.N = nx, ny, mode, nx * ny
        self.codes_np = random_codes(nx, ny, seed) if mode == 3 else None
        self.og = orc.Grid(nx, ny, mode, self.codes_np)
        self.codes = dev(torch, self.codes_np) if mode == 3 else None

    @property
    def cptr(self):
        return self.codes.data_ptr() if self.codes is not None else None


def assert_q_close(Q, Qref):
    """Weighted discharge against the reference's f32 sums: 1e-5 mean, 1e-4 max
    relative error (the reference's own summation rounding is the difference)."""
    rel = np.abs(np.asarray(Q, np.float64) - Qref) / np.maximum(np.abs(Qref), 1e-30)
    assert rel.mean() < 1e-5 and rel.max() < 1e-4, (float(rel.mean()), float(rel.max()))


def set_constants(g, dx):
    from pyfastflow_b200 import constants as cte

    cte.NX, cte.NY, cte.DX, cte.BOUND_MODE = g.nx, g.ny, dx, g.mode
    cte.boundaries = g.codes


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("kind", ["int", "spectral", "uniform"])
def test_receivers(orc, cuda, mode, kind):
    torch = cuda
    from pyfastflow_b200 import flow

    for (nx, ny) in [(97, 61), (256, 256)]:
        g = Grid(orc, torch, nx, ny, mode, seed=nx)
        z = make_case(kind, nx, ny, seed=ny + mode)
        dx = 3.0 if kind != "int" else 30.0
        set_constants(g, dx)
        zd = dev(torch, z.ravel())
        r = torch.empty(g.N, dtype=torch.int32, device="cuda")
        gr = torch.empty(g.N, dtype=torch.float32, device="cuda")
        flow.compute_receivers(zd, r, gr)
        ro, go = orc.compute_receivers(z, g.og, dx)
        assert np.array_equal(host(r), ro)
        assert np.array_equal(fbits(host(gr)), fbits(go))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_receivers_lean_kernel_variants(orc, cuda, mode):
    """Both variants of the lean receivers kernel (7 and 8 CTAs per SM) and the
    earlier 4-column walk against the oracle: single- and
    partial-strip widths, one- and many-band heights, 2-row grids, integer ties,
    near ties (drops a few ulps apart), tiny and huge cell sizes."""
    torch = cuda
    from pyfastflow_b200 import _lib, flow

    lib = _lib.load()
    cases = [(4, 2, "int", 30.0), (8, 3, "uniform", 3.0), (516, 77, "int", 30.0), (1024, 130, "spectral", 3.0),
             (2048, 70, "uniform", 1e-30), (1536, 9, "int", 1e30), (256, 40, "near", 10.0), (132, 33, "near", 0.3)]
    try:
        for (nx, ny, kind, dx) in cases:
            g = Grid(orc, torch, nx, ny, mode, seed=nx)
            if kind == "near":  # neighbours within a few ulps of each other: ties after rounding
                rng = np.random.default_rng(nx)
                base = np.float32(1000.0) + (rng.integers(0, 3, (ny, nx)) * np.float32(0.5)).astype(np.float32)
                z = (base.view(np.uint32) + rng.integers(-6, 7, (ny, nx)).astype(np.uint32)).view(np.float32)
            else:
                z = make_case(kind, nx, ny, seed=ny + mode)
            set_constants(g, dx)
            zd = dev(torch, z.ravel())
            ro, go = orc.compute_receivers(z, g.og, dx)
            for path in (1, 2, 0):
                lib.pff_receivers_set_path(path)
                r = torch.full((g.N,), -7, dtype=torch.int32, device="cuda")
                gr = torch.full((g.N,), -7.0, dtype=torch.float32, device="cuda")
                flow.compute_receivers(zd, r, gr)
                assert np.array_equal(host(r), ro), (nx, ny, kind, path)
                assert np.array_equal(fbits(host(gr)), fbits(go)), (nx, ny, kind, path)
    finally:
        lib.pff_receivers_set_path(1)


@pytest.mark.parametrize("dx", [30.0, 10.0, 3.0, 1.0, 0.3, 7.77, 123.456, 1e-3, 3e-20, 1e4, 0.1, 2.0 ** -20])
def test_receivers_division_exhaustive(cuda, dx):
    """The lean kernel's Markstein-corrected quotient equals the IEEE division for
    every float in the range of drops it is used for."""
    import ctypes as C

    from pyfastflow_b200 import _lib

    lib = _lib.load()
    bad, n = C.c_longlong(-1), C.c_longlong(0)
    assert lib.pff_receivers_div_selfcheck(np.float32(dx), C.byref(bad), C.byref(n)) == 0
    assert n.value > (100 << 23), n.value  # 135-200 binades of drops, by dx
    assert bad.value == 0


@pytest.mark.parametrize("mode", MODES)
def test_basin_labels(orc, cuda, mode):
    torch = cuda
    from pyfastflow_b200 import flow

    g = Grid(orc, torch, 203, 157, mode, seed=3)
    z = make_case("spectral", 203, 157, seed=11)
    set_constants(g, 10.0)
    rcv, _ = orc.compute_receivers(z, g.og, 10.0)
    bid = torch.empty(g.N, dtype=torch.int32, device="cuda")
    tmp = torch.empty_like(bid)
    flow.basin_identification(bid, dev(torch, rcv), tmp)
    assert np.array_equal(host(bid), orc.basin_labels(rcv, g.og))


@pytest.mark.parametrize("mode", MODES)
def test_depression_counter(orc, cuda, mode):
    """flow.depression_counter (lakeflow.py:25-44): interior self-receivers, on raw
    receivers (many pits), on flats (ties give self-receivers) and after a reroute
    (pits left only where the reference leaves them)."""
    torch = cuda
    from pyfastflow_b200 import flow

    for kind, (nx, ny) in [("spectral", (203, 157)), ("int", (64, 48)), ("uniform", (9, 7))]:
        g = Grid(orc, torch, nx, ny, mode, seed=5)
        z = make_case(kind, nx, ny, seed=13 + mode)
        set_constants(g, 10.0)
        rcv, _ = orc.compute_receivers(z, g.og, 10.0)
        want = orc.depression_counter(rcv, g.og)
        assert flow.depression_counter(dev(torch, rcv)) == want, (kind, mode)
        r2, _, _, _, _ = orc.reroute_flow(rcv, z, g.og)
        assert flow.depression_counter(dev(torch, r2)) == orc.depression_counter(r2, g.og)
    # a grid of one flat value: every cell is its own receiver; the count is the
    # number of cells that cannot leave the domain
    g = Grid(orc, torch, 16, 12, mode, seed=9)
    set_constants(g, 1.0)
    rcv = np.arange(g.N, dtype=np.int32)
    assert flow.depression_counter(dev(torch, rcv)) == orc.depression_counter(rcv, g.og)


@pytest.mark.parametrize("mode", MODES)
def test_saddlesort(orc, cuda, mode):
    torch = cuda
    from pyfastflow_b200 import flow

    g = Grid(orc, torch, 180, 140, mode, seed=5)
    z = make_case("spectral", 180, 140, seed=21)
    set_constants(g, 10.0)
    rcv, _ = orc.compute_receivers(z, g.og, 10.0)
    bid = orc.basin_labels(rcv, g.og)
    st = orc.saddlesort(bid, z, g.og)
    N = g.N
    isb = torch.zeros(N, dtype=torch.uint8, device="cuda")
    zp = torch.zeros(N, dtype=torch.float32, device="cuda")
    sad = torch.zeros(N + 1, dtype=torch.int64, device="cuda")
    sn = torch.zeros(N + 1, dtype=torch.int32, device="cuda")
    out = torch.zeros(N + 1, dtype=torch.int64, device="cuda")
    flow.saddlesort(dev(torch, bid), isb, zp, sad, sn, out, dev(torch, z.ravel()))
    assert np.array_equal(host(isb), st.is_border)
    assert np.array_equal(host(zp).view(np.uint32), st.z_prime.view(np.uint32))
    assert np.array_equal(host(sad), st.basin_saddle)
    assert np.array_equal(host(sn), st.basin_saddlenode)
    assert np.array_equal(host(out), st.outlet)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("carve", [True, False])
def test_reroute(orc, cuda, mode, carve):
    torch = cuda
    from pyfastflow_b200 import flow

    # uniform 400 x 300: about 24,000 pits, more than one CTA's basin relabelling takes
    for kind, (nx, ny) in [("spectral", (211, 173)), ("int", (64, 48)), ("int", (9, 7)), ("uniform", (130, 66)),
                           ("spectral", (512, 384)), ("uniform", (400, 300))]:
        g = Grid(orc, torch, nx, ny, mode, seed=7)
        z = make_case(kind, nx, ny, seed=31 + mode)
        set_constants(g, 10.0)
        rcv, _ = orc.compute_receivers(z, g.og, 10.0)
        r_o, r_o_, st, nd, nout = orc.reroute_flow(rcv, z, g.og, carve=carve)
        N = g.N
        T = lambda n, dt: torch.zeros(n, dtype=dt, device="cuda")  # noqa: E731
        rec = dev(torch, rcv)
        rec_, rec__, bid = T(N, torch.int32), T(N, torch.int32), T(N, torch.int32)
        zp, isb = T(N, torch.float32), T(N, torch.uint8)
        out, sad, sn = T(N + 1, torch.int64), T(N + 1, torch.int64), T(N + 1, torch.int32)
        tag, tag_ = T(N, torch.uint8), T(N, torch.uint8)
        n_outer = flow.reroute_flow(bid, rec, rec_, rec__, dev(torch, z.ravel()), zp, isb, out, sad, sn, tag, tag_,
                                    None, carve=carve)
        assert n_outer == nout
        assert np.array_equal(host(rec), r_o), (kind, mode, carve)
        assert np.array_equal(host(rec_), r_o_)
        assert np.array_equal(host(bid), st.bid)
        if nd:
            assert np.array_equal(host(sad)[:N], st.basin_saddle[:N])
            assert np.array_equal(host(out)[:N], st.outlet[:N])
            assert np.array_equal(host(sn)[:N], st.basin_saddlenode[:N])
            assert np.array_equal(host(isb), st.is_border)
            assert np.array_equal(host(zp).view(np.uint32), st.z_prime.view(np.uint32))
            if carve:
                assert np.array_equal(host(tag), st.tag)


def test_rake_compress_rounds_match_oracle(orc, cuda):
    """Kernel-level API, round by round: every buffer bit-identical."""
    torch = cuda
    from pyfastflow_b200 import flow

    rng = np.random.default_rng(4)
    nx, ny = 128, 96
    g = Grid(orc, torch, nx, ny, 1)
    z = make_case("spectral", nx, ny, seed=41)
    rcv, _ = orc.compute_receivers(z, g.og, 5.0)
    rcv, _, _, _, _ = orc.reroute_flow(rcv, z, g.og)
    N = g.N
    p0 = rng.lognormal(0, 0.5, N).astype(np.float32)
    # oracle buffers
    o = dict(dnr=np.zeros(4 * N, np.int32), ndnr=np.zeros(N, np.int32), p=p0.copy(), src=np.zeros(N, np.int32),
             dnr_=np.zeros(4 * N, np.int32), ndnr_=np.zeros(N, np.int32), p_=np.zeros(N, np.float32))
    d = {k: dev(torch, v) for k, v in o.items()}
    orc.rcv2donor(rcv, o["dnr"], o["ndnr"])
    flow.rcv2donor(dev(torch, rcv), d["dnr"], d["ndnr"])
    assert np.array_equal(host(d["ndnr"]), o["ndnr"])
    assert np.array_equal(host(d["dnr"]), o["dnr"])
    logn = orc.ceil_log2(N) + 1
    for it in range(logn + 1):
        orc.rake_compress_accum(o["dnr"], o["ndnr"], o["p"], o["src"], o["dnr_"], o["ndnr_"], o["p_"], it)
        flow.rake_compress_accum(d["dnr"], d["ndnr"], d["p"], d["src"], d["dnr_"], d["ndnr_"], d["p_"], it)
        for k in o:
            assert np.array_equal(host(d[k]).view(np.uint32), o[k].view(np.uint32)), (it, k)
    orc.fuse(o["p"], o["src"], o["p_"], logn)
    flow.fuse(d["p"], d["src"], d["p_"], logn)
    assert np.array_equal(host(d["p"]).view(np.uint32), o["p"].view(np.uint32))


@pytest.mark.parametrize("mode", [0, 1])
def test_flowrouter_pipeline(orc, cuda, mode):
    """FlowRouter: receivers -> carve reroute -> accumulate, constant and weighted."""
    torch = cuda
    import pyfastflow_b200 as pf

    nx, ny = (320, 256)
    z = synthetic.spectral_dem(nx, ny, 77, relief=800.0, npits=40, pit_scale=0.2)
    router = pf.flow.FlowRouter(nx, ny, 30.0, boundary_mode=["normal", "periodic_EW"][mode])
    router.set_z(z)
    router.compute_receivers()
    router.reroute_flow()
    router.accumulate_constant_Q(1.0, area=True)
    og = orc.Grid(nx, ny, mode)
    rcv, _ = orc.compute_receivers(z, og, 30.0)
    r2, _, _, _, _ = orc.reroute_flow(rcv, z, og)
    assert np.array_equal(router.get_receivers().ravel(), r2)
    Qo, co = orc.accumulate(r2, np.float32(900.0))
    # default path: exact counts; drainage area = count x dx^2 rounded once
    assert np.array_equal(router.get_counts().ravel(), co)
    assert np.array_equal(router.get_Q().ravel(), (co.astype(np.float64) * 900.0).astype(np.float32))
    assert_q_close(router.get_Q().ravel(), Qo)
    # exact_order: the reference's f32 summation order, bit for bit
    router.accumulate_constant_Q(1.0, area=True, exact_order=True)
    assert np.array_equal(router.get_Q().ravel().view(np.uint32), Qo.view(np.uint32))
    assert np.array_equal(router.get_counts().ravel(), co)
    w = synthetic.lognormal_weights(nx * ny, 5)
    Qw, _ = orc.accumulate(r2, w)
    router.accumulate_weighted_Q(w)
    assert_q_close(router.get_Q().ravel(), Qw)
    assert np.array_equal(router.get_counts().ravel(), co)
    router.accumulate_weighted_Q(w, exact_order=True)
    assert np.array_equal(router.get_Q().ravel().view(np.uint32), Qw.view(np.uint32))


def test_routing_plain_512_bit_exact(orc, cuda):
    """512 x 512, dx 30, tilt, all edges outlets, no reroute: receivers and
    drainage area (uint32 count x dx^2) bit-exact."""
    import pyfastflow_b200 as pf

    w = synthetic.routing_plain_512()
    router = pf.flow.FlowRouter(512, 512, 30.0, lakeflow=False)
    router.set_z(w["z"])
    router.compute_receivers()
    router.accumulate_constant_Q(1.0, area=False)
    og = orc.Grid(512, 512, 0)
    rcv, _ = orc.compute_receivers(w["z"], og, 30.0)
    assert np.array_equal(router.get_receivers().ravel(), rcv)
    cnt = orc.topo_accumulate(rcv)
    assert np.array_equal(router.get_counts().ravel(), cnt)
    assert np.array_equal(router.get_Q().ravel(), cnt.astype(np.float32))


@pytest.mark.parametrize("grid_given", [True, False])
def test_accumulate_general_forest(orc, cuda, grid_given):
    """Receivers that are not D4 neighbours (an arbitrary forest) take the
    scatter path; D4 receivers take the gather path; both bit-exact."""
    torch = cuda
    from pyfastflow_b200 import _dev, _lib

    rng = np.random.default_rng(12)
    nx, ny = 150, 120
    N = nx * ny
    forests = []
    # random forest, parent index below the child's, at most 4 donors per node
    rcv = np.arange(N, dtype=np.int32)
    nchild = np.zeros(N, np.int32)
    for i in range(1, N):
        if rng.random() < 0.03:
            continue
        for _ in range(8):
            p = int(rng.integers(max(0, i - 5000), i))
            if nchild[p] < 4:
                rcv[i] = p
                nchild[p] += 1
                break
    forests.append(rcv)
    z = make_case("spectral", nx, ny, seed=3)
    og = orc.Grid(nx, ny, 0)
    r_d4, _ = orc.compute_receivers(z, og, 10.0)
    forests.append(orc.reroute_flow(r_d4, z, og)[0])
    ws = _dev.Scratch()
    for rcv in forests:
        w = rng.lognormal(0, 0.5, N).astype(np.float32)
        Qd = dev(torch, w)
        cd = torch.zeros(N, dtype=torch.int32, device="cuda")
        wp, wn = ws.get(_lib.load().pff_accumulate_workspace_bytes(N))
        rd = dev(torch, rcv)  # held until the kernels have run
        if grid_given:
            _lib.call("pff_accumulate_grid", rd.data_ptr(), Qd.data_ptr(), cd.data_ptr(), nx, ny, 0,
                      None, N, wp, wn, _dev.stream())
        else:
            _lib.call("pff_accumulate", rd.data_ptr(), Qd.data_ptr(), cd.data_ptr(), N, wp, wn, _dev.stream())
        Qo, co = orc.accumulate(rcv, w)
        assert np.array_equal(host(cd).view(np.uint32), co)
        assert np.array_equal(host(Qd).view(np.uint32), Qo.view(np.uint32))


def test_routing_lakes_4096_bit_exact(orc, cuda):
    """The full 4096 x 4096 benchmark workload (2000 pits, periodic east-west,
    carve): rerouted receivers and uint32 counts bit-exact; weighted Q within the
    f32 tolerance (and bit-exact with exact_order=True)."""
    import pyfastflow_b200 as pf

    w = synthetic.routing_lakes(4096)
    z = w["z"]
    wt = synthetic.lognormal_weights(4096 * 4096, 102)
    router = pf.flow.FlowRouter(4096, 4096, 30.0, boundary_mode="periodic_EW")
    router.set_z(z)
    router.compute_receivers()
    router.reroute_flow()
    router.accumulate_weighted_Q(wt)
    og = orc.Grid(4096, 4096, 1)
    rcv, _ = orc.compute_receivers(z, og, 30.0)
    r2, _, _, _, nout = orc.reroute_flow(rcv, z, og)
    assert router.last_n_outer == nout
    assert np.array_equal(router.get_receivers().ravel(), r2)
    Qo, co = orc.accumulate(r2, wt)
    assert np.array_equal(router.get_counts().ravel(), co)
    assert_q_close(router.get_Q().ravel(), Qo)
    router.accumulate_weighted_Q(wt, exact_order=True)
    assert np.array_equal(router.get_counts().ravel(), co)
    assert np.array_equal(router.get_Q().ravel().view(np.uint32), Qo.view(np.uint32))
    assert orc.count_cycle_nodes(r2) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("dx", [0.3, 1.0, 7.3, 29.999, 1e-3, 1e4, 3.0e-20])
def test_receivers_division_any_dx(orc, cuda, dx):
    """The receivers kernel divides by dx with a reciprocal and an exact residual
    check (IEEE division only where the check cannot decide): receivers and
    gradients must equal the oracle's IEEE quotients for any dx, on drops from
    tiny (subnormal quotients) to huge."""
    torch = cuda
    from pyfastflow_b200 import flow

    rng = np.random.default_rng(int(dx * 1000) % 97)
    nx, ny = 256, 96
    z = (rng.random((ny, nx)) * 10.0 ** rng.integers(-30, 30, (ny, nx))).astype(np.float32)
    z[:8] = rng.integers(0, 5, (8, nx)).astype(np.float32)  # exact ties
    g = Grid(orc, torch, nx, ny, 0)
    set_constants(g, dx)
    rcv, grad = orc.compute_receivers(z, g.og, dx)
    r = torch.empty(g.N, dtype=torch.int32, device="cuda")
    gr = torch.empty(g.N, dtype=torch.float32, device="cuda")
    flow.compute_receivers(dev(torch, z.ravel()), r, gr)
    assert np.array_equal(host(r), rcv)
    assert np.array_equal(fbits(host(gr)), fbits(grad))
