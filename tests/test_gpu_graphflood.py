"""GraphFlood kernels vs the oracle: fill (snapshot rounds), diffusion (serial
summation order), Manning update, and whole Flooder iterations -- bit-exact."""
import numpy as np
import pytest

from pyfastflow_b200 import synthetic

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def bits(a):
    """Bit patterns, with every NaN mapped to one value: NaN positions must match,
    NaN payloads (0x7fffffff on the GPU, 0xffc00000 on x86) need not."""
    a = np.asarray(a, np.float32)
    b = a.view(np.uint32).copy()
    b[np.isnan(a)] = 0x7FC00000
    return b


def state(orc, nx, ny, mode, seed, h_scale=0.5):
    rng = np.random.default_rng(seed)
    z = synthetic.spectral_dem(nx, ny, seed, relief=50.0, npits=20, pit_scale=0.2)
    h = (rng.random(nx * ny) * h_scale).astype(np.float32)
    zh = (z.ravel() + h).astype(np.float32)
    og = orc.Grid(nx, ny, mode)
    rcv, _ = orc.compute_receivers(zh, og, 10.0)
    rcv, _, _, _, _ = orc.reroute_flow(rcv, zh, og)
    return og, zh, h, rcv


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_fill_z_add_delta(orc, cuda, mode):
    torch = cuda
    from pyfastflow_b200 import flow

    og, zh, h, rcv = state(orc, 150, 110, mode, 3)
    zd, hd = dev(torch, zh), dev(torch, h)
    z_ = torch.zeros_like(zd)
    r_, r__ = torch.zeros(og.N, dtype=torch.int32, device="cuda"), torch.zeros(og.N, dtype=torch.int32, device="cuda")
    flow.fill_z_add_delta(zd, hd, z_, dev(torch, rcv), r_, r__, epsilon=1e-3)
    zo, ho, z_o = orc.fill_z_add_delta(zh.copy(), h.copy(), rcv, eps=1e-3)
    assert np.array_equal(bits(host(zd)), bits(zo))
    assert np.array_equal(bits(host(hd)), bits(ho))
    assert np.array_equal(bits(host(z_)), bits(z_o))


def test_fill_arbitrary_pointers(orc, cuda):
    """Fill rounds on receivers that are not a forest: random pointers (cycles of
    every length, self-pointers made by jumping around a cycle) and NaN heights.
    The packed rounds read zh at such self-pointers; bit-exact against the oracle,
    including both receiver buffers."""
    torch = cuda
    from pyfastflow_b200 import flow

    rng = np.random.default_rng(21)
    for n in (2, 3, 1000, 70001):
        zh = (rng.random(n) * 100).astype(np.float32)
        zh[rng.random(n) < 0.01] = np.nan
        h = (rng.random(n) * 0.3).astype(np.float32)
        rcv = rng.integers(0, n, n).astype(np.int32)
        rcv[rng.random(n) < 0.2] = rng.integers(0, n)  # one cell with many donors
        roots = rng.random(n) < 0.1
        rcv[roots] = np.flatnonzero(roots)
        zd, hd = dev(torch, zh), dev(torch, h)
        z_ = torch.zeros_like(zd)
        r_ = torch.zeros(n, dtype=torch.int32, device="cuda")
        r__ = torch.zeros(n, dtype=torch.int32, device="cuda")
        flow.fill_z_add_delta(zd, hd, z_, dev(torch, rcv), r_, r__, epsilon=1e-3)
        zo, ho, z_o = orc.fill_z_add_delta(zh.copy(), h.copy(), rcv, eps=1e-3)
        assert np.array_equal(bits(host(zd)), bits(zo)), n
        assert np.array_equal(bits(host(hd)), bits(ho)), n
        assert np.array_equal(bits(host(z_)), bits(z_o)), n
        jumped = rcv.copy()
        for _ in range(int(np.ceil(np.log2(n)))):
            jumped = jumped[jumped]
        assert np.array_equal(host(r_), jumped) and np.array_equal(host(r__), jumped), n


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_diffuse(orc, cuda, mode):
    torch = cuda
    from pyfastflow_b200 import constants as cte
    from pyfastflow_b200.graphflood import diffuse_Q_constant_prec

    nx, ny = 131, 97
    rng = np.random.default_rng(mode)
    zh = synthetic.spectral_dem(nx, ny, 5, relief=20.0).ravel()
    codes = None
    if mode == 3:
        codes = rng.choice(np.array([1, 1, 1, 1, 3, 0, 9], np.uint8), nx * ny)
    og = orc.Grid(nx, ny, mode, codes)
    Q = (rng.random(nx * ny) * 10).astype(np.float32)
    cte.NX, cte.NY, cte.DX, cte.BOUND_MODE, cte.PREC = nx, ny, 10.0, mode, 1e-5
    cte.boundaries = dev(torch, codes) if codes is not None else None
    Qd, tmp = dev(torch, Q), torch.zeros(nx * ny, dtype=torch.float32, device="cuda")
    diffuse_Q_constant_prec(dev(torch, zh), Qd, tmp, nsweeps=5)
    Qo = Q.copy()
    for _ in range(5):
        orc.diffuse_q(zh, Qo, og, 10.0, 1e-5)
    assert np.array_equal(bits(host(Qd)), bits(Qo))
    assert np.array_equal(bits(host(tmp)), bits(Qo))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_diffuse_shapes_and_sweeps(orc, cuda, mode):
    """All sweeps of one call in one tiled pass (64 x 16 tiles, halo = sweeps): grids
    narrower than the halo, ragged tile edges, 1-8 sweeps and 9 (the per-sweep path),
    each bit-exact against the oracle's serial sweeps."""
    torch = cuda
    from pyfastflow_b200 import constants as cte
    from pyfastflow_b200.graphflood import diffuse_Q_constant_prec

    cases = [(3, 3, 5), (3, 40, 8), (70, 3, 5), (5, 7, 2), (65, 17, 1), (129, 33, 5), (200, 50, 8),
             (64, 16, 3), (90, 45, 9)]
    for nx, ny, ns in cases:
        rng = np.random.default_rng(nx * 1000 + ny + mode)
        zh = synthetic.spectral_dem(nx, ny, 11, relief=20.0).ravel() if min(nx, ny) > 8 else \
            (rng.random(nx * ny) * 5).astype(np.float32)
        zh[rng.random(nx * ny) < 0.05] = zh.min()  # flats and pits: cells with no outflow
        og = orc.Grid(nx, ny, mode)
        Q = (rng.random(nx * ny) * 10).astype(np.float32)
        cte.NX, cte.NY, cte.DX, cte.BOUND_MODE, cte.PREC = nx, ny, 7.5, mode, 2e-5
        cte.boundaries = None
        Qd, tmp = dev(torch, Q), torch.zeros(nx * ny, dtype=torch.float32, device="cuda")
        diffuse_Q_constant_prec(dev(torch, zh), Qd, tmp, nsweeps=ns)
        Qo = Q.copy()
        for _ in range(ns):
            orc.diffuse_q(zh, Qo, og, 7.5, 2e-5)
        assert np.array_equal(bits(host(Qd)), bits(Qo)), (nx, ny, ns)
        assert np.array_equal(bits(host(tmp)), bits(Qo)), (nx, ny, ns)


def test_manning_core(orc, cuda):
    torch = cuda
    from pyfastflow_b200 import constants as cte
    from pyfastflow_b200.graphflood import graphflood_core_cte_mannings

    og, zh, h, rcv = state(orc, 128, 128, 0, 9, h_scale=0.2)
    rng = np.random.default_rng(1)
    Q = (rng.random(og.N) * 50).astype(np.float32)
    h[::17] = -0.01  # negative depths take the reference's NaN path
    cte.DX, cte.MANNING, cte.EDGESW, cte.DT_HYDRO = 10.0, 0.033, 1e-2, 5e-3
    hd, zd, dh = dev(torch, h), dev(torch, zh), torch.zeros(og.N, dtype=torch.float32, device="cuda")
    graphflood_core_cte_mannings(hd, zd, dh, dev(torch, rcv), dev(torch, Q))
    ho, zo, dho = orc.graphflood_core(h.copy(), zh.copy(), rcv, Q, 10.0, 0.033, 1e-2, 5e-3)
    assert np.array_equal(bits(host(hd)), bits(ho))
    assert np.array_equal(bits(host(zd)), bits(zo))
    assert np.array_equal(bits(host(dh)), bits(dho))
    assert np.isnan(host(hd)[::17]).all()


def test_manning_core_one_pass(orc, cuda):
    """pff_graphflood_core_filled (slopes from a copy of zh, both loops in one pass)
    equals the two-loop update and the oracle bit for bit, residual included."""
    torch = cuda
    from pyfastflow_b200 import _dev, _lib

    og, zh, h, rcv = state(orc, 160, 96, 1, 17, h_scale=0.3)
    rng = np.random.default_rng(4)
    Q = (rng.random(og.N) * 40).astype(np.float32)
    h[::13] = -0.02
    h[5::29] = 0.0
    args = (og.N, 10.0, 100.0, 0.033, 1e-2, 5e-3)  # rounded to f32 by the binding
    out = {}
    rd, qd = dev(torch, rcv), dev(torch, Q)  # held: a freed temporary's block could be reused by the next
    for fn in ("pff_graphflood_core", "pff_graphflood_core_filled"):
        hd, zd, zf = dev(torch, h), dev(torch, zh), dev(torch, zh)
        dh = torch.zeros(og.N, dtype=torch.float32, device="cuda")
        href = dev(torch, h + 0.01)
        dmax = torch.zeros(1, dtype=torch.float32, device="cuda")
        ptrs = [hd.data_ptr(), zd.data_ptr()] + ([zf.data_ptr()] if fn.endswith("filled") else [])
        _lib.call(fn, *ptrs, dh.data_ptr(), rd.data_ptr(), qd.data_ptr(), *args, href.data_ptr(), dmax.data_ptr(),
                  _dev.stream())
        out[fn] = [host(hd), host(zd), host(dh), host(dmax)]
    ho, zo, dho = orc.graphflood_core(h.copy(), zh.copy(), rcv, Q, 10.0, 0.033, 1e-2, 5e-3)
    for a, b in zip(out["pff_graphflood_core"], out["pff_graphflood_core_filled"]):
        assert np.array_equal(bits(a), bits(b))
    got = out["pff_graphflood_core_filled"]
    assert np.array_equal(bits(got[0]), bits(ho)) and np.array_equal(bits(got[1]), bits(zo))
    assert np.array_equal(bits(got[2]), bits(dho))


@pytest.mark.parametrize("mode", [0, 1])
def test_flooder_iterations(orc, cuda, mode):
    """Flooder.run_graphflood vs the oracle's run of the same iterations."""
    import pyfastflow_b200 as pf

    nx, ny, dx, P = 160, 128, 10.0, 1e-5
    z = synthetic.spectral_dem(nx, ny, 13, relief=60.0, npits=10, pit_scale=0.2)
    router = pf.flow.FlowRouter(nx, ny, dx, boundary_mode=["normal", "periodic_EW"][mode])
    router.set_z(z)
    fl = pf.graphflood.Flooder(router, precipitation_rates=P, manning=0.033, edge_slope=1e-2)
    fl.run_graphflood(6)
    og = orc.Grid(nx, ny, mode)
    zh = z.ravel().copy()
    h = np.zeros(nx * ny, np.float32)
    Q = np.zeros(nx * ny, np.float32)
    orc.graphflood_run(zh, h, Q, og, dx, P, niter=6)
    assert np.array_equal(bits(fl.get_h().ravel()), bits(h))
    assert np.array_equal(bits(router.get_Z().ravel()), bits(zh))
    assert np.array_equal(bits(router.get_Q().ravel()), bits(Q))


@pytest.mark.parametrize("stop", ["max", "mean"])
def test_run_to_residual_stops_at_the_first_converged_iteration(cuda, stop):
    """run_to_residual reads each residual one iteration late (at the next reroute's
    synchronisation); it must still stop at the first iteration whose residual is
    below the threshold, with h, z and Q of that iteration, and report the same
    residual trace as a plain loop that checks after every iteration."""
    torch = cuda
    import pyfastflow_b200 as pf
    from pyfastflow_b200 import constants as cte

    nx, ny, dx, P = 128, 96, 10.0, 1e-5
    z = synthetic.spectral_dem(nx, ny, 21, relief=40.0, npits=8, pit_scale=0.2)

    def fresh():
        router = pf.flow.FlowRouter(nx, ny, dx)
        router.set_z(z)
        return router, pf.graphflood.Flooder(router, precipitation_rates=P, manning=0.033, edge_slope=1e-2)

    router, fl = fresh()
    res = []
    for _ in range(40):
        h0 = fl.h.clone()
        fl.iteration()
        d = (fl.h - h0).abs()
        res.append(float(d.max() if stop == "max" else d.float().mean()) / cte.DT_HYDRO)
    srt = sorted(res)  # a threshold halfway between two residuals from the middle of the run
    thr = 0.5 * (srt[len(srt) // 2] + srt[len(srt) // 2 + 1])
    first = next(k for k, r in enumerate(res) if r < thr) + 1
    r2, fl2 = fresh()
    for _ in range(first):
        fl2.iteration()
    torch.cuda.synchronize()
    # the pipelined loop (guarded post-reroute graphs), and the one-by-one loop it
    # falls back to where the device-driven reroute is switched off
    from pyfastflow_b200 import _lib

    for graphs in (1, 0):
        prev = _lib.load().pff_reroute_use_graphs(graphs)
        try:
            router, fl = fresh()
            n, why, r = fl.run_to_residual(tol_ratio=thr / P, max_iter=40, return_trace=False, stop=stop)
        finally:
            _lib.load().pff_reroute_use_graphs(prev)
        torch.cuda.synchronize()
        assert n == first and why == "residual", graphs
        assert r == pytest.approx(res[first - 1], rel=1e-5)
        assert torch.equal(fl.h, fl2.h) and torch.equal(router.z, r2.z) and torch.equal(router.Q, r2.Q)
    # the cap: max_iter iterations, the last residual reported
    router, fl = fresh()
    n, why, r, tr = fl.run_to_residual(tol_ratio=1e-30, max_iter=7, return_trace=True, stop=stop)
    assert n == 7 and why == "max_iter" and len(tr) == 7
    assert np.allclose(tr, res[:7], rtol=1e-5) and r == pytest.approx(res[6], rel=1e-5)


def test_pipelined_run_equals_iterations(cuda):
    """run_graphflood's pipelined loop (asynchronous reroute, guarded post-reroute
    graph) leaves h, z, Q and the router's fields exactly as the same number of
    single iterations does, periodic boundaries included, also when the two loops
    alternate on one Flooder (a workspace reallocated under a captured graph once
    made that fault)."""
    torch = cuda
    import pyfastflow_b200 as pf

    nx, ny = 192, 160
    z = synthetic.spectral_dem(nx, ny, 8, relief=80.0, npits=30, pit_scale=0.3)
    outs = []
    for pipelined in (True, False):
        router = pf.flow.FlowRouter(nx, ny, 10.0, boundary_mode="periodic_EW")
        router.set_z(z)
        fl = pf.graphflood.Flooder(router, precipitation_rates=2e-5, manning=0.04, edge_slope=1e-2)
        if pipelined:  # both loops on one Flooder: their graphs share its workspaces
            fl.run_graphflood(10)
            for _ in range(5):
                fl.iteration()
            fl.run_graphflood(10)
        else:
            for _ in range(25):
                fl.iteration()
        torch.cuda.synchronize()
        outs.append([t.clone() for t in (fl.h, router.z, router.Q, router.receivers, router.bid, router.z_)])
    for a, b in zip(*outs):  # bit patterns: NaN depths compare equal too
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))


@pytest.mark.gpu
def test_graphflood_2048_50_iterations_match_oracle_fixture(cuda):
    """The 2048 x 2048 GraphFlood benchmark DEM, 50 iterations through Flooder
    (each with receivers, carve rerouting, fill, 5 diffusion sweeps, Manning):
    h, zh and Q bit-identical to the CPU oracle's, compared through the SHA-256 of
    their bit patterns recorded in tests/golden/graphflood_2048_50.json (written by
    tests/golden/make_graphflood_2048_fixture.py)."""
    import hashlib
    import json
    import os

    import pyfastflow_b200 as pf

    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "graphflood_2048_50.json")))
    n = 2048
    z = synthetic.graphflood_plain(n)["z"]
    router = pf.flow.FlowRouter(n, n, 10.0)
    router.set_z(z)
    fl = pf.graphflood.Flooder(router, precipitation_rates=1e-5, manning=0.033, edge_slope=1e-2)
    fl.run_graphflood(fx["iterations"])
    cuda.cuda.synchronize()

    def sha(a):
        a = np.ascontiguousarray(a, np.float32).ravel()
        b = a.view(np.uint32).copy()
        b[np.isnan(a)] = 0x7FC00000
        return hashlib.sha256(b.tobytes()).hexdigest()

    assert sha(fl.get_h()) == fx["sha256"]["h"]
    assert sha(router.get_Z()) == fx["sha256"]["zh"]
    assert sha(router.get_Q()) == fx["sha256"]["Q"]
