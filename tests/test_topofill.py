"""topofill (pyfastflow/flow/fill_topo.py:48-78): the standalone DEM fill along the
receivers, increments 2^it * epsilon starting at epsilon."""
import numpy as np
import pytest

from pyfastflow_b200 import synthetic


def test_oracle_topofill_properties(orc):
    z = synthetic.spectral_dem(48, 40, 7, relief=50.0, dx=10.0, npits=6, pit_scale=0.2)
    g = orc.Grid(48, 40, 0)
    rcv0, _ = orc.compute_receivers(z, g, 10.0)
    rcv, _, _, _, _ = orc.reroute_flow(rcv0, z, g)  # carved paths climb out of the pits
    zf = orc.topofill(z, rcv, 1e-3)
    assert (zf >= z.ravel()).all()
    assert (zf > z.ravel()).any()  # the pits were raised
    assert np.array_equal(orc.topofill(z, rcv0, 1e-3), z.ravel())  # plain descent: nothing to fill
    # increments 2^it * eps are the fill's 2^(it-1) * (2 eps)
    zh = z.ravel().copy()
    h = np.zeros_like(zh)
    _, _, z_ = orc.fill_z_add_delta(zh, h, rcv, eps=2e-3)
    assert np.array_equal(zf.view(np.uint32), z_.view(np.uint32))
    # a cell already above its receiver chain is untouched: outlets and roots keep z
    roots = rcv == np.arange(rcv.size)
    assert np.array_equal(zf[roots], z.ravel()[roots])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["normal", "periodic_EW"])
def test_gpu_topofill_bit_exact(orc, cuda, mode):
    torch = cuda
    import pyfastflow_b200 as pf

    n = 256
    z = synthetic.routing_lakes(n, seed=9)["z"]
    r = pf.flow.FlowRouter(n, n, 30.0, boundary_mode=mode)
    r.set_z(z)
    r.compute_receivers()
    r.reroute_flow()
    g = orc.Grid(n, n, {"normal": 0, "periodic_EW": 1}[mode])
    rcv0, _ = orc.compute_receivers(z, g, 30.0)
    rcv, _, _, _, _ = orc.reroute_flow(rcv0, z, g)
    ref = orc.topofill(z, rcv, 1e-6)
    out = torch.zeros(n * n, dtype=torch.float32, device="cuda")
    pf.flow.topofill(r, epsilon=1e-6, custom_z=out)  # custom_z: z is left as it was
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(r.get_Z().ravel().view(np.uint32), z.ravel().view(np.uint32))
    pf.flow.topofill(r, epsilon=1e-6)  # default: z replaced by the filled surface
    torch.cuda.synchronize()
    assert np.array_equal(r.get_Z().ravel().view(np.uint32), ref.view(np.uint32))
