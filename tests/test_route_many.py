"""FlowRouter.route_many: a sequence of DEMs routed with the copies of neighbouring
DEMs overlapped on copy streams gives, for every DEM, exactly the results of the
plain call sequence."""
import numpy as np
import pytest

from pyfastflow_b200 import synthetic


@pytest.mark.gpu
def test_route_many_matches_single_calls(cuda):
    torch = cuda
    import pyfastflow_b200 as pf

    n = 256
    dems = [synthetic.routing_lakes(n, seed=s)["z"] for s in (3, 4, 5, 3)]
    ws = [synthetic.lognormal_weights(n * n, 10 + k) for k in range(4)]
    r = pf.flow.FlowRouter(n, n, 30.0, boundary_mode="periodic_EW")
    zh = [torch.from_numpy(d.ravel().copy()).pin_memory() for d in dems]
    wh = [torch.from_numpy(w.copy()).pin_memory() for w in ws]
    qh = [torch.empty(n * n, dtype=torch.float32).pin_memory() for _ in dems]
    ch = [torch.empty(n * n, dtype=torch.int32).pin_memory() for _ in dems]
    r.route_many(zh, wh, qh, ch)
    torch.cuda.synchronize()
    for k, d in enumerate(dems):
        r1 = pf.flow.FlowRouter(n, n, 30.0, boundary_mode="periodic_EW")
        r1.set_z(d)
        r1.compute_receivers()
        r1.reroute_flow()
        r1.accumulate_weighted_Q(ws[k])
        torch.cuda.synchronize()
        assert np.array_equal(qh[k].numpy().view(np.uint32), r1.Q.cpu().numpy().view(np.uint32)), k
        assert np.array_equal(ch[k].numpy(), r1.counts.cpu().numpy()), k
