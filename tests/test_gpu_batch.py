"""Batched instances on one GPU (llg_batch_*): concurrent integration of
independent instances of uneven size on their own streams (demag chains
replayed as CUDA graphs, transform launch shapes autotuned) gives the same
results as integrating each instance alone on the default stream."""
import numpy as np
import pytest

import llg

pytestmark = pytest.mark.gpu


def test_batch_matches_instances_run_alone(gpu):
    import torch
    small = ((64, 64), (96, 48), (64, 96), (128, 64))
    insts = llg.config4_instances(10, 2024, sizes=small)
    opts = llg.default_solver_opts()
    b = llg.Batch([x["params"] for x in insts])
    y0 = [torch.from_numpy(llg.setup_instance(b.ctx[i], x)).cuda() for i, x in enumerate(insts)]
    outs = [torch.zeros_like(y) for y in y0]
    b.integrator_init(0.0, y0, opts)
    for k in range(1, 6):
        rcs = b.integrate(0.1 * k, outs, nthreads=len(insts))
        assert all(r == 0 for r in rcs)
    torch.cuda.synchronize()
    stats = b.stats()
    for i, x in enumerate(insts):
        c = llg.Context(x["params"])
        y = torch.from_numpy(llg.setup_instance(c, x)).cuda()
        c.integrator_init(0.0, y, opts)
        yo = torch.zeros_like(y)
        for k in range(1, 6):
            c.integrate(0.1 * k, yo)
        torch.cuda.synchronize()
        d = np.abs(yo.cpu().numpy() - outs[i].cpu().numpy()).max()
        print(x["name"], "max|batch - alone| =", d, "nst", stats[i]["nst"], c.stats()["nst"])
        assert d == 0.0
        assert stats[i]["nst"] == c.stats()["nst"]
        c.close()
    b.close()


def test_single_graph_batch_matches_device_resident_instances(gpu):
    """llg_batch_integrate_graph: every instance's device-resident step loop
    as one branch of ONE CUDA graph, one launch per output time.  Each
    instance must end bit for bit where the same instance ends when its
    device-resident step graph runs alone, with the same counters."""
    import torch
    small = ((64, 64), (96, 48), (64, 96), (128, 64))
    insts = llg.config4_instances(10, 77, sizes=small)
    opts = llg.default_solver_opts(gs_type=llg.GS_CLASSICAL)
    b = llg.Batch([x["params"] for x in insts])
    y0 = [torch.from_numpy(llg.setup_instance(b.ctx[i], x)).cuda() for i, x in enumerate(insts)]
    outs = [torch.zeros_like(y) for y in y0]
    b.integrator_init(0.0, y0, opts)
    assert all(r == 0 for r in b.integrate(0.1, outs))          # host start-up
    for k in range(2, 7):
        assert all(r == 0 for r in b.integrate_graph(0.1 * k, outs))
    torch.cuda.synchronize()
    stats = b.stats()
    dopts = llg.default_solver_opts(gs_type=llg.GS_CLASSICAL, device_resident=1)
    for i, x in enumerate(insts):
        c = llg.Context(x["params"])
        y = torch.from_numpy(llg.setup_instance(c, x)).cuda()
        c.integrator_init(0.0, y, dopts)
        yo = torch.zeros_like(y)
        for k in range(1, 7):
            c.integrate(0.1 * k, yo)
        torch.cuda.synchronize()
        d = np.abs(yo.cpu().numpy() - outs[i].cpu().numpy()).max()
        s = c.stats()
        print(x["name"], "max|graph batch - alone| =", d, "nst", stats[i]["nst"], s["nst"])
        assert d == 0.0
        for key in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups"):
            assert stats[i][key] == s[key], (x["name"], key)
        c.close()
    # switching back to the host-driven batch continues from the same state
    assert all(r == 0 for r in b.integrate(0.8, outs))
    b.close()
