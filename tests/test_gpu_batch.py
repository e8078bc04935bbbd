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
