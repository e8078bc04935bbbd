"""Device-resident integrator (llg_solver_opts.device_resident = 1) on the GPU.

The step control of the BDF/Newton/SPGMR integrator runs in control kernels
and CUDA graph conditional nodes instead of on the host.  It must take the
same decisions as the host-driven integrator: identical solver counters and
final states equal to rounding (same kernels, same arithmetic; the only
difference is where pow() of the step-size formulas is evaluated).

Tolerances: counters identical; max|dm| vs the host-driven path <= 1e-9 for
the FP64 chain and <= 1e-5 for the mixed chain (its FP32 rounding of the
demag input turns a last-bit difference of the state, from pow() and fused
multiply-adds in the device-side step-size arithmetic, into an FP32-level
difference of the field); vs the oracle (config 0) <= 1e-6 with identical
counters, as for the host path.
"""
import numpy as np
import pytest

import llg

pytestmark = pytest.mark.gpu

COUNTERS = ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups", "njvevals", "npsolves", "npe")


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def _integrate(p, geo_setup, y0_host, t_end, dt_out, opts):
    import torch
    ctx = llg.Context(p)
    geo_setup(ctx)
    y0 = dev(torch, y0_host)
    ctx.integrator_init(0.0, y0, opts)
    yout = torch.zeros_like(y0)
    tr = []
    for k in range(1, int(round(t_end / dt_out)) + 1):
        tr.append(ctx.integrate(dt_out * k, yout))
    torch.cuda.synchronize()
    st = ctx.stats()
    y = yout.cpu().numpy()
    ctx.close()
    return y, st, tr


def test_config0_device_resident_matches_oracle(oracle_lib, gpu):
    """The reference's CPU-runnable film (128x64, no demag, t 0 -> 100) with the step control
    on the device: identical counters to the oracle's CVODE restatement."""
    import torch
    p = llg.default_params(128, 64)
    geo = llg.build_geometry(llg.default_geom(128, 64, ic_jitter_eps=0.01))
    opts = llg.default_solver_opts(rtol=1e-4, atol=1e-6, maxl=5, device_resident=1)
    ctx = llg.Context(p)
    o = oracle_lib.Oracle(p)
    y0 = dev(torch, geo["y0"])
    ctx.integrator_init(0.0, y0, opts)
    o.integrator_init(geo["y0"], opts)
    yout = torch.zeros_like(y0)
    for k in range(1, 1001):
        ctx.integrate(0.1 * k, yout)
        rc, _, y_o = o.integrate(0.1 * k)
        assert rc == 0
    torch.cuda.synchronize()
    sg, so = ctx.stats(), o.stats()
    dm = np.abs(yout.cpu().numpy() - y_o).max()
    print("config0 device-resident max|dm| =", dm, "gpu", sg, "oracle", so)
    assert dm <= 1e-6
    for k in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups"):
        assert sg[k] == so[k], (k, sg[k], so[k])


def _shape_cases():
    # one small instance of each batched-workload shape (hole, annulus, compact
    # ellipse, windowed polycrystal) with open demag, FP64 and mixed precision
    cases = []
    for prec, tag in ((llg.DEMAG_FP64, "fp64"), (llg.DEMAG_MIXED, "mixed")):
        seen = set()
        for inst in llg.config4_instances(64, 777, demag_precision=prec, sizes=((96, 64),) * 4):
            if inst["shape"] not in seen:
                seen.add(inst["shape"])
                cases.append((f"{inst['shape']}-{tag}", inst))
    return cases


CASES = _shape_cases()


@pytest.mark.parametrize("name,inst", CASES, ids=[c[0] for c in CASES])
def test_device_resident_equals_host_driven(gpu, name, inst):
    geo_y0 = {}

    def setup(ctx):
        geo_y0["y0"] = llg.setup_instance(ctx, inst)

    # geometry once, to get y0
    c0 = llg.Context(inst["params"])
    y0 = llg.setup_instance(c0, inst)
    c0.close()
    res = {}
    for dr in (0, 1):
        opts = llg.default_solver_opts(device_resident=dr)
        res[dr] = _integrate(inst["params"], setup, y0, 1.0, 0.1, opts)
    (ya, sa, ta), (yb, sb, tb) = res[0], res[1]
    dm = float(np.abs(ya - yb).max())
    print(name, "host", sa, "device", sb, "max|dm|", dm)
    for k in COUNTERS:
        assert sa[k] == sb[k], (k, sa[k], sb[k])
    assert ta == tb
    assert dm <= (1e-5 if name.endswith("mixed") else 1e-9)


def test_device_resident_mxstep_and_resume(gpu):
    """A call that runs out of steps returns CV_TOO_MUCH_WORK with y = zn0 at
    the last step, as on the host path; the next call continues."""
    import torch
    p = llg.default_params(64, 48, demag_mode=llg.DEMAG_OPEN, demag_strength=2.0)
    geo = llg.build_geometry(llg.default_geom(64, 48, ic_jitter_eps=0.01))
    out = {}
    for dr in (0, 1):
        ctx = llg.Context(p)
        y0 = dev(torch, geo["y0"])
        ctx.integrator_init(0.0, y0, llg.default_solver_opts(mxstep=40, device_resident=dr))
        yout = torch.zeros_like(y0)
        ctx.integrate(0.02, yout)           # start-up call (host path in both forms)
        with pytest.raises(llg.LLGError, match="TOO_MUCH_WORK"):
            ctx.integrate(5.0, yout)
        y_fail = yout.cpu().numpy().copy()
        st_fail = ctx.stats()
        ctx.integrate(st_fail["tcur"] + 1e-3, yout)
        torch.cuda.synchronize()
        out[dr] = (y_fail, st_fail, yout.cpu().numpy().copy(), ctx.stats())
        ctx.close()
    for i in (1, 3):
        for k in COUNTERS:
            assert out[0][i][k] == out[1][i][k], (k, out[0][i][k], out[1][i][k])
    assert np.abs(out[0][0] - out[1][0]).max() <= 1e-12
    assert np.abs(out[0][2] - out[1][2]).max() <= 1e-12


def test_device_resident_launch_tally(gpu):
    """The graph's launches are tallied on the device: one fused Arnoldi
    operator per Jacobian-vector product and one predict per attempt."""
    import torch
    lib = llg.load()
    import ctypes as C
    p = llg.default_params(96, 64, demag_mode=llg.DEMAG_OPEN, demag_strength=3.0)
    geo = llg.build_geometry(llg.default_geom(96, 64, ic_jitter_eps=0.01))
    ctx = llg.Context(p)
    y0 = dev(torch, geo["y0"])
    ctx.integrator_init(0.0, y0, llg.default_solver_opts(device_resident=1))
    yout = torch.zeros_like(y0)
    ctx.integrate(0.1, yout)
    st0 = ctx.stats()
    c0 = (C.c_int64 * 16)()
    lib.llg_kernel_counts(c0, 16)
    for k in range(2, 11):
        ctx.integrate(0.1 * k, yout)
    c1 = (C.c_int64 * 16)()
    lib.llg_kernel_counts(c1, 16)
    st1 = ctx.stats()
    d = [c1[k] - c0[k] for k in range(16)]
    print("launch deltas", d, "njv", st1["njvevals"] - st0["njvevals"])
    assert d[2] == st1["njvevals"] - st0["njvevals"]          # KID_ARNOLDI
    assert d[8] == st1["nfe_demag"] - st0["nfe_demag"]        # KID_DEMAG_ROWS_INV
    ctx.close()
