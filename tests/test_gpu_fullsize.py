"""Parity at the benchmark sizes, against the FP64 oracle.

The square-hole film the metric is quoted on (1536x512 cells, open demag of
strength 4 on the 3072x1024 transform grid) and the 72-grain polycrystal
(1536x512, windowed open demag of strength 1): one RHS / demag / Jv /
block-Jacobi setup and solve each, with the launch shapes the benchmark
uses (autotuned transform shapes of these sizes), and a plain FP64
integration over t 0 -> 0.1 with both Gram-Schmidt variants — the
reference's own choice at this size (modified, neq >= 5e5,
src/irregular/2d_fft/2d_i2/2d_fft.cu:674-679) and classical.

Tolerances: RHS / Jv / block-Jacobi solve rel 1e-11 (FP64 with demag),
demag field rel 1e-11 (FP64 chain) and 5e-6 (mixed chain); integration:
identical solver counters and max|dm| <= 1e-6.
"""
import numpy as np
import pytest

import llg
from conftest import rel_err

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _square_hole(prec=llg.DEMAG_FP64, **kw):
    p = llg.default_params(1536, 512, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0, bc=llg.BC_FREE,
                           norm_kind=llg.NORM_REG, demag_precision=prec, **kw)
    g = llg.default_geom(1536, 512, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                         ic_jitter_eps=0.01, init_random_seed=12345)
    return p, llg.build_geometry(g)


def _polycrystal(prec=llg.DEMAG_MIXED):
    p = llg.default_params(1536, 512, demag_mode=llg.DEMAG_OPEN, demag_strength=1.0, windowed=1, chb=0.3,
                           norm_kind=llg.NORM_REG, demag_precision=prec, bc=llg.BC_FREE)
    g = llg.default_geom(1536, 512, geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=72, dead_grain_frac=0.16,
                         grain_z_bias=1.0, ic_kind=llg.IC_TWO_DOMAIN_X, ic_jitter_eps=0.01, init_random_seed=7)
    return p, llg.build_geometry(g)


def _pair(oracle_lib, p, geo):
    ctx = llg.Context(p)
    o = oracle_lib.Oracle(p)
    if p.windowed:
        ctx.set_window(geo["w"], geo["msk3"], geo["nsk3"])
        o.set_window(geo["w"], geo["msk3"], geo["nsk3"])
    else:
        ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
        o.set_active(geo["active"])
    return ctx, o


@pytest.mark.parametrize("case", ["square_hole_fp64", "square_hole_mixed", "polycrystal_mixed"])
def test_operators_at_benchmark_size(oracle_lib, gpu, case):
    import torch
    if case.startswith("square_hole"):
        p, geo = _square_hole(llg.DEMAG_MIXED if case.endswith("mixed") else llg.DEMAG_FP64)
    else:
        p, geo = _polycrystal()
    mixed = p.demag_precision == llg.DEMAG_MIXED
    ctx, o = _pair(oracle_lib, p, geo)
    n3 = geo["y0"].size
    rng = np.random.default_rng(31)
    act3 = np.tile(geo["active"], 3)
    y = geo["y0"] + 0.05 * rng.standard_normal(n3) * act3
    v = rng.standard_normal(n3) * act3
    r = rng.standard_normal(n3)
    gamma = 0.0123
    f_ref = o.rhs(yr := y.copy())
    h_ref = o.hdemag().copy()
    jv_ref = o.jtv(v, yr)
    o.psetup(yr, gamma)
    z_ref = o.psolve(r)
    dy, f = _dev(torch, y), torch.zeros(n3, dtype=torch.float64, device="cuda")
    ctx.rhs(0.0, dy, f)
    h = torch.zeros_like(f)
    ctx.demag_apply(dy, h)
    jv = torch.zeros_like(f)
    ctx.jtv(_dev(torch, v), jv, 0.0, dy)
    ctx.psetup(0.0, dy, f, 0, gamma)
    z = torch.zeros_like(f)
    ctx.psolve(0.0, dy, f, _dev(torch, r), z, gamma)
    torch.cuda.synchronize()
    e = {"y": rel_err(dy.cpu().numpy(), yr), "h": rel_err(h.cpu().numpy(), h_ref),
         "f": rel_err(f.cpu().numpy(), f_ref), "jv": rel_err(jv.cpu().numpy(), jv_ref),
         "z": rel_err(z.cpu().numpy(), z_ref)}
    print(case, " ".join(f"{k} {x:.2e}" for k, x in e.items()))
    assert e["y"] <= 1e-15
    assert e["jv"] <= 1e-13                    # the reference's Jv: no demag term
    if mixed:
        assert e["h"] <= 5e-6
        assert e["f"] <= 5e-5 and e["z"] <= 5e-5   # through the field: FP32-level
    else:
        assert e["h"] <= 1e-11 and e["f"] <= 1e-11 and e["z"] <= 1e-10


@pytest.mark.parametrize("gs", [llg.GS_AUTO, llg.GS_CLASSICAL])
def test_plain_fp64_integration_at_benchmark_size(oracle_lib, gpu, gs):
    """t 0 -> 0.1 of the benchmark film from its seeded state: the GPU
    integrator takes the oracle's steps (GS_AUTO selects modified
    Gram-Schmidt at neq = 2.36e6, as the reference does)."""
    import torch
    p, geo = _square_hole()
    ctx, o = _pair(oracle_lib, p, geo)
    opts = llg.default_solver_opts(gs_type=gs)
    y0 = _dev(torch, geo["y0"])
    ctx.integrator_init(0.0, y0, opts)
    o.integrator_init(geo["y0"], opts)
    yout = torch.zeros_like(y0)
    ctx.integrate(0.1, yout)
    rc, _, yo = o.integrate(0.1)
    assert rc == 0
    torch.cuda.synchronize()
    a, b = ctx.stats(), o.stats()
    print("gs", gs, {k: (a[k], b[k]) for k in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups")})
    for key in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups"):
        assert a[key] == b[key], (key, a[key], b[key])
    assert np.abs(yout.cpu().numpy() - yo).max() <= 1e-6
