"""GPU parity: libllg.so (CUDA, through the C ABI) against the FP64 oracle.

Tolerances (FP64 on both sides; differences come only from FMA contraction,
reduction order and the FFT algorithm):
  per-cell operators (RHS without demag, Jv, P solve)   rel 1e-13
  demag chain (FFT, 81-point tensor on device vs host)  rel 1e-11
  integrated state (config 0, t 0→100, rtol 1e-4)        max|Δm| <= 1e-6
"""
import ctypes as C
import os

import numpy as np
import pytest

import llg
from conftest import REPO, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    # name, ng, ny, param overrides, geometry overrides
    ("cfg0_local_free", 128, 64, dict(), dict(ic_jitter_eps=0.01)),
    ("odd_periodic_cubic", 37, 23, dict(bc=llg.BC_PERIODIC, aniso_kind=llg.ANISO_CUBIC, msk=(1, 1, 1), che=50.0,
                                        alpha=0.2, chk=1.0, norm_kind=llg.NORM_REG),
     dict(geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.2, ic_jitter_eps=0.05)),
    ("hole_open_demag", 64, 48, dict(bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0),
     dict(geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125, ic_jitter_eps=0.01)),
    ("linear_dmi_periodic_demag", 48, 30, dict(bc=llg.BC_PERIODIC, chb=0.3, chk=4.0, che=4.0, alpha=0.2,
                                               demag_mode=llg.DEMAG_PERIODIC, demag_strength=2.0,
                                               norm_kind=llg.NORM_EXACT),
     dict(ic_kind=llg.IC_HEAD_ON_STRIPES)),
    ("ellipse_compact", 40, 40, dict(exec_model=llg.EXEC_COMPACT, bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_OPEN,
                                     demag_strength=2.0, aniso_kind=llg.ANISO_CUBIC, msk=(1, 1, 1)),
     dict(geometry_kind=llg.GEOM_ELLIPSE, ic_kind=llg.IC_VORTEX, ic_jitter_eps=0.01)),
    ("polycrystal_windowed", 60, 36, dict(bc=llg.BC_PERIODIC, windowed=1, chb=0.6, che=4.0, demag_mode=llg.DEMAG_OPEN,
                                          demag_strength=1.0, norm_kind=llg.NORM_REG),
     dict(geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=12, dead_grain_frac=0.2, ic_kind=llg.IC_TWO_DOMAIN_X,
          ic_jitter_eps=0.01)),
]


def setup_case(oracle_lib, torch, ng, ny, pover, gover):
    p = llg.default_params(ng, ny, **pover)
    g = llg.default_geom(ng, ny, **gover)
    geo = llg.build_geometry(g)
    ctx = llg.Context(p)
    o = oracle_lib.Oracle(p)
    n = ng * ny
    act = geo["active"]
    if p.windowed:
        ctx.set_window(geo["w"], geo["msk3"], geo["nsk3"])
        o.set_window(geo["w"], geo["msk3"], geo["nsk3"])
    elif p.exec_model == llg.EXEC_COMPACT:
        ids = np.arange(n, dtype=np.int32)
        ctx.set_active_ids(ids[act == 1], ids[act == 0])
        o.set_active(act)
    else:
        ctx.set_mask(np.tile(act.astype(np.float64), 3))
        o.set_active(act)
    return p, geo, ctx, o


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


@pytest.mark.parametrize("name,ng,ny,pover,gover", CASES, ids=[c[0] for c in CASES])
def test_rhs_matches_oracle(oracle_lib, gpu, name, ng, ny, pover, gover):
    import torch
    p, geo, ctx, o = setup_case(oracle_lib, torch, ng, ny, pover, gover)
    rng = np.random.default_rng(3)
    y = geo["y0"] + 0.05 * rng.standard_normal(3 * ng * ny) * np.tile(geo["active"], 3)
    yd_ref = o.rhs(y_ref := y.copy())
    dy = dev(torch, y)
    dyd = torch.zeros_like(dy)
    ctx.rhs(0.0, dy, dyd)
    torch.cuda.synchronize()
    assert rel_err(dy.cpu().numpy(), y_ref) < 1e-15   # in-place normalisation
    tol = 1e-11 if p.demag_mode != llg.DEMAG_OFF else 1e-13
    if p.demag_mode != llg.DEMAG_OFF:
        hd = torch.empty_like(dy)
        ctx.demag_apply(dy, hd)   # dy already normalised, same input as the oracle's
        torch.cuda.synchronize()
        assert rel_err(hd.cpu().numpy(), o.hdemag()) < 1e-11
    assert rel_err(dyd.cpu().numpy(), yd_ref) < tol


@pytest.mark.parametrize("name,ng,ny,pover,gover", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("jv_mode", [llg.JV_REFERENCE, llg.JV_FULL_FIELD, llg.JV_FULL_DEMAG])
def test_jtv_matches_oracle(oracle_lib, gpu, name, ng, ny, pover, gover, jv_mode):
    import torch
    pover = dict(pover, jv_mode=jv_mode)
    p, geo, ctx, o = setup_case(oracle_lib, torch, ng, ny, pover, gover)
    rng = np.random.default_rng(4)
    n = ng * ny
    y = geo["y0"] + 0.05 * rng.standard_normal(3 * n) * np.tile(geo["active"], 3)
    v = rng.standard_normal(3 * n)
    o.rhs(y.copy())  # demag field for JV_FULL_FIELD
    dy = dev(torch, y)
    ctx.rhs(0.0, dy.clone(), torch.zeros_like(dy))
    ref = o.jtv(v, y)
    dv = dev(torch, v)
    djv = torch.zeros_like(dv)
    ctx.jtv(dv, djv, 0.0, dy)
    torch.cuda.synchronize()
    tol = 1e-11 if (p.demag_mode != llg.DEMAG_OFF and jv_mode != llg.JV_REFERENCE) else 1e-13
    assert rel_err(djv.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("name,ng,ny,pover,gover", CASES, ids=[c[0] for c in CASES])
def test_psetup_psolve_match_oracle(oracle_lib, gpu, name, ng, ny, pover, gover):
    import torch
    p, geo, ctx, o = setup_case(oracle_lib, torch, ng, ny, pover, gover)
    rng = np.random.default_rng(5)
    n = ng * ny
    y = geo["y0"] + 0.05 * rng.standard_normal(3 * n) * np.tile(geo["active"], 3)
    yn = y.copy()
    o.rhs(yn)
    gamma = 0.0731
    o.psetup(yn, gamma)
    dy = dev(torch, y)
    ctx.rhs(0.0, dy, torch.zeros_like(dy))
    jcur = ctx.psetup(0.0, dy, None, 0, gamma)
    assert jcur == 1
    r = rng.standard_normal(3 * n)
    z_ref = o.psolve(r)
    dz = torch.zeros_like(dy)
    ctx.psolve(0.0, dy, None, dev(torch, r), dz, gamma)
    torch.cuda.synchronize()
    tol = 1e-10 if p.demag_mode != llg.DEMAG_OFF else 1e-12
    assert rel_err(dz.cpu().numpy(), z_ref) < tol


@pytest.mark.parametrize("mode,ng,ny", [(llg.DEMAG_PERIODIC, 64, 32), (llg.DEMAG_PERIODIC, 45, 27),
                                        (llg.DEMAG_OPEN, 96, 40), (llg.DEMAG_OPEN, 35, 21),
                                        (llg.DEMAG_PERIODIC, 7, 11), (llg.DEMAG_OPEN, 1, 5)])
def test_demag_matches_oracle(oracle_lib, gpu, mode, ng, ny):
    import torch
    p = llg.default_params(ng, ny, demag_mode=mode, demag_strength=3.0, bc=llg.BC_PERIODIC)
    ctx = llg.Context(p)
    o = oracle_lib.Oracle(p)
    y = np.random.default_rng(9).standard_normal(3 * ng * ny)
    dh = torch.zeros(3 * ng * ny, dtype=torch.float64, device="cuda")
    ctx.demag_apply(dev(torch, y), dh)
    torch.cuda.synchronize()
    assert rel_err(dh.cpu().numpy(), o.demag(y)) < 1e-11
    assert rel_err(np.array(ctx.demag_self_coupling()), np.array(o.demag_self())) < 1e-13
    for comp, dx, dyy in ((0, 0, 0), (4, 3, -2), (1, 2, 1), (8, -1, 0)):
        if mode == llg.DEMAG_OPEN and (abs(dx) >= ng or abs(dyy) >= ny):
            continue  # padding lines: never touched by the linear convolution
        assert abs(ctx.demag_tensor(comp, dx, dyy) - o.tensor(comp, dx, dyy)) < 1e-13


REF_SO = os.path.join(REPO, "oracle", "_ref", "libref_demag.so")


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference demag module not built (needs the reference tree)")
@pytest.mark.parametrize("ng,ny,strength", [(64, 64, 2.0), (128, 32, 4.0), (96, 48, 1.0)])
@pytest.mark.parametrize("windowed", [0, 1])
def test_demag_matches_reference_cufft_module(gpu, ng, ny, strength, windowed):
    """The reference's own demag_fft.cu (cuFFT D2Z/Z2D, periodic), compiled
    from its sources into oracle/_ref, against Demag_* of libllg.so."""
    import torch
    ref = C.CDLL(REF_SO)
    ref.Demag_Init.restype = C.c_void_p
    ref.Demag_Init.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
    ref.Demag_Apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    ref.Demag_ApplyWindowed.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    ref.Demag_GetSelfCoupling.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3
    ref.Demag_Destroy.argtypes = [C.c_void_p]
    mine = llg.load()
    mine.Demag_Init.restype = C.c_void_p
    mine.Demag_Init.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double]
    mine.Demag_Apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    mine.Demag_ApplyWindowed.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    mine.Demag_GetSelfCoupling.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3
    mine.Demag_Destroy.argtypes = [C.c_void_p]
    dr = ref.Demag_Init(ng, ny, 1.0, strength)
    dm = mine.Demag_Init(ng, ny, 1.0, strength)
    assert dr and dm
    rng = np.random.default_rng(21)
    y = dev(torch, rng.standard_normal(3 * ng * ny))
    w = dev(torch, rng.uniform(0.0, 1.0, ng * ny))
    hr = torch.zeros_like(y)
    hm = torch.zeros_like(y)
    if windowed:
        ref.Demag_ApplyWindowed(dr, y.data_ptr(), w.data_ptr(), hr.data_ptr())
        mine.Demag_ApplyWindowed(dm, y.data_ptr(), w.data_ptr(), hm.data_ptr())
    else:
        ref.Demag_Apply(dr, y.data_ptr(), hr.data_ptr())
        mine.Demag_Apply(dm, y.data_ptr(), hm.data_ptr())
    torch.cuda.synchronize()
    assert rel_err(hm.cpu().numpy(), hr.cpu().numpy()) < 1e-10
    a = [C.c_double() for _ in range(3)]
    b = [C.c_double() for _ in range(3)]
    ref.Demag_GetSelfCoupling(dr, *[C.byref(x) for x in a])
    mine.Demag_GetSelfCoupling(dm, *[C.byref(x) for x in b])
    for x, z in zip(a, b):
        assert abs(x.value - z.value) <= 1e-12 * abs(x.value)
    ref.Demag_Destroy(dr)
    mine.Demag_Destroy(dm)


def test_compact_and_dense_models_agree(oracle_lib, gpu):
    import torch
    ng = ny = 48
    base = dict(bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_OPEN, demag_strength=2.0)
    gover = dict(geometry_kind=llg.GEOM_ELLIPSE, ic_kind=llg.IC_VORTEX, ic_jitter_eps=0.01)
    _, geo, c1, _ = setup_case(oracle_lib, torch, ng, ny, dict(base), gover)
    _, _, c2, _ = setup_case(oracle_lib, torch, ng, ny, dict(base, exec_model=llg.EXEC_COMPACT), gover)
    y = dev(torch, geo["y0"])
    a, b = torch.zeros_like(y), torch.zeros_like(y)
    c1.rhs(0.0, y.clone(), a)
    c2.rhs(0.0, y.clone(), b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_vector_ops_and_deterministic_reductions(gpu):
    import torch
    p = llg.default_params(333, 129)
    ctx = llg.Context(p)
    n = 3 * 333 * 129
    rng = np.random.default_rng(0)
    xs = [rng.standard_normal(n) for _ in range(7)]
    dxs = [dev(torch, x) for x in xs]
    got = ctx.dot_multi(dxs[0], dxs)
    ref = [float(np.dot(xs[0], x)) for x in xs]
    assert max(abs(g - r) / max(abs(r), 1.0) for g, r in zip(got, ref)) < 1e-12
    for _ in range(3):
        assert ctx.dot_multi(dxs[0], dxs) == got  # bitwise reproducible
    z = torch.zeros_like(dxs[0])
    coef = [0.5, -1.25, 2.0, 0.1]
    ctx.linear_combination(coef, dxs[:4], z)
    torch.cuda.synchronize()
    assert rel_err(z.cpu().numpy(), sum(c * x for c, x in zip(coef, xs[:4]))) < 1e-14
    w = np.abs(xs[1]) + 0.1
    wr = ctx.wrms_norm(dxs[2], dev(torch, w))
    assert abs(wr - np.sqrt(np.mean((xs[2] * w) ** 2))) < 1e-12 * wr


def run_integration(oracle_lib, p, geo, t_end, dt_out, opts, set_geom):
    import torch
    ctx = llg.Context(p)
    o = oracle_lib.Oracle(p)
    set_geom(ctx, o)
    y0 = dev(torch, geo["y0"])
    ctx.integrator_init(0.0, y0, opts)
    o.integrator_init(geo["y0"], opts)
    yout = torch.zeros_like(y0)
    nout = int(round(t_end / dt_out))
    for k in range(1, nout + 1):
        t = ctx.integrate(dt_out * k, yout)
        rc, t_o, y_o = o.integrate(dt_out * k)
        assert rc == 0
    torch.cuda.synchronize()
    return yout.cpu().numpy(), y_o, ctx.stats(), o.stats()


def test_integrator_config0_matches_oracle(oracle_lib, gpu):
    """The reference's CPU-runnable film: 128x64, free edges, A=1, k=0.1 (+x), h=(0,0,0.05),
    alpha=0.02, jittered uniform IC (srand 12345), rtol 1e-4, atol 1e-6,
    SPGMR(5) + block-Jacobi, t 0→100 in 0.1 output intervals."""
    p = llg.default_params(128, 64)
    geo = llg.build_geometry(llg.default_geom(128, 64, ic_jitter_eps=0.01))
    opts = llg.default_solver_opts(rtol=1e-4, atol=1e-6, maxl=5)
    yg, yo, sg, so = run_integration(oracle_lib, p, geo, 100.0, 0.1, opts, lambda c, o: None)
    dm = np.abs(yg - yo).max()
    print("config0 max|dm| =", dm, "gpu", sg, "oracle", so)
    assert dm <= 1e-6
    for k in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups"):
        assert sg[k] == so[k], (k, sg[k], so[k])


def test_integrator_hole_demag_matches_oracle(oracle_lib, gpu):
    """Square hole + open demag (config 1 physics) on a small grid, t 0→5."""
    ng, ny = 48, 32
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0, bc=llg.BC_PERIODIC)
    geo = llg.build_geometry(llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                                              ic_jitter_eps=0.01))
    act = geo["active"]

    def sg(ctx, o):
        ctx.set_mask(np.tile(act.astype(np.float64), 3))
        o.set_active(act)

    opts = llg.default_solver_opts(rtol=1e-4, atol=1e-6, maxl=5)
    yg, yo, s1, s2 = run_integration(oracle_lib, p, geo, 5.0, 0.1, opts, sg)
    dm = np.abs(yg - yo).max()
    print("hole+demag max|dm| =", dm, s1, s2)
    assert dm <= 1e-6


@pytest.mark.parametrize("bc,jv_mode", [(llg.BC_FREE, llg.JV_FULL_FIELD), (llg.BC_PERIODIC, llg.JV_FULL_FIELD),
                                        (llg.BC_FREE, llg.JV_REFERENCE)],
                         ids=["free-fullfield", "periodic-fullfield", "free-reference"])
def test_integrator_ragged_grid_matches_oracle(oracle_lib, gpu, bc, jv_mode):
    """A 45x27 film with a hole and open demag, t 0→2: partial 32x8 tiles at
    both grid edges, both boundary rules (zero-filled or wrapped halo) and
    both Jacobian field models (the full-field one stages the demag field of
    every tile), through the persistent Arnoldi operator, against the oracle."""
    ng, ny = 45, 27
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=2.0, bc=bc, jv_mode=jv_mode)
    geo = llg.build_geometry(llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                                              ic_jitter_eps=0.01))
    act = geo["active"]

    def sg(ctx, o):
        ctx.set_mask(np.tile(act.astype(np.float64), 3))
        o.set_active(act)

    opts = llg.default_solver_opts(rtol=1e-4, atol=1e-6, maxl=5)
    yg, yo, s1, s2 = run_integration(oracle_lib, p, geo, 2.0, 0.1, opts, sg)
    dm = np.abs(yg - yo).max()
    print("ragged", bc, jv_mode, "max|dm| =", dm, s1, s2)
    assert dm <= 1e-6
    assert s1["nst"] == s2["nst"]


# ── spin-wave slit: soft source on one column, absorbing edge layers ──────
def _slit(oracle_lib, ng=96, ny=48, **pover):
    p = llg.slit_params(ng, ny, pml_cells=8, **pover)
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_SLIT, init_m=(0.0, 0.0, 1.0), ic_jitter_eps=0.01)
    geo = llg.build_geometry(g)
    ctx = llg.Context(p)
    ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
    o = oracle_lib.Oracle(p)
    o.set_active(geo["active"])
    return p, geo, ctx, o


@pytest.mark.parametrize("t", [0.0, 4.3, 31.7])
def test_slit_rhs_with_source_and_absorbing_layers(oracle_lib, gpu, t):
    """src/slit/2d_slit.cu:255-360: h_x += H ramp(t) sin(omega t) on the source
    column, alpha ramped towards the x edges, periodic demag strength 1."""
    import torch
    p, geo, ctx, o = _slit(oracle_lib)
    rng = np.random.default_rng(8)
    y = geo["y0"] + 0.05 * rng.standard_normal(geo["y0"].size) * np.tile(geo["active"], 3)
    ref = o.rhs(y.copy(), t)
    dy = dev(torch, y)
    dyd = torch.zeros_like(dy)
    ctx.rhs(t, dy, dyd)
    torch.cuda.synchronize()
    assert rel_err(dyd.cpu().numpy(), ref) < 1e-11
    # without the source and the layers the RHS differs (the terms are live)
    p0 = llg.slit_params(96, 48, pml_cells=0, src_amp=0.0)
    o0 = oracle_lib.Oracle(p0)
    o0.set_active(geo["active"])
    if t > 0.0:
        assert np.abs(o0.rhs(y.copy(), t) - ref).max() > 1e-6


def test_slit_integration_matches_oracle(oracle_lib, gpu):
    """A driven slit film over t 0 -> 2 (source ramping up): the same BDF
    step sequence as the oracle (counters equal) and max|dm| <= 1e-6."""
    import torch
    p, geo, ctx, o = _slit(oracle_lib, src_ramp=1.0, src_amp=0.5)
    opts = llg.default_solver_opts()
    y0 = dev(torch, geo["y0"])
    ctx.integrator_init(0.0, y0, opts)
    o.integrator_init(geo["y0"], opts)
    yout = torch.zeros_like(y0)
    for k in range(1, 21):
        ctx.integrate(0.1 * k, yout)
        rc, _, yo = o.integrate(0.1 * k)
        assert rc == 0
    torch.cuda.synchronize()
    a, b = ctx.stats(), o.stats()
    for key in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups"):
        assert a[key] == b[key], (key, a[key], b[key])
    assert np.abs(yout.cpu().numpy() - yo).max() <= 1e-6
    # the source drove the film: mx on the source column moved
    n = p.ng * p.ny
    col = yout.cpu().numpy()[:n].reshape(p.ny, p.ng)[:, p.src_col]
    assert np.abs(col).max() > 1e-3


# ── the demag derivative in Jv (LLG_JV_FULL_DEMAG) ──────────────────────────
@pytest.mark.parametrize("windowed", [0, 1])
def test_full_demag_jv_is_the_derivative_of_f(oracle_lib, gpu, windowed):
    """Without normalisation inside f, f is the LLG torque of the full field
    and LLG_JV_FULL_DEMAG must be its exact derivative: against a central
    difference (f(y + e v) - f(y - e v)) / 2e the error is O(e^2), while
    the reference's Jv (no demag term) is off by the demag part."""
    import torch
    ng, ny = 48, 40
    pover = dict(bc=llg.BC_FREE, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0, norm_kind=llg.NORM_NONE,
                 windowed=windowed)
    gover = (dict(geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=8, dead_grain_frac=0.25, ic_jitter_eps=0.05)
             if windowed else dict(geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125, ic_jitter_eps=0.05))
    rng = np.random.default_rng(21)
    errs = {}
    for mode in (llg.JV_FULL_DEMAG, llg.JV_FULL_FIELD):
        p, geo, ctx, o = setup_case(oracle_lib, torch, ng, ny, dict(pover, jv_mode=mode), gover)
        n = ng * ny
        y = geo["y0"].copy()
        v = rng.standard_normal(3 * n) * np.tile(geo["active"], 3) if mode == llg.JV_FULL_DEMAG else v
        eps = 1e-5
        fp, fm, f0 = (torch.zeros(3 * n, dtype=torch.float64, device="cuda") for _ in range(3))
        ctx.rhs(0.0, dev(torch, y + eps * v), fp)
        ctx.rhs(0.0, dev(torch, y - eps * v), fm)
        dy = dev(torch, y)
        ctx.rhs(0.0, dy, f0)   # leaves h_demag(y) for the full field
        djv = torch.zeros_like(dy)
        ctx.jtv(dev(torch, v), djv, 0.0, dy)
        torch.cuda.synchronize()
        fd = ((fp - fm) / (2 * eps)).cpu().numpy()
        errs[mode] = rel_err(djv.cpu().numpy(), fd)
    print(f"windowed={windowed}: |Jv - FD| rel: full demag {errs[llg.JV_FULL_DEMAG]:.2e}, "
          f"without the demag derivative {errs[llg.JV_FULL_FIELD]:.2e}")
    assert errs[llg.JV_FULL_DEMAG] < 1e-7
    assert errs[llg.JV_FULL_FIELD] > 1e-3


def test_full_demag_jacobian_integration_matches_oracle(oracle_lib, gpu):
    """The integrator with the demag derivative in its Krylov operator (one
    more demag evaluation per Arnoldi step) takes the oracle's step sequence;
    GMRES iterations per Newton iteration are reported beside the
    reference's Jacobian."""
    import torch
    ng, ny = 64, 48
    gover = dict(geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125, ic_jitter_eps=0.01)
    its = {}
    for mode in (llg.JV_REFERENCE, llg.JV_FULL_DEMAG):
        p, geo, ctx, o = setup_case(oracle_lib, torch, ng, ny, dict(bc=llg.BC_FREE, demag_mode=llg.DEMAG_OPEN,
                                                                     demag_strength=8.0, norm_kind=llg.NORM_REG,
                                                                     jv_mode=mode), gover)
        opts = llg.default_solver_opts()
        y0 = dev(torch, geo["y0"])
        ctx.integrator_init(0.0, y0, opts)
        o.integrator_init(geo["y0"], opts)
        yout = torch.zeros_like(y0)
        for k in range(1, 11):
            ctx.integrate(0.1 * k, yout)
            rc, _, yo = o.integrate(0.1 * k)
            assert rc == 0
        torch.cuda.synchronize()
        a, b = ctx.stats(), o.stats()
        for key in ("nst", "nfe", "nni", "nli", "netf", "ncfn", "nsetups"):
            assert a[key] == b[key], (mode, key, a[key], b[key])
        assert np.abs(yout.cpu().numpy() - yo).max() <= 1e-6
        its[mode] = a["nli"] / a["nni"]
    print(f"GMRES iterations per Newton iteration, strength 8: reference Jv {its[llg.JV_REFERENCE]:.3f}, "
          f"with the demag derivative {its[llg.JV_FULL_DEMAG]:.3f}")
    assert its[llg.JV_FULL_DEMAG] <= its[llg.JV_REFERENCE] + 1e-12


# Every compile-time transform length (1024, 2048, 3072, 4096: fixed_radices,
# dev_fft.cuh) in the row and in the column direction, open and periodic,
# against the oracle: FP64 rel 1e-11, the mixed chain (FP32 rows, FP32 or
# tensor-core columns) rel 5e-6.
FIXED_SHAPES = [(llg.DEMAG_OPEN, 512, 24), (llg.DEMAG_OPEN, 1024, 12), (llg.DEMAG_OPEN, 1536, 8),
                (llg.DEMAG_OPEN, 2048, 6), (llg.DEMAG_PERIODIC, 3072, 5), (llg.DEMAG_OPEN, 20, 512),
                (llg.DEMAG_OPEN, 12, 1024), (llg.DEMAG_OPEN, 6, 2048), (llg.DEMAG_PERIODIC, 9, 4096)]


@pytest.mark.parametrize("prec", [llg.DEMAG_FP64, llg.DEMAG_MIXED])
@pytest.mark.parametrize("mode,ng,ny", FIXED_SHAPES)
def test_demag_fixed_plan_lengths_match_oracle(oracle_lib, gpu, mode, ng, ny, prec):
    import torch
    p = llg.default_params(ng, ny, demag_mode=mode, demag_strength=2.0, bc=llg.BC_PERIODIC, demag_precision=prec)
    ctx = llg.Context(p)
    o = oracle_lib.Oracle(p)
    y = np.random.default_rng(21).uniform(-1.0, 1.0, 3 * ng * ny)
    dh = torch.zeros(3 * ng * ny, dtype=torch.float64, device="cuda")
    ctx.demag_apply(dev(torch, y), dh)
    torch.cuda.synchronize()
    err = rel_err(dh.cpu().numpy(), o.demag(y))
    print(f"{'open' if mode == llg.DEMAG_OPEN else 'periodic'} {ng}x{ny} "
          f"{'FP64' if prec == llg.DEMAG_FP64 else 'mixed'}: rel err {err:.2e}")
    assert err < (1e-11 if prec == llg.DEMAG_FP64 else 5e-6)
