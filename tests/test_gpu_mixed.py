"""Mixed-precision demag (LLG_DEMAG_MIXED) on the GPU, through the C ABI.

The mixed chain runs the row transforms in FP32 and the column stage either
as tensor-core DFT stages (FP16 hi+lo split operands, FP32 accumulation) or,
for column lengths that stage does not cover, as FP32 Stockham transforms.
The FP64 quantities around it (state, norms, Newton update, |m| = 1) are
unchanged.

Tolerances:
  demag field vs the FP64 oracle       rel (2-norm) <= 5e-6
  integrated state vs the FP64 GPU path  max|dm| <= 1e-4 (the mixed form's bar)
    where the dynamics do not amplify perturbations exponentially; where they
    do, the divergence is compared with that of an FP64 run perturbed by 1e-9
"""
import numpy as np
import pytest

import llg
from conftest import rel_err

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


SHAPES = [
    (llg.DEMAG_PERIODIC, 64, 32), (llg.DEMAG_PERIODIC, 45, 27), (llg.DEMAG_OPEN, 96, 40),
    (llg.DEMAG_OPEN, 35, 21), (llg.DEMAG_OPEN, 64, 512), (llg.DEMAG_OPEN, 40, 512),
    (llg.DEMAG_PERIODIC, 32, 1024),
]


@pytest.mark.parametrize("mode,ng,ny", SHAPES)
@pytest.mark.parametrize("windowed", [0, 1])
def test_mixed_demag_matches_fp64_oracle(oracle_lib, gpu, mode, ng, ny, windowed):
    import torch
    p = llg.default_params(ng, ny, demag_mode=mode, demag_strength=3.0, bc=llg.BC_PERIODIC,
                           demag_precision=llg.DEMAG_MIXED)
    rng = np.random.default_rng(11)
    n = ng * ny
    y = rng.uniform(-1.0, 1.0, 3 * n)
    w = rng.uniform(0.0, 1.0, n) if windowed else None
    o = oracle_lib.Oracle(p)
    ref = o.demag(y * np.tile(w, 3)) if windowed else o.demag(y)
    ctx = llg.Context(p)
    dh = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    if windowed:
        ctx.demag_apply(dev(torch, y * np.tile(w, 3)), dh)
    else:
        ctx.demag_apply(dev(torch, y), dh)
    torch.cuda.synchronize()
    err = rel_err(dh.cpu().numpy(), ref)
    print(f"mixed demag {mode} {ng}x{ny} rel err {err:.3e}")
    assert err <= 5e-6


def _hole_demag_run(torch, prec, alpha, strength, t_out):
    ng, ny = 128, 512
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                         ic_jitter_eps=0.01)
    geo = llg.build_geometry(g)
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=strength, alpha=alpha,
                           norm_kind=llg.NORM_REG, demag_precision=prec)
    ctx = llg.Context(p)
    ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
    y0 = dev(torch, geo["y0"])
    ctx.integrator_init(0.0, y0, llg.default_solver_opts())
    yout = torch.zeros_like(y0)
    outs = {}
    for k in range(1, int(round(max(t_out) / 0.1)) + 1):
        ctx.integrate(0.1 * k, yout)
        if any(abs(0.1 * k - t) < 1e-9 for t in t_out):
            torch.cuda.synchronize()
            outs[round(0.1 * k, 6)] = yout.cpu().numpy().copy()
    return outs


def test_mixed_integration_within_1e4_of_fp64_stable(gpu):
    """Periodic 32x1024 film (periodic demag strength 4, so the column stage
    runs on the tensor cores), jittered uniform state, alpha 0.2: the state
    turns over and relaxes, and an FP64 run perturbed by 1e-9 ends 1e-12 from
    the unperturbed one.  At rtol 1e-6 the mixed form stays within 1e-4 of the
    plain FP64 form over t 0 -> 5 (measured: <= 1e-5).  At rtol 1e-4 the two
    forms take a few different accepted steps and differ at the tolerance
    level (~1e-4), which measures the integrator, not the demag precision."""
    import torch
    ng, ny = 32, 1024
    geo = llg.build_geometry(llg.default_geom(ng, ny, ic_jitter_eps=0.01))
    outs = {}
    for prec in (llg.DEMAG_FP64, llg.DEMAG_MIXED):
        p = llg.default_params(ng, ny, bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_PERIODIC, demag_strength=4.0,
                               alpha=0.2, norm_kind=llg.NORM_REG, demag_precision=prec)
        ctx = llg.Context(p)
        y0 = dev(torch, geo["y0"])
        ctx.integrator_init(0.0, y0, llg.default_solver_opts(rtol=1e-6, atol=1e-8))
        yout = torch.zeros_like(y0)
        outs[prec] = []
        for k in range(1, 51):
            ctx.integrate(0.1 * k, yout)
            if k % 10 == 0:
                torch.cuda.synchronize()
                outs[prec].append(yout.cpu().numpy().copy())
    for i, (a, b) in enumerate(zip(outs[llg.DEMAG_FP64], outs[llg.DEMAG_MIXED])):
        dm = np.abs(b - a).max()
        print(f"stable film t={i + 1}: mixed vs fp64 max|dm| = {dm:.3e}")
        assert dm <= 1e-4


def test_mixed_divergence_tracks_physical_sensitivity(gpu):
    """alpha = 0.02: the jittered uniform state under demag is unstable and
    any perturbation grows exponentially.  The mixed form meets 1e-4 early
    (t = 0.5); later its distance from FP64 grows at the same rate as a plain
    FP64 run whose demag strength is perturbed by 1e-9 relative."""
    import torch
    ts = (0.1, 0.5, 2.0)
    a = _hole_demag_run(torch, llg.DEMAG_FP64, 0.02, 4.0, ts)
    b = _hole_demag_run(torch, llg.DEMAG_MIXED, 0.02, 4.0, ts)
    c = _hole_demag_run(torch, llg.DEMAG_FP64, 0.02, 4.0 * (1 + 1e-9), ts)
    dm = {t: np.abs(b[t] - a[t]).max() for t in ts}
    dc = {t: np.abs(c[t] - a[t]).max() for t in ts}
    for t in ts:
        print(f"alpha 0.02 t={t}: mixed-fp64 {dm[t]:.3e}   fp64(strength*(1+1e-9))-fp64 {dc[t]:.3e}")
    assert dm[0.5] <= 1e-4
    growth_mixed = dm[2.0] / dm[0.1]
    growth_ctl = dc[2.0] / dc[0.1]
    assert growth_mixed <= 10.0 * growth_ctl


@pytest.mark.parametrize("a_mn_major", [0, 1])
def test_tcgen05_gemm_known_answer(gpu, a_mn_major):
    """The descriptor encodings the tensor-core column stage relies on: a
    128x64x64 FP16 GEMM into tensor memory (A K-major or MN-major) against a
    host FP64 product.  FP16 inputs are exact, so only FP32 accumulation
    rounding remains (<= 2^-21 relative to sum |a b|)."""
    err = llg.selftest_tcgen05(a_mn_major)
    print("tcgen05 self-test", a_mn_major, err)
    assert 0.0 <= err < 1e-6


@pytest.mark.parametrize("scale", [2.0 ** -20, 2.0 ** 12])
def test_mixed_demag_accuracy_independent_of_magnitude(oracle_lib, gpu, scale):
    """The column stage splits every FP32 operand into an FP16 high part and a
    2^11-scaled FP16 remainder, with exact power-of-two scalings keeping both
    in FP16's normal range; so the chain's relative accuracy must not depend
    on the magnitude of the input (tiny inputs would otherwise land in FP16's
    subnormal range and lose their low bits, large ones would overflow).
    Field of m * scale vs the FP64 oracle, rel <= 5e-6, on an open 64x512
    film (tensor-core columns of length 1024)."""
    import torch
    ng, ny = 64, 512
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=3.0, bc=llg.BC_PERIODIC,
                           demag_precision=llg.DEMAG_MIXED)
    rng = np.random.default_rng(12)
    y = rng.uniform(-1.0, 1.0, 3 * ng * ny) * scale
    ref = oracle_lib.Oracle(p).demag(y)
    ctx = llg.Context(p)
    dh = torch.zeros(3 * ng * ny, dtype=torch.float64, device="cuda")
    ctx.demag_apply(dev(torch, y), dh)
    torch.cuda.synchronize()
    err = rel_err(dh.cpu().numpy(), ref)
    print(f"mixed demag, input scale {scale:g}: rel err {err:.3e}")
    assert err <= 5e-6
