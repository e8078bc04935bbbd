"""The compact and the linear-anisotropy + DMI operators against the
reference's OWN kernels of those variants.

oracle/_ref/libref_i6.so is compiled (oracle/Makefile, target ref) from the
reference's src/irregular/2d_fft/2d_i6 sources where they lie: the compact RHS
wrapper f with zero_inactive_kernel and f_kernel_compact (2d_i6.cu:250-397),
JtvProduct / jtv_kernel_compact (jtv.cu:47-183), PrecondSetup / PrecondSolve
with build_J_kernel_compact / apply_P_kernel_compact (precond.cu:98-396) and
the periodic cuFFT demag module.  oracle/_ref/libref_i1.so is the same for
src/irregular/2d_fft/2d_i1: f with normalize_m_kernel and
f_kernel_unified_soa_periodic (linear anisotropy + DMI, 2d_fft.cu:253-440),
JtvProduct / jtv_kernel (jtv.cu:43-119), PrecondSetup / PrecondSolve
(precond.cu:108-372).  The callbacks are called exactly as CVODE would call
them (a vector handle holding a device pointer, the reference's user-data
layout of that variant), with their __constant__ material constants set to
the values of llg_params.  Same seeded inputs on both sides.

Tolerances: normalised state rel 1e-15; RHS, Jv and the block-Jacobi solve
rel 1e-13 without demag; with demag rel 1e-11 (cuFFT against this library's
FFT).  2048x2048 is the compact circle's full size.
"""
import ctypes as C
import os

import numpy as np
import pytest

import llg
from conftest import REPO, rel_err

pytestmark = pytest.mark.gpu

REF_I6 = os.path.join(REPO, "oracle", "_ref", "libref_i6.so")
REF_I1 = os.path.join(REPO, "oracle", "_ref", "libref_i1.so")
VP, D, I = C.c_void_p, C.c_double, C.c_int


def _common(lib):
    lib.Precond_Create.restype = VP
    lib.Precond_Create.argtypes = [I, I, I]
    lib.Precond_Destroy.argtypes = [VP]
    lib.Demag_Init.restype = VP
    lib.Demag_Init.argtypes = [I, I, D, D]
    lib.Demag_GetSelfCoupling.argtypes = [VP, C.POINTER(D), C.POINTER(D), C.POINTER(D)]
    lib.Demag_Destroy.argtypes = [VP]


def _self_coupling(lib, demag):
    n0 = (D * 3)()
    if demag:
        a, b, c = D(), D(), D()
        lib.Demag_GetSelfCoupling(demag, C.byref(a), C.byref(b), C.byref(c))
        n0[:] = (a.value, b.value, c.value)
    return n0


def _ours(p, y, v, r, gamma, setup, dev, zeros):
    ctx = llg.Context(p)
    setup(ctx)
    oy, oydot = dev(y), zeros()
    ctx.rhs(0.0, oy, oydot)
    ojv = zeros()
    ctx.jtv(dev(v), ojv, 0.0, oy)
    ctx.psetup(0.0, oy, oydot, 0, gamma)
    oz = zeros()
    ctx.psolve(0.0, oy, oydot, dev(r), oz, gamma)
    s3 = ctx.demag_self_coupling() if p.demag_mode != llg.DEMAG_OFF else None
    return oy, oydot, ojv, oz, s3


def _check(label, ours, ref, n0, strength):
    import torch
    torch.cuda.synchronize()
    oy, oydot, ojv, oz, s3 = ours
    ry, rydot, rjv, rz = ref
    if s3 is not None:
        assert np.allclose(s3, tuple(n0), rtol=1e-12, atol=1e-15), (s3, tuple(n0))
    tol = 1e-11 if strength > 0 else 1e-13
    errs = {"y": rel_err(oy.cpu().numpy(), ry.cpu().numpy()), "f": rel_err(oydot.cpu().numpy(), rydot.cpu().numpy()),
            "jv": rel_err(ojv.cpu().numpy(), rjv.cpu().numpy()), "psolve": rel_err(oz.cpu().numpy(), rz.cpu().numpy())}
    print(label + ": " + ", ".join(f"{k} {e:.2e}" for k, e in errs.items()))
    assert errs["y"] <= 1e-15
    assert errs["f"] <= tol
    assert errs["jv"] <= 1e-13
    assert errs["psolve"] <= tol


# the reference's 2d_i6 material constants (2d_i6.cu:165-173, jtv.cu:31-34, precond.cu:53-56)
I6 = dict(chk=1.0, che=10.0, alpha=0.2, chg=1.0)


@pytest.mark.skipif(not os.path.exists(REF_I6), reason="reference i6 checker not built (needs the reference tree)")
@pytest.mark.parametrize("ng,ny,strength", [(64, 48, 0.0), (64, 48, 2.0), (45, 27, 1.5), (2048, 2048, 2.0)])
def test_compact_operators_match_reference_kernels(gpu, ng, ny, strength):
    import torch
    lib = C.CDLL(REF_I6)
    _common(lib)
    lib.ref_i6_set_rhs_consts.argtypes = [C.POINTER(D), D, D, D, D]
    lib.ref_i6_rhs.argtypes = [D, VP, VP, VP, VP, I, VP, I, I, I, VP]
    lib.ref_i6_set_jtv_consts.argtypes = [D, D, D, D]
    lib.ref_i6_jtv.argtypes = [VP, VP, VP, VP, I, VP, I, I, I]
    lib.ref_i6_set_precond_consts.argtypes = [D, D, D, D]
    lib.ref_i6_psetup.argtypes = [VP, VP, VP, C.POINTER(D), D, VP, I, VP, I, I, I]
    lib.ref_i6_psolve.argtypes = [VP, VP, VP, VP, I, VP, I, I, I]
    k = I6
    assert lib.ref_i6_set_rhs_consts((D * 3)(1.0, 1.0, 1.0), k["chk"], k["che"], k["alpha"], k["chg"]) == 0
    assert lib.ref_i6_set_jtv_consts(k["chk"], k["che"], k["alpha"], k["chg"]) == 0
    assert lib.ref_i6_set_precond_consts(k["chk"], k["che"], k["alpha"], k["chg"]) == 0

    p = llg.default_params(ng, ny, exec_model=llg.EXEC_COMPACT, bc=llg.BC_PERIODIC, aniso_kind=llg.ANISO_CUBIC,
                           msk=(1.0, 1.0, 1.0), happ=(0.0, 0.0, 0.0), norm_kind=llg.NORM_NONE,
                           demag_mode=llg.DEMAG_PERIODIC if strength > 0 else llg.DEMAG_OFF,
                           demag_strength=strength, demag_thick=1.0, **k)
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_ELLIPSE, init_m=(1.0, -0.0175, 0.0), ic_jitter_eps=0.01)
    geo = llg.build_geometry(g)
    n = ng * ny
    act = geo["active"].astype(bool)
    act3 = np.tile(act.astype(np.float64), 3)
    ids = np.arange(n, dtype=np.int32)
    a_ids, i_ids = ids[act], ids[~act]
    rng = np.random.default_rng(23)
    y = (geo["y0"] + 0.05 * rng.standard_normal(3 * n)) * act3   # hole cells hold 0, as in the reference
    v = rng.standard_normal(3 * n) * act3
    r = rng.standard_normal(3 * n)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()   # noqa: E731
    zeros = lambda: torch.zeros(3 * n, dtype=torch.float64, device="cuda")   # noqa: E731
    da, di = dev(a_ids), dev(i_ids)
    na, ni = len(a_ids), len(i_ids)
    demag = lib.Demag_Init(ng, ny, 1.0, strength) if strength > 0 else None
    assert strength == 0 or demag
    n0 = _self_coupling(lib, demag)
    ry, rydot, rhd = dev(y), zeros(), zeros()
    assert lib.ref_i6_rhs(0.0, ry.data_ptr(), rydot.data_ptr(), rhd.data_ptr(), da.data_ptr(), na, di.data_ptr(), ni,
                          ng, ny, demag) == 0
    rjv = zeros()
    assert lib.ref_i6_jtv(dev(v).data_ptr(), rjv.data_ptr(), ry.data_ptr(), da.data_ptr(), na, di.data_ptr(), ni,
                          ng, ny) == 0
    pd = lib.Precond_Create(ng, ny, n)
    gamma = 0.0173
    assert lib.ref_i6_psetup(pd, ry.data_ptr(), rhd.data_ptr(), n0, gamma, da.data_ptr(), na, di.data_ptr(), ni,
                             ng, ny) == 0
    rz = zeros()
    assert lib.ref_i6_psolve(pd, dev(r).data_ptr(), rz.data_ptr(), da.data_ptr(), na, di.data_ptr(), ni, ng, ny) == 0
    lib.Precond_Destroy(pd)
    if demag:
        lib.Demag_Destroy(demag)
    ours = _ours(p, y, v, r, gamma, lambda ctx: ctx.set_active_ids(a_ids, i_ids), dev, zeros)
    _check(f"i6 {ng}x{ny} strength {strength}", ours, (ry, rydot, rjv, rz), n0, strength)


# the reference's 2d_i1 material constants (2d_fft.cu:156-166, jtv.cu:30-35, precond.cu:58-63);
# cha is also run non-zero
I1 = dict(chk=4.0, che=4.0, alpha=0.2, chg=1.0, chb=0.3)


@pytest.mark.skipif(not os.path.exists(REF_I1), reason="reference i1 checker not built (needs the reference tree)")
@pytest.mark.parametrize("ng,ny,strength,cha", [(64, 48, 0.0, 0.0), (64, 48, 2.0, 0.0), (45, 27, 1.5, 0.25),
                                                (512, 512, 1.0, 0.0)])
def test_linear_dmi_operators_match_reference_kernels(gpu, ng, ny, strength, cha):
    import torch
    lib = C.CDLL(REF_I1)
    _common(lib)
    lib.ref_i1_set_rhs_consts.argtypes = [C.POINTER(D), C.POINTER(D), D, D, D, D, D, D]
    lib.ref_i1_rhs.argtypes = [D, VP, VP, VP, I, I, VP]
    lib.ref_i1_set_jtv_consts.argtypes = [D, D, D, D, D, D]
    lib.ref_i1_jtv.argtypes = [VP, VP, VP, I, I]
    lib.ref_i1_set_precond_consts.argtypes = [D, D, D, D, D, D]
    lib.ref_i1_psetup.argtypes = [VP, VP, VP, C.POINTER(D), D, I, I]
    lib.ref_i1_psolve.argtypes = [VP, VP, VP, I, I]
    k = I1
    axis = (D * 3)(1.0, 0.0, 0.0)   # easy axis and DMI direction along x (the variant's kernels bake these in)
    assert lib.ref_i1_set_rhs_consts(axis, axis, k["chk"], k["che"], k["alpha"], k["chg"], cha, k["chb"]) == 0
    assert lib.ref_i1_set_jtv_consts(k["chk"], k["che"], k["alpha"], k["chg"], cha, k["chb"]) == 0
    assert lib.ref_i1_set_precond_consts(k["chk"], k["che"], k["alpha"], k["chg"], cha, k["chb"]) == 0

    p = llg.default_params(ng, ny, bc=llg.BC_PERIODIC, aniso_kind=llg.ANISO_LINEAR, msk=(1.0, 0.0, 0.0),
                           nsk=(1.0, 0.0, 0.0), happ=(0.0, 0.0, 0.0), norm_kind=llg.NORM_EXACT, cha=cha,
                           demag_mode=llg.DEMAG_PERIODIC if strength > 0 else llg.DEMAG_OFF,
                           demag_strength=strength, demag_thick=1.0, **k)
    g = llg.default_geom(ng, ny, ic_kind=llg.IC_HEAD_ON_STRIPES)
    geo = llg.build_geometry(g)
    n = ng * ny
    rng = np.random.default_rng(29)
    y = geo["y0"] + 0.05 * rng.standard_normal(3 * n)
    v = rng.standard_normal(3 * n)
    r = rng.standard_normal(3 * n)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()   # noqa: E731
    zeros = lambda: torch.zeros(3 * n, dtype=torch.float64, device="cuda")   # noqa: E731
    demag = lib.Demag_Init(ng, ny, 1.0, strength) if strength > 0 else None
    assert strength == 0 or demag
    n0 = _self_coupling(lib, demag)
    ry, rydot, rhd = dev(y), zeros(), zeros()
    assert lib.ref_i1_rhs(0.0, ry.data_ptr(), rydot.data_ptr(), rhd.data_ptr(), ng, ny, demag) == 0
    rjv = zeros()
    assert lib.ref_i1_jtv(dev(v).data_ptr(), rjv.data_ptr(), ry.data_ptr(), ng, ny) == 0
    pd = lib.Precond_Create(ng, ny, n)
    gamma = 0.0211
    assert lib.ref_i1_psetup(pd, ry.data_ptr(), rhd.data_ptr(), n0, gamma, ng, ny) == 0
    rz = zeros()
    assert lib.ref_i1_psolve(pd, dev(r).data_ptr(), rz.data_ptr(), ng, ny) == 0
    lib.Precond_Destroy(pd)
    if demag:
        lib.Demag_Destroy(demag)
    ours = _ours(p, y, v, r, gamma, lambda ctx: ctx.set_mask(np.ones(3 * n)), dev, zeros)
    _check(f"i1 {ng}x{ny} strength {strength} cha {cha}", ours, (ry, rydot, rjv, rz), n0, strength)
