"""The per-cell operators against the reference's OWN kernels.

oracle/_ref/libref_i2.so is compiled (oracle/Makefile, target ref) from the
reference's src/irregular/2d_fft/2d_i2 sources where they lie: the RHS
wrapper f with normalize_m_kernel and f_kernel_unified_soa_periodic
(2d_fft.cu:262-411), JtvProduct / jtv_kernel (jtv.cu:49-149),
PrecondSetup / PrecondSolve with build_J_kernel / apply_P_kernel
(precond.cu:119-384) and the periodic cuFFT demag module (demag_fft.cu).
The reference's callbacks are called exactly as CVODE would call them (a
vector handle holding a device pointer, the reference's user-data layout),
with its __constant__ material constants set to the same values as
llg_params.  Same seeded inputs on both sides.

Tolerances: normalised state rel 1e-15; RHS, Jv and the block-Jacobi solve
rel 1e-13 without demag; with demag rel 1e-11 (cuFFT against this library's
FFT).  At 1536x512 the same checks run on the reference method's full size.
"""
import ctypes as C
import os

import numpy as np
import pytest

import llg
from conftest import REPO, rel_err

pytestmark = pytest.mark.gpu

REF_SO = os.path.join(REPO, "oracle", "_ref", "libref_i2.so")
needs_ref = pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference i2 checker not built "
                                                                  "(needs the reference tree)")
# the reference's 2d_i2 material constants (2d_fft.cu:169-177, jtv.cu:36-41, precond.cu:65-70)
CHK, CHE, ALPHA, CHG = 1.0, 50.0, 0.2, 1.0


def _ref():
    lib = C.CDLL(REF_SO)
    VP, D, I = C.c_void_p, C.c_double, C.c_int
    lib.ref_i2_set_rhs_consts.argtypes = [C.POINTER(D), D, D, D, D]
    lib.ref_i2_rhs.argtypes = [D, VP, VP, VP, VP, I, I, VP]
    lib.ref_i2_set_jtv_consts.argtypes = [D, D, D, D]
    lib.ref_i2_jtv.argtypes = [VP, VP, VP, VP, I, I]
    lib.ref_i2_set_precond_consts.argtypes = [D, D, D, D]
    lib.ref_i2_psetup.argtypes = [VP, VP, VP, C.POINTER(D), D, I, I]
    lib.ref_i2_psolve.argtypes = [VP, VP, VP, VP, I, I]
    lib.Precond_Create.restype = VP
    lib.Precond_Create.argtypes = [I, I, I]
    lib.Precond_Destroy.argtypes = [VP]
    lib.Demag_Init.restype = VP
    lib.Demag_Init.argtypes = [I, I, D, D]
    lib.Demag_GetSelfCoupling.argtypes = [VP, C.POINTER(D), C.POINTER(D), C.POINTER(D)]
    lib.Demag_Destroy.argtypes = [VP]
    msk = (D * 3)(1.0, 1.0, 1.0)
    assert lib.ref_i2_set_rhs_consts(msk, CHK, CHE, ALPHA, CHG) == 0
    assert lib.ref_i2_set_jtv_consts(CHK, CHE, ALPHA, CHG) == 0
    assert lib.ref_i2_set_precond_consts(CHK, CHE, ALPHA, CHG) == 0
    return lib


def _case(ng, ny, strength):
    p = llg.default_params(ng, ny, bc=llg.BC_PERIODIC, aniso_kind=llg.ANISO_CUBIC, msk=(1.0, 1.0, 1.0), chk=CHK,
                           che=CHE, alpha=ALPHA, chg=CHG, happ=(0.0, 0.0, 0.0), norm_kind=llg.NORM_REG,
                           demag_mode=llg.DEMAG_PERIODIC if strength > 0 else llg.DEMAG_OFF,
                           demag_strength=strength, demag_thick=1.0)
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                         init_m=(1.0, -0.0175, 0.0), ic_jitter_eps=0.01)
    geo = llg.build_geometry(g)
    return p, geo


@needs_ref
@pytest.mark.parametrize("ng,ny,strength", [(96, 40, 0.0), (96, 40, 2.0), (45, 27, 1.5), (1536, 512, 4.0)])
def test_operators_match_reference_kernels(gpu, ng, ny, strength):
    import torch
    lib = _ref()
    p, geo = _case(ng, ny, strength)
    n = ng * ny
    act3 = np.tile(geo["active"].astype(np.float64), 3)
    rng = np.random.default_rng(17)
    y = (geo["y0"] + 0.05 * rng.standard_normal(3 * n)) * act3   # hole cells hold 0, as in the reference
    v = rng.standard_normal(3 * n) * act3
    r = rng.standard_normal(3 * n)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()   # noqa: E731
    zeros = lambda: torch.zeros(3 * n, dtype=torch.float64, device="cuda")   # noqa: E731
    demag = lib.Demag_Init(ng, ny, 1.0, strength) if strength > 0 else None
    assert strength == 0 or demag
    n0 = (C.c_double * 3)()
    if demag:
        nx0, ny0, nz0 = C.c_double(), C.c_double(), C.c_double()
        lib.Demag_GetSelfCoupling(demag, C.byref(nx0), C.byref(ny0), C.byref(nz0))
        n0[:] = (nx0.value, ny0.value, nz0.value)
    ymsk = dev(act3)
    # reference: f (normalise, demag, RHS), JtvProduct, PrecondSetup / PrecondSolve
    ry, rydot, rhd = dev(y), zeros(), zeros()
    assert lib.ref_i2_rhs(0.0, ry.data_ptr(), rydot.data_ptr(), rhd.data_ptr(), ymsk.data_ptr(), ng, ny, demag) == 0
    rjv = zeros()
    assert lib.ref_i2_jtv(dev(v).data_ptr(), rjv.data_ptr(), ry.data_ptr(), ymsk.data_ptr(), ng, ny) == 0
    pd = lib.Precond_Create(ng, ny, n)
    gamma = 0.0173
    assert lib.ref_i2_psetup(pd, ry.data_ptr(), rhd.data_ptr(), n0, gamma, ng, ny) == 0
    rz = zeros()
    assert lib.ref_i2_psolve(pd, dev(r).data_ptr(), rz.data_ptr(), ymsk.data_ptr(), ng, ny) == 0
    lib.Precond_Destroy(pd)
    if demag:
        lib.Demag_Destroy(demag)
    # this library through its C ABI, same inputs
    ctx = llg.Context(p)
    ctx.set_mask(act3)
    if demag:
        s3 = ctx.demag_self_coupling()
        assert np.allclose(s3, tuple(n0), rtol=1e-12, atol=1e-15), (s3, tuple(n0))
    oy, oydot = dev(y), zeros()
    ctx.rhs(0.0, oy, oydot)
    ojv = zeros()
    ctx.jtv(dev(v), ojv, 0.0, oy)
    ctx.psetup(0.0, oy, oydot, 0, gamma)
    oz = zeros()
    ctx.psolve(0.0, oy, oydot, dev(r), oz, gamma)
    torch.cuda.synchronize()
    tol = 1e-11 if strength > 0 else 1e-13
    errs = {"y": rel_err(oy.cpu().numpy(), ry.cpu().numpy()), "f": rel_err(oydot.cpu().numpy(), rydot.cpu().numpy()),
            "jv": rel_err(ojv.cpu().numpy(), rjv.cpu().numpy()), "psolve": rel_err(oz.cpu().numpy(), rz.cpu().numpy())}
    print(f"{ng}x{ny} strength {strength}: " + ", ".join(f"{k} {e:.2e}" for k, e in errs.items()))
    assert errs["y"] <= 1e-15
    assert errs["f"] <= tol
    assert errs["jv"] <= 1e-13
    assert errs["psolve"] <= tol
