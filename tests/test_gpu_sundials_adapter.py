"""The SUNDIALS-signature callbacks of this library (csrc/sundials_adapter.cpp:
f, JtvProduct, PrecondSetup, PrecondSolve, FusedNVec_InitCtx) called the way
CVODE calls them.  SUNDIALS is not installed here, so oracle/Makefile target
`adapter` compiles the adapter against the stand-in headers of
oracle/ref_i2/shim (a vector handle = device pointer + length + an
operation table with the nvclone / nvdotprodmulti slots) and links it to
libllg.so.  Each callback must give exactly what the C ABI entry point it
forwards to gives, with the reference's status convention, and the
installed multi-dot slot must be llg_dot_multi (also on clones)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import llg
from conftest import REPO

pytestmark = pytest.mark.gpu

ADAPTER = os.path.join(REPO, "oracle", "_build", "libadapter_check.so")


class Ops(C.Structure):
    _fields_ = [("nvclone", C.c_void_p), ("nvdotprodmulti", C.c_void_p)]


class NVec(C.Structure):
    _fields_ = [("dev", C.c_void_p), ("host", C.c_void_p), ("n", C.c_long), ("ops", C.POINTER(Ops))]


DOTMULTI = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(NVec), C.POINTER(C.POINTER(NVec)), C.POINTER(C.c_double))
CLONE = C.CFUNCTYPE(C.POINTER(NVec), C.POINTER(NVec))


def _lib():
    llg.load()
    if not os.path.exists(ADAPTER):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "adapter"], check=True)
    a = C.CDLL(ADAPTER)
    P = C.POINTER(NVec)
    a.f.argtypes = [C.c_double, P, P, C.c_void_p]
    a.JtvProduct.argtypes = [P, P, C.c_double, P, P, C.c_void_p, P]
    a.PrecondSetup.argtypes = [C.c_double, P, P, C.c_int, C.POINTER(C.c_int), C.c_double, C.c_void_p]
    a.PrecondSolve.argtypes = [C.c_double, P, P, P, P, C.c_double, C.c_double, C.c_int, C.c_void_p]
    a.FusedNVec_InitCtx.argtypes = [P, C.c_void_p]
    a.llg_shim_nv_clone.restype = P
    a.llg_shim_nv_clone.argtypes = [P]
    a.llg_shim_nv_free.argtypes = [P]
    return a


def test_callbacks_forward_exactly(gpu):
    import torch
    a = _lib()
    ng, ny = 64, 48
    p = llg.default_params(ng, ny, bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_OPEN, demag_strength=3.0,
                           norm_kind=llg.NORM_REG)
    geo = llg.build_geometry(llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                                              ic_jitter_eps=0.01))
    ctx = llg.Context(p)
    ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
    n3 = 3 * ng * ny
    rng = np.random.default_rng(9)
    dv = lambda a_: torch.from_numpy(np.ascontiguousarray(a_)).cuda()   # noqa: E731
    nv = lambda t: NVec(t.data_ptr(), None, n3, None)                    # noqa: E731
    y = geo["y0"] + 0.05 * rng.standard_normal(n3)
    v, r = rng.standard_normal(n3), rng.standard_normal(n3)
    gamma = 0.031
    # through the adapter, as CVODE calls the callbacks
    ya, fa, jva, za = dv(y), torch.zeros(n3, dtype=torch.float64, device="cuda"), None, None
    assert a.f(0.3, C.byref(nv(ya)), C.byref(nv(fa)), ctx.h) == 0
    jva = torch.zeros_like(fa)
    assert a.JtvProduct(C.byref(nv(dv(v))), C.byref(nv(jva)), 0.3, C.byref(nv(ya)), C.byref(nv(fa)), ctx.h,
                        None) == 0
    jcur = C.c_int(0)
    assert a.PrecondSetup(0.3, C.byref(nv(ya)), C.byref(nv(fa)), 0, C.byref(jcur), gamma, ctx.h) == 0
    assert jcur.value == 1   # always rebuilds, as the reference
    za = torch.zeros_like(fa)
    assert a.PrecondSolve(0.3, C.byref(nv(ya)), C.byref(nv(fa)), C.byref(nv(dv(r))), C.byref(nv(za)), gamma, 0.0, 1,
                          ctx.h) == 0
    # the C ABI directly, same inputs
    yb, fb = dv(y), torch.zeros_like(fa)
    ctx.rhs(0.3, yb, fb)
    jvb = torch.zeros_like(fa)
    ctx.jtv(dv(v), jvb, 0.3, yb, fb)
    ctx.psetup(0.3, yb, fb, 0, gamma)
    zb = torch.zeros_like(fa)
    ctx.psolve(0.3, yb, fb, dv(r), zb, gamma)
    torch.cuda.synchronize()
    for x, y_ in ((ya, yb), (fa, fb), (jva, jvb), (za, zb)):
        assert torch.equal(x, y_)


def test_fused_multidot_slot_is_installed_on_vectors_and_clones(gpu):
    import torch
    a = _lib()
    ctx = llg.Context(llg.default_params(40, 30))
    n3 = 3 * 40 * 30
    rng = np.random.default_rng(10)
    xs = [torch.from_numpy(rng.standard_normal(n3)).cuda() for _ in range(6)]
    ops = Ops(C.cast(a.llg_shim_nv_clone, C.c_void_p).value, None)
    base = NVec(xs[0].data_ptr(), None, n3, C.pointer(ops))
    a.FusedNVec_InitCtx(C.byref(base), ctx.h)
    assert base.ops.contents.nvdotprodmulti is not None
    dot = DOTMULTI(base.ops.contents.nvdotprodmulti)
    Ys = [NVec(t.data_ptr(), None, n3, base.ops) for t in xs[1:]]
    arr = (C.POINTER(NVec) * 5)(*[C.pointer(v) for v in Ys])
    out = (C.c_double * 5)()
    assert dot(5, C.byref(base), arr, out) == 0
    ref = ctx.dot_multi(xs[0], xs[1:])
    assert list(out) == ref   # the library's deterministic multi-dot, bit for bit
    clone = CLONE(base.ops.contents.nvclone)(C.byref(base))
    assert clone and clone.contents.ops.contents.nvdotprodmulti == base.ops.contents.nvdotprodmulti
    a.llg_shim_nv_free(clone)
