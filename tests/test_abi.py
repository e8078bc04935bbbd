"""CPU checks of libllg.so's host side: exported symbols, builders, knobs,
and that there is no silent CPU path."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import llg
from conftest import REPO, has_gpu

HEADERS = [os.path.join(REPO, "include", h) for h in sorted(os.listdir(os.path.join(REPO, "include")))
           if h.endswith(".h")]


def declared_functions():
    names = []
    for path in HEADERS:
        text = open(path).read()
        # drop blocks compiled only with SUNDIALS headers present
        text = re.sub(r"#ifdef LLG_HAVE_SUNDIALS.*?#endif", "", text, flags=re.S)
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\([^;{]*\)\s*;", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "for", "while", "return", "sizeof"):
                names.append(name)
    return sorted(set(names))


def test_headers_declare_the_boundary():
    names = declared_functions()
    for must in ("llg_create", "llg_rhs", "llg_jtv", "llg_psetup", "llg_psolve", "llg_demag_apply",
                 "llg_dot_multi", "llg_integrate", "Demag_Init", "Demag_Apply", "Precond_Create"):
        assert must in names


def test_library_exports_every_declared_symbol(llg_lib):
    lib = C.CDLL(llg_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_create_fails_loudly_without_gpu(llg_lib):
    p = llg.default_params(16, 8)
    with pytest.raises(llg.LLGError, match="no CUDA device"):
        llg.Context(p)


def _cmp_geometry(oracle_lib, spec):
    a = llg.build_geometry(spec)
    b = oracle_lib.build_geometry(spec)
    assert a["n_active"] == b["n_active"]
    for k in ("active", "w", "msk3", "nsk3", "grain_id", "y0"):
        assert np.array_equal(a[k], b[k]), k
    return a


@pytest.mark.parametrize("kind,ic,kw", [
    (llg.GEOM_BULK, llg.IC_UNIFORM, dict(ic_jitter_eps=0.01)),
    (llg.GEOM_HOLE_SQUARE, llg.IC_UNIFORM, dict(hole_radius_frac_y=0.125, ic_jitter_eps=0.01)),
    (llg.GEOM_HOLE_SQUARE, llg.IC_TWO_DOMAIN, dict()),
    (llg.GEOM_RING, llg.IC_UNIFORM, dict(init_m=(1.0, -0.0175, 0.0))),
    (llg.GEOM_RING, llg.IC_UNIFORM, dict(inner_w_frac_of_outer=0.0, inner_h_frac_of_outer=0.0)),
    (llg.GEOM_ELLIPSE, llg.IC_VORTEX, dict(ic_jitter_eps=0.01)),
    (llg.GEOM_ANNULUS, llg.IC_UNIFORM, dict()),
    (llg.GEOM_BULK, llg.IC_HEAD_ON_STRIPES, dict()),
    (llg.GEOM_POLYCRYSTAL, llg.IC_GRAIN_BUMPS, dict(num_grains=24, dead_grain_frac=0.1)),
    (llg.GEOM_POLYCRYSTAL, llg.IC_TWO_DOMAIN_X, dict(num_grains=72, dead_grain_frac=0.16,
                                                     grain_z_bias=1.0, ic_jitter_eps=0.01)),
    (llg.GEOM_SLIT, llg.IC_UNIFORM, dict(init_m=(0.0, 0.0, 1.0))),
    (llg.GEOM_BULK, llg.IC_NEEL, dict()),
    (llg.GEOM_BULK, llg.IC_NEEL, dict(circle_r_frac_y=0.05, texture_width_frac=0.1, ic_jitter_eps=0.01)),
])
@pytest.mark.parametrize("ng,ny", [(64, 40), (37, 23)])
def test_geometry_builders_match_oracle_exactly(oracle_lib, kind, ic, kw, ng, ny):
    spec = llg.default_geom(ng, ny, geometry_kind=kind, ic_kind=ic, **kw)
    g = _cmp_geometry(oracle_lib, spec)
    n = ng * ny
    y = g["y0"].reshape(3, n)
    nrm = np.linalg.norm(y, axis=0)
    act = g["active"].astype(bool)
    if kind != llg.GEOM_POLYCRYSTAL and not (ic == llg.IC_NEEL and not kw.get("ic_jitter_eps")):
        # (the reference's Néel texture leaves a cell exactly at the centre at (0, 0, mz0), |m| < 1)
        assert np.allclose(nrm[act], 1.0) and np.all(nrm[~act] == 0.0)


def test_square_hole_matches_reference_predicate():
    """2d_i2/2d_fft.cu:545-556: hole iff |i-cx| <= hs and |j-cy| <= hs."""
    ng, ny = 1536, 512
    spec = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125)
    g = llg.build_geometry(spec, want=("active",))
    cx, cy, hs = 0.5 * (ng - 1), 0.5 * (ny - 1), 0.125 * ny
    i = np.arange(ng)[None, :]
    j = np.arange(ny)[:, None]
    ref = ~((np.abs(i - cx) <= hs) & (np.abs(j - cy) <= hs))
    assert np.array_equal(g["active"].reshape(ny, ng).astype(bool), ref)


def test_slit_matches_reference_predicate():
    """src/slit/2d_slit.cu:482-486, 541-560: the screen column is a hole
    except the slit rows [ny/2 - w/2, ny/2 - w/2 + w), w = (int)(0.1 ny + 0.5)."""
    ng, ny = 256, 85
    g = llg.build_geometry(llg.default_geom(ng, ny, geometry_kind=llg.GEOM_SLIT), want=("active",))
    act = g["active"].reshape(ny, ng).astype(bool)
    col, w = int(0.5 * ng + 0.5), int(0.1 * ny + 0.5)
    lo = ny // 2 - w // 2
    ref = np.ones((ny, ng), bool)
    ref[:, col] = False
    ref[lo:lo + w, col] = True
    assert np.array_equal(act, ref)


def test_neel_texture_matches_reference_formula():
    """src/2d_fft/2d_fft.cu:533-580 restated in numpy: tanh wall between core
    and outer mz, radial in-plane part."""
    ng, ny = 48, 40
    g = llg.build_geometry(llg.default_geom(ng, ny, ic_kind=llg.IC_NEEL), want=("y0",))
    cx, cy, r = 0.5 * (ng - 1), 0.5 * (ny - 1), 0.22 * ny
    width = max(1.0, 0.35 * r)
    i, j = np.meshgrid(np.arange(ng), np.arange(ny))
    dx, dy = i - cx, j - cy
    rho = np.hypot(dx, dy)
    mz = np.clip(0.998 + (-0.998 - 0.998) * 0.5 * (1 - np.tanh((rho - r) / width)), -1, 1)
    mp = np.sqrt(np.maximum(0, 1 - mz * mz))
    y = g["y0"].reshape(3, ny, ng)
    assert np.allclose(y[2], mz, rtol=0, atol=1e-15)
    assert np.allclose(y[0], mp * (dx / rho), rtol=0, atol=1e-13)   # sqrt(1 - mz^2) amplifies tanh ulps
    assert np.allclose(y[1], mp * (dy / rho), rtol=0, atol=1e-13)


def test_source_value_smoothstep():
    """src/slit/2d_slit.cu:236-240, 331-340: H ramp(t) sin(omega t)."""
    p = llg.slit_params(128, 64)
    for t in (0.0, 7.5, 29.0, 30.0, 55.0):
        x = min(t / 30.0, 1.0)
        ramp = 1.0 if t >= 30.0 else x * x * (3 - 2 * x)
        assert abs(llg.source_value(p, t) - 0.1 * ramp * np.sin(2 * np.pi * 0.12 * t)) <= 1e-15
    assert llg.source_value(llg.default_params(16, 8), 5.0) == 0.0


def test_polycrystal_window_large_grid_fast(oracle_lib):
    """The O(N) distance transform reproduces the reference's O(N·N_hole)
    window at 1536x512 / 72 grains (checked on a 96x64 crop of the logic)."""
    spec = llg.default_geom(96, 64, geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=20, dead_grain_frac=0.3)
    _cmp_geometry(oracle_lib, spec)


def test_parse_config_reference_knob_names(llg_lib):
    lib = llg.load()
    p, g, o = llg.Params(), llg.GeomSpec(), llg.SolverOpts()
    lib.llg_default_params(C.byref(p))
    lib.llg_default_geom_spec(C.byref(g))
    lib.llg_default_solver_opts(C.byref(o))
    text = b"""# configs/README.md style recipe
    NX_VAL=1536 NY_VAL=512
    GEOMETRY_KIND=GEOMETRY_HOLE_SQUARE HOLE_RADIUS_FRAC_Y=0.125
    DEMAG_STRENGTH=4.0 DEMAG_THICK=1.0 DEMAG_MODE=DEMAG_OPEN
    KRYLOV_DIM=5 RTOL_VAL=1.0e-4 ATOL_VAL=1.0e-6 -DMAX_BDF_ORDER=5
    ANISO_KIND=ANISO_CUBIC PHYS_C_CHE=50.0 HAPP_ENABLE=1 HAPP_X=-0.2
    """
    n = lib.llg_parse_config(text, C.byref(p), C.byref(g), C.byref(o))
    assert n == 15
    assert (p.ng, p.ny, g.ng, g.ny) == (512, 512, 512, 512)
    assert g.geometry_kind == llg.GEOM_HOLE_SQUARE and g.hole_radius_frac_y == 0.125
    assert p.demag_strength == 4.0 and p.demag_mode == llg.DEMAG_OPEN
    assert o.maxl == 5 and o.rtol == 1e-4 and o.maxord == 5
    assert p.aniso_kind == llg.ANISO_CUBIC and p.che == 50.0 and tuple(p.happ) == (-0.2, 0.0, 0.05)


def test_parse_config_slit_and_texture_knobs(llg_lib):
    lib = llg.load()
    p, g, o = llg.Params(), llg.GeomSpec(), llg.SolverOpts()
    lib.llg_default_params(C.byref(p))
    lib.llg_default_geom_spec(C.byref(g))
    lib.llg_default_solver_opts(C.byref(o))
    text = (b"NX_VAL=768 NY_VAL=256 GEOMETRY_KIND=GEOMETRY_SLIT SCREEN_X_FRAC=0.5 SLIT_W_FRAC=0.1 "
            b"SRC_X_FRAC=0.25 DRIVE_FREQ=0.12 H_DRIVE=0.1 RAMP_TIME=30 PML_CELLS=20 PML_ALPHA_MAX=0.5 "
            b"IC_KIND=IC_NEEL TEXTURE_CORE_MZ=-0.998 CIRCLE_RADIUS_FRAC_Y=0.22")
    assert lib.llg_parse_config(text, C.byref(p), C.byref(g), C.byref(o)) == 14
    assert p.ng == 256 and p.src_col == 64 and abs(p.src_omega - 2 * np.pi * 0.12) < 1e-15
    assert (p.src_amp, p.src_ramp, p.pml_cells, p.pml_alpha_max) == (0.1, 30.0, 20, 0.5)
    assert g.geometry_kind == llg.GEOM_SLIT and g.ic_kind == llg.IC_NEEL and g.texture_core_mz == -0.998


@pytest.mark.parametrize("bad", [b"NX_VAL=1537", b"NOT_A_KNOB=1", b"RTOL_VAL=abc", b"KRYLOV_DIM"])
def test_parse_config_rejects_corrupt_input(llg_lib, bad):
    lib = llg.load()
    p, g, o = llg.Params(), llg.GeomSpec(), llg.SolverOpts()
    assert lib.llg_parse_config(bad, C.byref(p), C.byref(g), C.byref(o)) < 0
