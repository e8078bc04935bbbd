"""Host-side binding of libllg.so, the C ABI declared in include/llg.h.

This module is a thin ctypes layer for Python callers (the test-suite and
bench.py); it mirrors the POD structs of include/llg.h field for field and
exposes the operator callbacks with the reference's argument meaning:

    rhs(t, y, ydot)                     f(t, y, ydot, user_data)       2d_i2/2d_fft.cu:366
    jtv(v, Jv, t, y, fy)                JtvProduct(v, Jv, t, y, fy, …)  2d_i2/jtv.cu:131
    psetup(t, y, fy, jok, gamma)        PrecondSetup(…)                 2d_i2/precond.cu:323
    psolve(t, y, fy, r, z, gamma, δ, lr) PrecondSolve(…)                2d_i2/precond.cu:360

Device buffers are passed as integer device addresses (torch tensors'
data_ptr()).  A call that returns a negative status raises LLGError; the
CUDA library must be present — there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libllg.so")

# ── constants (include/llg.h) ───────────────────────────────────────────
LLG_SUCCESS = 0
EXEC_YMSK, EXEC_COMPACT = 0, 1
BC_PERIODIC, BC_FREE = 0, 1
NORM_NONE, NORM_EXACT, NORM_REG = 0, 1, 2
ANISO_LINEAR, ANISO_CUBIC = 0, 1
DEMAG_OFF, DEMAG_PERIODIC, DEMAG_OPEN = 0, 1, 2
DEMAG_FP64, DEMAG_MIXED = 0, 1
JV_REFERENCE, JV_FULL_FIELD, JV_FULL_DEMAG = 0, 1, 2
GS_AUTO, GS_CLASSICAL, GS_MODIFIED = 0, 1, 2
KRYLOV_FP64, KRYLOV_FP32 = 0, 1
PREC_BLOCK_JACOBI, PREC_LEARNED = 0, 1
GEOM_BULK, GEOM_HOLE_SQUARE, GEOM_RING, GEOM_POLYCRYSTAL, GEOM_CUSTOM, GEOM_ELLIPSE, GEOM_ANNULUS, GEOM_SLIT = range(8)
IC_UNIFORM, IC_HEAD_ON_STRIPES, IC_TWO_DOMAIN, IC_GRAIN_BUMPS, IC_CUSTOM, IC_TWO_DOMAIN_X, IC_VORTEX, IC_NEEL = range(8)

CV_CODES = {0: "CV_SUCCESS", -1: "CV_TOO_MUCH_WORK", -2: "CV_TOO_MUCH_ACC", -3: "CV_ERR_FAILURE",
            -4: "CV_CONV_FAILURE", -6: "CV_LSETUP_FAIL", -7: "CV_LSOLVE_FAIL", -8: "CV_RHSFUNC_FAIL",
            -22: "CV_ILL_INPUT", -27: "CV_TOO_CLOSE", -40: "CV_BAD_STATE", -100: "LLG_ERR_ARG",
            -101: "LLG_ERR_CUDA", -102: "LLG_ERR_NOMEM", -103: "LLG_ERR_STATE", -104: "LLG_ERR_TIMEOUT",
            -105: "LLG_ERR_NOTSUP"}


class Params(C.Structure):
    _fields_ = [
        ("ng", C.c_int32), ("ny", C.c_int32), ("exec_model", C.c_int32), ("bc", C.c_int32),
        ("norm_kind", C.c_int32), ("aniso_kind", C.c_int32), ("demag_mode", C.c_int32),
        ("demag_precision", C.c_int32), ("windowed", C.c_int32), ("jv_mode", C.c_int32),
        ("precond_kind", C.c_int32), ("reserved0", C.c_int32),
        ("norm_eps", C.c_double), ("che", C.c_double), ("chk", C.c_double), ("cha", C.c_double),
        ("chb", C.c_double), ("alpha", C.c_double), ("chg", C.c_double),
        ("msk", C.c_double * 3), ("nsk", C.c_double * 3), ("happ", C.c_double * 3),
        ("demag_strength", C.c_double), ("demag_thick", C.c_double),
        ("src_col", C.c_int32), ("pml_cells", C.c_int32), ("src_amp", C.c_double), ("src_omega", C.c_double),
        ("src_ramp", C.c_double), ("pml_alpha_max", C.c_double),
    ]


class SolverOpts(C.Structure):
    _fields_ = [
        ("rtol", C.c_double), ("atol", C.c_double), ("maxl", C.c_int32), ("maxord", C.c_int32),
        ("gs_type", C.c_int32), ("mxstep", C.c_int32), ("device_resident", C.c_int32),
        ("krylov_precision", C.c_int32),
    ]


class TrainOpts(C.Structure):
    _fields_ = [("iters", C.c_int32), ("batch", C.c_int32), ("patch", C.c_int32), ("seed", C.c_int32),
                ("lr", C.c_double), ("init_scale", C.c_double)]


LEARNED_NWEIGHTS = 4032


class Stats(C.Structure):
    _fields_ = [
        ("nst", C.c_int64), ("nfe", C.c_int64), ("nsetups", C.c_int64), ("nni", C.c_int64),
        ("ncfn", C.c_int64), ("netf", C.c_int64), ("nli", C.c_int64), ("nlcf", C.c_int64),
        ("njvevals", C.c_int64), ("npsolves", C.c_int64), ("npe", C.c_int64),
        ("nfe_demag", C.c_int64), ("qlast", C.c_int32), ("qcur", C.c_int32),
        ("hlast", C.c_double), ("hcur", C.c_double), ("tcur", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CkptInfo(C.Structure):
    _fields_ = [
        ("magic", C.c_char * 8), ("version", C.c_uint32), ("header_bytes", C.c_uint32),
        ("scalar_bytes", C.c_uint32), ("krylov_precision", C.c_uint32), ("ng", C.c_int32), ("ny", C.c_int32),
        ("neq", C.c_int64), ("qmax", C.c_int32), ("maxl", C.c_int32), ("classical_gs", C.c_int32),
        ("mxstep", C.c_int32), ("device_resident", C.c_int32), ("have_setup", C.c_int32),
        ("rtol", C.c_double), ("atol", C.c_double), ("gamma_setup", C.c_double), ("tn", C.c_double),
        ("nst", C.c_int64), ("nfe_demag", C.c_int64), ("payload_bytes", C.c_uint64), ("checksum", C.c_uint64),
        ("params", Params),
    ]


FRAME_TRAJECTORY, FRAME_FINAL = 0, 1


class GeomSpec(C.Structure):
    _fields_ = [
        ("ng", C.c_int32), ("ny", C.c_int32), ("geometry_kind", C.c_int32), ("ic_kind", C.c_int32),
        ("hole_center_x_frac", C.c_double), ("hole_center_y_frac", C.c_double),
        ("hole_radius_frac_y", C.c_double),
        ("outer_w_frac", C.c_double), ("outer_h_frac", C.c_double),
        ("inner_w_frac_of_outer", C.c_double), ("inner_h_frac_of_outer", C.c_double),
        ("active_rx_frac", C.c_double), ("active_ry_frac", C.c_double),
        ("annulus_r_in_frac", C.c_double), ("annulus_r_out_frac", C.c_double),
        ("num_grains", C.c_int32), ("hole_seed", C.c_uint32),
        ("dead_grain_frac", C.c_double), ("mask_eps_cells", C.c_double), ("grain_z_bias", C.c_double),
        ("init_m", C.c_double * 3), ("init_random_seed", C.c_uint32), ("reserved0", C.c_int32),
        ("init_random_eps", C.c_double), ("stripe_left_frac", C.c_double),
        ("stripe_right_frac", C.c_double), ("two_domain_split_frac", C.c_double),
        ("two_domain_tail_my", C.c_double), ("ic_core_mz", C.c_double), ("ic_jitter_eps", C.c_double),
        ("texture_core_mz", C.c_double), ("texture_outer_mz", C.c_double), ("texture_width_frac", C.c_double),
        ("texture_eps", C.c_double), ("circle_cx_frac", C.c_double), ("circle_cy_frac", C.c_double),
        ("circle_r_frac_y", C.c_double), ("screen_x_frac", C.c_double), ("slit_w_frac", C.c_double),
    ]


def default_params(ng, ny, **kw) -> Params:
    """Physics of the 128x64 local case: A=1, k=0.1 along +x (linear/uniaxial),
    h_app=(0,0,0.05), alpha=0.02, free edges, no demag, no normalisation."""
    p = Params()
    p.ng, p.ny = ng, ny
    p.exec_model, p.bc, p.norm_kind = EXEC_YMSK, BC_FREE, NORM_NONE
    p.aniso_kind, p.demag_mode, p.demag_precision = ANISO_LINEAR, DEMAG_OFF, DEMAG_FP64
    p.windowed, p.jv_mode, p.precond_kind = 0, JV_REFERENCE, PREC_BLOCK_JACOBI
    p.norm_eps = 1e-3
    p.che, p.chk, p.cha, p.chb, p.alpha, p.chg = 1.0, 0.1, 0.0, 0.0, 0.02, 1.0
    p.msk[:] = (1.0, 0.0, 0.0)
    p.nsk[:] = (1.0, 0.0, 0.0)
    p.happ[:] = (0.0, 0.0, 0.05)
    p.demag_strength, p.demag_thick = 0.0, 1.0
    for k, v in kw.items():
        if k in ("msk", "nsk", "happ"):
            getattr(p, k)[:] = v
        else:
            setattr(p, k, v)
    return p


def slit_params(ng, ny, **kw) -> Params:
    """The reference's spin-wave single-slit run (src/slit/2d_slit.cu:69-135):
    easy axis z (cubic form, k = 0.5), exchange 4, DMI 0.1 along x, alpha
    0.005 with 20-cell absorbing layers ramping to 0.5 at the x edges, a soft
    source h_x = 0.1 ramp(t) sin(2 pi 0.12 t) (30-unit smoothstep ramp) on
    column 0.25 ng, periodic neighbours and periodic FFT demag of strength 1,
    regularised normalisation.  Pair it with GEOM_SLIT and m0 = (0, 0, 1)."""
    base = dict(bc=BC_PERIODIC, norm_kind=NORM_REG, aniso_kind=ANISO_CUBIC, che=4.0, chk=0.5, chb=0.1,
                alpha=0.005, chg=1.0, msk=(0.0, 0.0, 1.0), nsk=(1.0, 0.0, 0.0), happ=(0.0, 0.0, 0.0),
                demag_mode=DEMAG_PERIODIC, demag_strength=1.0, demag_thick=1.0,
                src_col=int(0.25 * ng + 0.5), src_amp=0.10, src_omega=2.0 * 3.14159265358979323846 * 0.12,
                src_ramp=30.0, pml_cells=20, pml_alpha_max=0.5)
    base.update(kw)
    return default_params(ng, ny, **base)


def source_value(params: Params, t: float) -> float:
    """The soft source's field at time t (0 when inactive)."""
    return float(load().llg_source_value(C.byref(params), float(t)))


def default_solver_opts(**kw) -> SolverOpts:
    o = SolverOpts()
    o.rtol, o.atol, o.maxl, o.maxord = 1e-4, 1e-6, 5, 5
    o.gs_type, o.mxstep, o.device_resident = GS_AUTO, 500, 0
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_geom(ng, ny, **kw) -> GeomSpec:
    g = GeomSpec()
    g.ng, g.ny = ng, ny
    g.geometry_kind, g.ic_kind = GEOM_BULK, IC_UNIFORM
    g.hole_center_x_frac, g.hole_center_y_frac, g.hole_radius_frac_y = 0.5, 0.5, 0.22
    g.outer_w_frac, g.outer_h_frac = 0.5, 0.5
    g.inner_w_frac_of_outer, g.inner_h_frac_of_outer = 0.5, 0.5
    g.active_rx_frac, g.active_ry_frac = 0.25, 0.25
    g.annulus_r_in_frac, g.annulus_r_out_frac = 0.15, 0.35
    g.num_grains, g.hole_seed = 72, 20251104
    g.dead_grain_frac, g.mask_eps_cells, g.grain_z_bias = 0.16, 2.2, 1.6
    g.init_m[:] = (1.0, 0.0, 0.0)
    g.init_random_seed = 12345
    g.init_random_eps = 0.01
    g.stripe_left_frac, g.stripe_right_frac = 0.25, 0.75
    g.two_domain_split_frac, g.two_domain_tail_my = 0.875, -0.0175
    g.ic_core_mz, g.ic_jitter_eps = 0.95, 0.0
    g.texture_core_mz, g.texture_outer_mz, g.texture_width_frac, g.texture_eps = -0.998, 0.998, 0.35, 1e-12
    g.circle_cx_frac, g.circle_cy_frac, g.circle_r_frac_y = 0.5, 0.5, 0.22
    g.screen_x_frac, g.slit_w_frac = 0.5, 0.10
    for k, v in kw.items():
        if k == "init_m":
            g.init_m[:] = v
        else:
            setattr(g, k, v)
    return g


class LLGError(RuntimeError):
    pass


_lib = None


def load(path: str | None = None):
    """Load libllg.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise LLGError(f"libllg.so not built at {p}; run __graft_entry__.build()")
    lib = C.CDLL(p)
    P, VP, D, I = C.POINTER, C.c_void_p, C.c_double, C.c_int
    sig = {
        "llg_default_params": (I, [P(Params)]),
        "llg_default_solver_opts": (I, [P(SolverOpts)]),
        "llg_create": (I, [P(Params), P(VP)]),
        "llg_destroy": (None, [VP]),
        "llg_set_stream": (I, [VP, VP]),
        "llg_last_error": (C.c_char_p, []),
        "llg_set_mask": (I, [VP, P(D)]),
        "llg_set_active_ids": (I, [VP, P(C.c_int32), C.c_int32, P(C.c_int32), C.c_int32]),
        "llg_set_window": (I, [VP, P(D), P(D), P(D)]),
        "llg_rhs": (I, [VP, D, VP, VP]),
        "llg_jtv": (I, [VP, VP, VP, D, VP, VP]),
        "llg_psetup": (I, [VP, D, VP, VP, I, P(I), D]),
        "llg_psolve": (I, [VP, D, VP, VP, VP, VP, D, D, I]),
        "llg_normalize": (I, [VP, VP]),
        "llg_demag_apply": (I, [VP, VP, VP]),
        "llg_demag_self_coupling": (I, [VP, P(D)]),
        "llg_demag_tensor_host": (I, [VP, I, I, I, P(D)]),
        "llg_hdemag_device": (VP, [VP]),
        "llg_dot_multi": (I, [VP, I, VP, P(VP), P(D)]),
        "llg_linear_combination": (I, [VP, I, P(D), P(VP), VP]),
        "llg_wrms_norm": (I, [VP, VP, VP, P(D)]),
        "llg_integrator_init": (I, [VP, D, VP, P(SolverOpts)]),
        "llg_integrate": (I, [VP, D, VP, P(D)]),
        "llg_get_stats": (I, [VP, P(Stats)]),
        "llg_default_geom_spec": (I, [P(GeomSpec)]),
        "llg_source_value": (D, [P(Params), D]),
        "llg_build_geometry": (I, [P(GeomSpec), VP, VP, VP, VP, VP, VP]),
        "llg_build_geometry_device": (I, [P(GeomSpec), VP, VP, VP, VP, VP, VP]),
        "llg_parse_config": (I, [C.c_char_p, P(Params), P(GeomSpec), P(SolverOpts)]),
        "llg_selftest_tcgen05": (I, [I, P(D)]),
        "llg_trace_control": (I, [VP, VP, C.c_int32]),
        "llg_kernel_timer_start": (I, [VP, C.c_uint32, C.c_int32, C.c_int32]),
        "llg_kernel_timer_stop": (I, [VP, P(D), P(C.c_int64), C.c_int32]),
        "llg_trace_count": (I, [VP]),
        "llg_batch_create": (I, [C.c_int32, P(Params), P(VP)]),
        "llg_batch_size": (I, [VP]),
        "llg_batch_ctx": (VP, [VP, C.c_int32]),
        "llg_batch_integrator_init": (I, [VP, D, P(VP), P(SolverOpts)]),
        "llg_batch_integrate": (I, [VP, D, P(VP), C.c_int32, P(C.c_int32)]),
        "llg_batch_destroy": (None, [VP]),
        "llg_batch_integrate_graph": (I, [VP, D, P(VP), P(C.c_int32)]),
        "llg_partition_lpt": (I, [C.c_int32, P(D), C.c_int32, P(C.c_int32), P(D)]),
        "llg_integrator_record_steps": (I, [VP, C.c_int32]),
        "llg_integrator_recorded_steps": (I, [VP, P(D), P(C.c_int32), C.c_int32]),
        "llg_integrator_replay_steps": (I, [VP, P(D), P(C.c_int32), C.c_int32]),
        "llg_integrator_replay_status": (I, [VP, P(C.c_int32), P(C.c_int64)]),
        "llg_inject_rhs_failure": (I, [VP, C.c_int64]),
        "llg_set_control_op_limit": (I, [VP, C.c_int64]),
        "llg_checkpoint_size": (I, [VP, P(C.c_uint64)]),
        "llg_checkpoint_save": (I, [VP, VP, C.c_uint64, P(C.c_uint64)]),
        "llg_checkpoint_load": (I, [VP, VP, C.c_uint64]),
        "llg_checkpoint_inspect": (I, [VP, C.c_uint64, P(CkptInfo)]),
        "llg_checkpoint_write_file": (I, [VP, C.c_char_p]),
        "llg_checkpoint_read_file": (I, [VP, C.c_char_p]),
        "llg_write_frame": (I, [C.c_char_p, C.c_int32, D, C.c_int32, C.c_int32, P(D), C.c_int32]),
        "llg_write_frame_device": (I, [VP, C.c_char_p, C.c_int32, D, VP, C.c_int32]),
        "llg_should_write_frame": (I, [C.c_int64, D, D, C.c_int32, C.c_int32]),
        "llg_write_aux_files": (I, [C.c_char_p, C.c_int32, C.c_int32, P(D), P(C.c_int32)]),
        "llg_learned_harvest": (I, [VP, C.c_int32, C.c_int32]),
        "llg_learned_num_samples": (I, [VP]),
        "llg_learned_train": (I, [VP, P(TrainOpts), P(D), P(D)]),
        "llg_learned_set_weights": (I, [VP, P(C.c_float), C.c_int32]),
        "llg_learned_get_weights": (I, [VP, P(C.c_float), C.c_int32]),
        "llg_learned_status": (I, [VP, P(C.c_int32), P(C.c_int32), P(C.c_int64)]),
        "llg_learned_set_fused": (I, [VP, C.c_int32]),
        "llg_learned_policy": (I, [VP, P(D), P(D), P(D)]),
        "llg_learned_set_policy": (I, [VP, C.c_int32]),
        "llg_learned_apply": (I, [VP, VP, VP, VP, D, VP, P(D)]),
        "llg_learned_loss_grad": (I, [P(C.c_float), C.c_int32, C.c_int32] + [P(C.c_float)] * 6
                                  + [P(D), P(C.c_float), P(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(rc, what):
    if rc < 0:
        msg = _lib.llg_last_error() if _lib is not None else b""
        raise LLGError(f"{what} failed with status {rc}: {(msg or b'').decode(errors='replace')}")
    return rc


def _ptr(x):
    """Device/host address of a torch tensor, numpy array or int."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(type(x))


class Context:
    """Owns one llg_ctx (one problem instance on the current CUDA device)."""

    def __init__(self, params: Params, stream=None):
        self.lib = load()
        self.params = params
        h = C.c_void_p()
        _check(self.lib.llg_create(C.byref(params), C.byref(h)), "llg_create")
        self.h = h
        self.ncell = params.ng * params.ny
        if stream is not None:
            _check(self.lib.llg_set_stream(self.h, _ptr(stream) if not hasattr(stream, "cuda_stream") else stream.cuda_stream), "llg_set_stream")

    @classmethod
    def _borrowed(cls, lib, handle, params):
        """Non-owning view of a context that a Batch owns."""
        c = cls.__new__(cls)
        c.lib, c.params, c.h, c.ncell, c._borrowed_ref = lib, params, C.c_void_p(handle), params.ng * params.ny, True
        return c

    def close(self):
        if getattr(self, "_borrowed_ref", False):
            self.h = None
            return
        if getattr(self, "h", None):
            self.lib.llg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # geometry
    def set_mask(self, ymsk3):
        import numpy as np
        a = np.ascontiguousarray(ymsk3, dtype=np.float64)
        _check(self.lib.llg_set_mask(self.h, a.ctypes.data_as(C.POINTER(C.c_double))), "llg_set_mask")

    def set_active_ids(self, active, inactive):
        import numpy as np
        a = np.ascontiguousarray(active, dtype=np.int32)
        b = np.ascontiguousarray(inactive, dtype=np.int32)
        _check(self.lib.llg_set_active_ids(self.h, a.ctypes.data_as(C.POINTER(C.c_int32)), len(a),
                                           b.ctypes.data_as(C.POINTER(C.c_int32)), len(b)), "llg_set_active_ids")

    def set_window(self, w, msk3, nsk3):
        import numpy as np
        f = lambda x: None if x is None else np.ascontiguousarray(x, dtype=np.float64)
        w, msk3, nsk3 = f(w), f(msk3), f(nsk3)
        cp = lambda x: None if x is None else x.ctypes.data_as(C.POINTER(C.c_double))
        _check(self.lib.llg_set_window(self.h, cp(w), cp(msk3), cp(nsk3)), "llg_set_window")

    # operators
    def rhs(self, t, y, ydot):
        return _check(self.lib.llg_rhs(self.h, t, _ptr(y), _ptr(ydot)), "llg_rhs")

    def jtv(self, v, Jv, t, y, fy=None):
        return _check(self.lib.llg_jtv(self.h, _ptr(v), _ptr(Jv), t, _ptr(y), _ptr(fy)), "llg_jtv")

    def psetup(self, t, y, fy, jok, gamma):
        jcur = C.c_int(0)
        _check(self.lib.llg_psetup(self.h, t, _ptr(y), _ptr(fy), jok, C.byref(jcur), gamma), "llg_psetup")
        return jcur.value

    def psolve(self, t, y, fy, r, z, gamma, delta=0.0, lr=1):
        return _check(self.lib.llg_psolve(self.h, t, _ptr(y), _ptr(fy), _ptr(r), _ptr(z), gamma, delta, lr), "llg_psolve")

    def normalize(self, y):
        return _check(self.lib.llg_normalize(self.h, _ptr(y)), "llg_normalize")

    def demag_apply(self, y, h):
        return _check(self.lib.llg_demag_apply(self.h, _ptr(y), _ptr(h)), "llg_demag_apply")

    def demag_self_coupling(self):
        out = (C.c_double * 3)()
        _check(self.lib.llg_demag_self_coupling(self.h, out), "llg_demag_self_coupling")
        return tuple(out)

    def demag_tensor(self, comp, dx, dy):
        out = C.c_double()
        _check(self.lib.llg_demag_tensor_host(self.h, comp, dx, dy, C.byref(out)), "llg_demag_tensor_host")
        return out.value

    def hdemag_ptr(self):
        return self.lib.llg_hdemag_device(self.h)

    def dot_multi(self, x, Ys):
        n = len(Ys)
        arr = (C.c_void_p * n)(*[_ptr(y) for y in Ys])
        out = (C.c_double * n)()
        _check(self.lib.llg_dot_multi(self.h, n, _ptr(x), arr, out), "llg_dot_multi")
        return list(out)

    def linear_combination(self, coeffs, Xs, z):
        n = len(Xs)
        arr = (C.c_void_p * n)(*[_ptr(x) for x in Xs])
        c = (C.c_double * n)(*coeffs)
        return _check(self.lib.llg_linear_combination(self.h, n, c, arr, _ptr(z)), "llg_linear_combination")

    def wrms_norm(self, x, w):
        out = C.c_double()
        _check(self.lib.llg_wrms_norm(self.h, _ptr(x), _ptr(w), C.byref(out)), "llg_wrms_norm")
        return out.value

    # integrator
    def integrator_init(self, t0, y0, opts: SolverOpts):
        return _check(self.lib.llg_integrator_init(self.h, t0, _ptr(y0), C.byref(opts)), "llg_integrator_init")

    def integrate(self, tout, yout):
        tret = C.c_double()
        rc = self.lib.llg_integrate(self.h, tout, _ptr(yout), C.byref(tret))
        if rc < 0:
            raise LLGError(f"llg_integrate -> {CV_CODES.get(rc, rc)}: "
                           f"{(self.lib.llg_last_error() or b'').decode(errors='replace')}")
        return tret.value

    def stats(self):
        st = Stats()
        _check(self.lib.llg_get_stats(self.h, C.byref(st)), "llg_get_stats")
        return st.as_dict()

    # ── step-sequence record / replay ──
    def record_steps(self, cap: int):
        """Record the (h, q) of every accepted step from now on (cap <= 0 stops)."""
        _check(self.lib.llg_integrator_record_steps(self.h, int(cap)), "llg_integrator_record_steps")

    def recorded_steps(self):
        n = _check(self.lib.llg_integrator_recorded_steps(self.h, None, None, 0), "llg_integrator_recorded_steps")
        h = np.zeros(n, np.float64)
        q = np.zeros(n, np.int32)
        _check(self.lib.llg_integrator_recorded_steps(self.h, h.ctypes.data_as(C.POINTER(C.c_double)),
                                                      q.ctypes.data_as(C.POINTER(C.c_int32)), n),
               "llg_integrator_recorded_steps")
        return h, q

    def replay_steps(self, h, q):
        """Make the next run (after integrator_init) take exactly these steps."""
        h = np.ascontiguousarray(h, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.int32)
        _check(self.lib.llg_integrator_replay_steps(self.h, h.ctypes.data_as(C.POINTER(C.c_double)),
                                                    q.ctypes.data_as(C.POINTER(C.c_int32)), len(h)),
               "llg_integrator_replay_steps")

    def replay_status(self):
        pos, forced = C.c_int32(), C.c_int64()
        _check(self.lib.llg_integrator_replay_status(self.h, C.byref(pos), C.byref(forced)),
               "llg_integrator_replay_status")
        return {"position": pos.value, "forced_accepts": forced.value}

    # ── test hooks ──
    def inject_rhs_failure(self, after: int):
        _check(self.lib.llg_inject_rhs_failure(self.h, int(after)), "llg_inject_rhs_failure")

    def set_control_op_limit(self, limit: int):
        _check(self.lib.llg_set_control_op_limit(self.h, int(limit)), "llg_set_control_op_limit")

    # ── checkpoint / restart ──
    def checkpoint(self) -> np.ndarray:
        """The integrator's complete state as a byte array (host)."""
        n = C.c_uint64()
        _check(self.lib.llg_checkpoint_size(self.h, C.byref(n)), "llg_checkpoint_size")
        buf = np.zeros(n.value, np.uint8)
        w = C.c_uint64()
        _check(self.lib.llg_checkpoint_save(self.h, buf.ctypes.data, n.value, C.byref(w)), "llg_checkpoint_save")
        return buf[: w.value]

    def restore(self, buf):
        b = np.ascontiguousarray(buf, dtype=np.uint8)
        _check(self.lib.llg_checkpoint_load(self.h, b.ctypes.data, b.size), "llg_checkpoint_load")

    def write_checkpoint(self, path):
        _check(self.lib.llg_checkpoint_write_file(self.h, os.fsencode(path)), "llg_checkpoint_write_file")

    def read_checkpoint(self, path):
        _check(self.lib.llg_checkpoint_read_file(self.h, os.fsencode(path)), "llg_checkpoint_read_file")

    def write_frame(self, path, t, y, append=True, style=FRAME_TRAJECTORY):
        """One magnetisation frame of device vector y in the reference's text format."""
        _check(self.lib.llg_write_frame_device(self.h, os.fsencode(path), int(bool(append)), float(t), _ptr(y),
                                               int(style)), "llg_write_frame_device")

    # ── learned preconditioner ──
    def learned_harvest(self, max_samples: int, stride: int = 1):
        _check(self.lib.llg_learned_harvest(self.h, int(max_samples), int(stride)), "llg_learned_harvest")

    def learned_num_samples(self) -> int:
        return int(self.lib.llg_learned_num_samples(self.h))

    def learned_train(self, iters=400, batch=16, patch=32, seed=1, lr=3e-3, init_scale=0.05):
        o = TrainOpts(int(iters), int(batch), int(patch), int(seed), float(lr), float(init_scale))
        l0, l1 = C.c_double(), C.c_double()
        _check(self.lib.llg_learned_train(self.h, C.byref(o), C.byref(l0), C.byref(l1)), "llg_learned_train")
        return l0.value, l1.value

    def learned_set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(self.lib.llg_learned_set_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size),
               "llg_learned_set_weights")

    def learned_get_weights(self):
        w = np.zeros(LEARNED_NWEIGHTS, dtype=np.float32)
        _check(self.lib.llg_learned_get_weights(self.h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size),
               "llg_learned_get_weights")
        return w

    def learned_set_policy(self, cost_aware: bool):
        _check(self.lib.llg_learned_set_policy(self.h, int(bool(cost_aware))), "llg_learned_set_policy")

    def learned_set_fused(self, fused: bool):
        _check(self.lib.llg_learned_set_fused(self.h, int(bool(fused))), "llg_learned_set_fused")

    def learned_apply(self, z, m, ewt, gamma, out):
        n2 = C.c_double()
        _check(self.lib.llg_learned_apply(self.h, _ptr(z), _ptr(m), _ptr(ewt), float(gamma), _ptr(out),
                                          C.byref(n2)), "llg_learned_apply")
        return n2.value

    def learned_status(self):
        a, f, n = C.c_int32(), C.c_int32(), C.c_int64()
        _check(self.lib.llg_learned_status(self.h, C.byref(a), C.byref(f), C.byref(n)), "llg_learned_status")
        il, ib, k = C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.llg_learned_policy(self.h, C.byref(il), C.byref(ib), C.byref(k)), "llg_learned_policy")
        return {"active": a.value, "fell_back": f.value, "napply": n.value, "it_learned": il.value,
                "it_block_jacobi": ib.value, "kappa": k.value}


class Batch:
    """Independent instances integrated concurrently (one stream each)."""

    def __init__(self, params_list):
        self.lib = load()
        n = len(params_list)
        arr = (Params * n)(*params_list)
        h = C.c_void_p()
        _check(self.lib.llg_batch_create(n, arr, C.byref(h)), "llg_batch_create")
        self.h = h
        self.params = list(params_list)
        self.ctx = [Context._borrowed(self.lib, self.lib.llg_batch_ctx(self.h, i), params_list[i]) for i in range(n)]

    def __len__(self):
        return len(self.ctx)

    def integrator_init(self, t0, ys, opts):
        ptrs = (C.c_void_p * len(ys))(*[_ptr(y) for y in ys])
        _check(self.lib.llg_batch_integrator_init(self.h, float(t0), ptrs, C.byref(opts)), "llg_batch_integrator_init")

    def integrate(self, tout, youts, nthreads=0):
        ptrs = (C.c_void_p * len(youts))(*[_ptr(y) for y in youts])
        rcs = (C.c_int32 * len(youts))()
        _check(self.lib.llg_batch_integrate(self.h, float(tout), ptrs, int(nthreads), rcs), "llg_batch_integrate")
        return list(rcs)

    def integrate_graph(self, tout, youts):
        """Every instance to tout in one CUDA graph launch (see llg.h)."""
        ptrs = (C.c_void_p * len(youts))(*[_ptr(y) for y in youts])
        rcs = (C.c_int32 * len(youts))()
        _check(self.lib.llg_batch_integrate_graph(self.h, float(tout), ptrs, rcs), "llg_batch_integrate_graph")
        return list(rcs)

    def stats(self):
        return [c.stats() for c in self.ctx]

    def close(self):
        for c in getattr(self, "ctx", []):
            c.close()
        if getattr(self, "h", None):
            self.lib.llg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return state, z ^ (z >> 31)


CONFIG4_SIZES = ((256, 256), (512, 256), (512, 512), (1024, 512))
CONFIG4_SHAPES = ("square_hole", "annulus", "ellipse", "polycrystal")


def config4_instances(n=64, master_seed=12345, demag_precision=DEMAG_MIXED, precond_kind=PREC_BLOCK_JACOBI,
                      sizes=CONFIG4_SIZES):
    """The batched mixed workload: n instances with seeded sizes from
    256x256 .. 1024x512, shapes from {square hole, annulus r 0.15..0.35 N,
    ellipse rx 0.3 NX ry 0.2 NY (compact index lists), polycrystal 24 grains
    10 % dead (windowed)}, open demag of strength U[1, 4], jittered uniform or
    two-domain initial states.  Seeds: master seed -> splitmix64 -> one 64-bit
    draw per instance (size, shape, strength, IC and srand seed from its bits).
    Returns a list of dicts with params, geom and a name."""
    out = []
    state = master_seed & 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        state, z = _splitmix64(state)
        ng, ny = sizes[z & 3]
        shape = CONFIG4_SHAPES[(z >> 2) & 3]
        strength = 1.0 + 3.0 * (((z >> 8) & 0xFFFF) / 65535.0)
        two_domain = bool((z >> 24) & 1)
        seed = int((z >> 32) & 0x7FFFFFFF) or 1
        pkw = dict(demag_mode=DEMAG_OPEN, demag_strength=strength, norm_kind=NORM_REG,
                   demag_precision=demag_precision, precond_kind=precond_kind)
        gkw = dict(ic_kind=IC_TWO_DOMAIN_X if two_domain else IC_UNIFORM, ic_jitter_eps=0.01,
                   init_random_seed=seed)
        if shape == "square_hole":
            gkw.update(geometry_kind=GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125)
        elif shape == "annulus":
            gkw.update(geometry_kind=GEOM_ANNULUS, annulus_r_in_frac=0.15, annulus_r_out_frac=0.35)
        elif shape == "ellipse":
            gkw.update(geometry_kind=GEOM_ELLIPSE, active_rx_frac=0.3, active_ry_frac=0.2)
            pkw.update(exec_model=EXEC_COMPACT)
        else:
            gkw.update(geometry_kind=GEOM_POLYCRYSTAL, num_grains=24, dead_grain_frac=0.10, grain_z_bias=1.0,
                       hole_seed=seed)
            pkw.update(windowed=1)
        out.append(dict(name=f"{i:02d}-{shape}-{ng}x{ny}", params=default_params(ng, ny, **pkw),
                        geom=default_geom(ng, ny, **gkw), shape=shape))
    return out


def setup_instance(ctx, inst):
    """Geometry of one config4_instances() entry into a context; returns y0 (host)."""
    geo = build_geometry(inst["geom"])
    p = inst["params"]
    n = p.ng * p.ny
    if p.windowed:
        ctx.set_window(geo["w"], geo["msk3"], geo["nsk3"])
    elif p.exec_model == EXEC_COMPACT:
        ids = np.arange(n, dtype=np.int32)
        act = geo["active"]
        ctx.set_active_ids(ids[act == 1], ids[act == 0])
    else:
        ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
    return geo["y0"]


def learned_loss_grad(w, u, m, mask, ewt, x, gamma, want_z=True):
    """Loss, weight gradient (and output z) of the CUDA training kernels on
    FP32 patches: u, m, ewt, x (nb, 3, P, P), mask (nb, P, P), gamma (nb,)."""
    lib = load()
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    w, u, m, mask, ewt, x, gamma = map(f32, (w, u, m, mask, ewt, x, gamma))
    nb, _, P, _ = u.shape
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    loss = C.c_double()
    grad = np.zeros(LEARNED_NWEIGHTS, dtype=np.float32)
    z = np.zeros_like(u) if want_z else None
    _check(lib.llg_learned_loss_grad(fp(w), nb, P, fp(u), fp(m), fp(mask), fp(ewt), fp(x), fp(gamma),
                                     C.byref(loss), fp(grad), fp(z) if want_z else None),
           "llg_learned_loss_grad")
    return loss.value, grad, z


def checkpoint_inspect(buf):
    """Validate a checkpoint blob (header, layout, checksum) without a GPU."""
    lib = load()
    b = np.ascontiguousarray(buf, dtype=np.uint8)
    info = CkptInfo()
    _check(lib.llg_checkpoint_inspect(b.ctypes.data, b.size, C.byref(info)), "llg_checkpoint_inspect")
    return info


def write_frame(path, t, ng, ny, m3, append=True, style=FRAME_TRAJECTORY):
    """One magnetisation frame (host SoA array) in the reference's text format."""
    lib = load()
    a = np.ascontiguousarray(m3, dtype=np.float64)
    if a.size != 3 * ng * ny:
        raise LLGError("write_frame: m3 must hold 3*ng*ny values")
    _check(lib.llg_write_frame(os.fsencode(path), int(bool(append)), float(t), int(ng), int(ny),
                               a.ctypes.data_as(C.POINTER(C.c_double)), int(style)), "llg_write_frame")


def should_write_frame(iout, t, early_until, early_every, late_every):
    return bool(_check(load().llg_should_write_frame(int(iout), float(t), float(early_until), int(early_every),
                                                     int(late_every)), "llg_should_write_frame"))


def write_aux_files(directory, ng, ny, w=None, grain_id=None):
    """mask.txt (window w) and grain_id.txt in the reference's format."""
    lib = load()
    wa = None if w is None else np.ascontiguousarray(w, dtype=np.float64)
    ga = None if grain_id is None else np.ascontiguousarray(grain_id, dtype=np.int32)
    _check(lib.llg_write_aux_files(os.fsencode(directory), int(ng), int(ny),
                                   None if wa is None else wa.ctypes.data_as(C.POINTER(C.c_double)),
                                   None if ga is None else ga.ctypes.data_as(C.POINTER(C.c_int32))),
           "llg_write_aux_files")


def read_frames(path):
    """Parse a frame file (trajectory or final state): list of (t, nx, ny, m[ncell, 3])."""
    frames = []
    with open(path) as f:
        lines = [ln for ln in f.read().split("\n")]
    i = 0
    while i < len(lines):
        if not lines[i].strip():
            i += 1
            continue
        t, nx, ny = lines[i].split()
        ncell = (int(nx) // 3) * int(ny)
        m = np.array([[float(v) for v in lines[i + 1 + k].split()] for k in range(ncell)])
        frames.append((float(t), int(nx), int(ny), m))
        i += 1 + ncell
    return frames


def selftest_tcgen05(flags: int) -> float:
    """One tensor-core GEMM (tcgen05, FP16 in, FP32 accumulate) against a
    host FP64 product; returns the max error relative to sum |a b|."""
    lib = load()
    err = C.c_double()
    _check(lib.llg_selftest_tcgen05(int(flags), C.byref(err)), "llg_selftest_tcgen05")
    return err.value


def build_geometry_device(spec: GeomSpec, stream=None):
    """Device geometry builder: torch tensors active (uint8), w, msk3, nsk3,
    grain_id (int32) on the current CUDA device, plus n_active."""
    import torch
    lib = load()
    n = spec.ng * spec.ny
    dev = torch.device("cuda")
    out = {"active": torch.empty(n, dtype=torch.uint8, device=dev),
           "w": torch.empty(n, dtype=torch.float64, device=dev),
           "msk3": torch.empty(3 * n, dtype=torch.float64, device=dev),
           "nsk3": torch.empty(3 * n, dtype=torch.float64, device=dev),
           "grain_id": torch.empty(n, dtype=torch.int32, device=dev)}
    rc = lib.llg_build_geometry_device(C.byref(spec), *[out[k].data_ptr() for k in ("active", "w", "msk3", "nsk3",
                                                                                    "grain_id")],
                                       None if stream is None else stream.cuda_stream)
    _check(rc, "llg_build_geometry_device")
    out["n_active"] = rc
    return out


def build_geometry(spec: GeomSpec, want=("active", "w", "msk3", "nsk3", "grain_id", "y0")):
    """Host geometry/IC builder of libllg.so; returns numpy arrays."""
    import numpy as np
    lib = load()
    n = spec.ng * spec.ny
    out = {
        "active": np.zeros(n, np.uint8) if "active" in want else None,
        "w": np.zeros(n, np.float64) if "w" in want else None,
        "msk3": np.zeros(3 * n, np.float64) if "msk3" in want else None,
        "nsk3": np.zeros(3 * n, np.float64) if "nsk3" in want else None,
        "grain_id": np.zeros(n, np.int32) if "grain_id" in want else None,
        "y0": np.zeros(3 * n, np.float64) if "y0" in want else None,
    }
    ptr = lambda a: None if a is None else a.ctypes.data
    rc = lib.llg_build_geometry(C.byref(spec), ptr(out["active"]), ptr(out["w"]), ptr(out["msk3"]),
                                ptr(out["nsk3"]), ptr(out["grain_id"]), ptr(out["y0"]))
    _check(rc, "llg_build_geometry")
    out["n_active"] = rc
    return out
