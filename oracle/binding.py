"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py, as the checker.  The product
(libllg.so and its host module) never imports this file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "gpu-micromagnetics-irregular_b200"))
import llg  # noqa: E402  (struct mirrors of include/llg.h)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P, VP, D, I = C.POINTER, C.c_void_p, C.c_double, C.c_int
    sig = {
        "or_create": (VP, [P(llg.Params)]),
        "or_destroy": (None, [VP]),
        "or_set_active": (I, [VP, VP]),
        "or_set_window": (I, [VP, VP, VP, VP]),
        "or_set_threads": (I, [I]),
        "or_normalize": (None, [VP, VP]),
        "or_rhs": (I, [VP, D, VP, VP]),
        "or_jtv": (I, [VP, VP, VP, VP]),
        "or_psetup": (I, [VP, VP, D]),
        "or_psolve": (I, [VP, VP, VP]),
        "or_hdemag": (VP, [VP]),
        "or_pinv": (VP, [VP]),
        "or_demag_apply": (I, [VP, VP, VP]),
        "or_demag_direct": (I, [VP, VP, VP]),
        "or_demag_self": (I, [VP, P(D)]),
        "or_demag_tensor": (D, [VP, I, I, I]),
        "or_newell_point": (None, [D, D, D, P(D)]),
        "or_newell_avg": (None, [D, I, I, P(D)]),
        "or_fft": (I, [I, VP, I]),
        "or_integrator_init": (I, [VP, D, VP, P(llg.SolverOpts)]),
        "or_integrate": (I, [VP, D, VP, P(D)]),
        "or_get_stats": (I, [VP, P(llg.Stats)]),
        "or_build_geometry": (I, [P(llg.GeomSpec), VP, VP, VP, VP, VP, VP]),
        "or_wrms": (D, [VP, VP, C.c_long]),
        "or_dot": (D, [VP, VP, C.c_long]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """One CPU problem instance (FP64)."""

    def __init__(self, params: "llg.Params"):
        self.lib = load()
        self.params = params
        self.h = self.lib.or_create(C.byref(params))
        if not self.h:
            raise RuntimeError("or_create failed")
        self.n = params.ng * params.ny

    def __del__(self):
        try:
            if self.h:
                self.lib.or_destroy(self.h)
        except Exception:
            pass

    def set_active(self, active):
        self._act = None if active is None else np.ascontiguousarray(active, np.uint8)
        self.lib.or_set_active(self.h, _p(self._act))

    def set_window(self, w, msk3, nsk3):
        f = lambda x: None if x is None else np.ascontiguousarray(x, np.float64)
        self._w = (f(w), f(msk3), f(nsk3))
        self.lib.or_set_window(self.h, *[_p(a) for a in self._w])

    def normalize(self, y):
        self.lib.or_normalize(self.h, _p(y))

    def rhs(self, y, t=0.0):
        """Returns ydot; y is normalised in place like the product's f."""
        yd = np.zeros_like(y)
        assert self.lib.or_rhs(self.h, t, _p(y), _p(yd)) == 0
        return yd

    def jtv(self, v, y):
        out = np.zeros_like(v)
        self.lib.or_jtv(self.h, _p(v), _p(out), _p(y))
        return out

    def psetup(self, y, gamma):
        self.lib.or_psetup(self.h, _p(y), gamma)

    def psolve(self, r):
        z = np.zeros_like(r)
        self.lib.or_psolve(self.h, _p(r), _p(z))
        return z

    def hdemag(self):
        ptr = self.lib.or_hdemag(self.h)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), (3 * self.n,)).copy()

    def pinv(self):
        ptr = self.lib.or_pinv(self.h)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_double)), (9 * self.n,)).copy()

    def demag(self, y, direct=False):
        h = np.zeros_like(y)
        fn = self.lib.or_demag_direct if direct else self.lib.or_demag_apply
        fn(self.h, _p(y), _p(h))
        return h

    def demag_self(self):
        out = (C.c_double * 3)()
        self.lib.or_demag_self(self.h, out)
        return tuple(out)

    def tensor(self, comp, dx, dy):
        return self.lib.or_demag_tensor(self.h, comp, dx, dy)

    def integrator_init(self, y0, opts, t0=0.0):
        self._y0 = np.ascontiguousarray(y0, np.float64).copy()
        return self.lib.or_integrator_init(self.h, t0, _p(self._y0), C.byref(opts))

    def integrate(self, tout):
        y = np.zeros(3 * self.n)
        tret = C.c_double()
        rc = self.lib.or_integrate(self.h, tout, _p(y), C.byref(tret))
        return rc, tret.value, y

    def stats(self):
        st = llg.Stats()
        self.lib.or_get_stats(self.h, C.byref(st))
        return st.as_dict()


def newell_avg(thick, dx, dy):
    out = (C.c_double * 9)()
    load().or_newell_avg(thick, dx, dy, out)
    return np.array(out)


def fft(x, sign=-1):
    a = np.ascontiguousarray(x, np.complex128).copy()
    load().or_fft(len(a), a.ctypes.data, sign)
    return a


def build_geometry(spec):
    n = spec.ng * spec.ny
    out = dict(active=np.zeros(n, np.uint8), w=np.zeros(n), msk3=np.zeros(3 * n), nsk3=np.zeros(3 * n),
               grain_id=np.zeros(n, np.int32), y0=np.zeros(3 * n))
    rc = load().or_build_geometry(C.byref(spec), *[_p(out[k]) for k in ("active", "w", "msk3", "nsk3", "grain_id", "y0")])
    out["n_active"] = rc
    return out


def set_threads(n):
    return load().or_set_threads(n)
