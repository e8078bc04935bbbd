"""The compact variant's ellipse geometry against the reference's own host
builder (CPU only).

BuildEllipticalActiveLists (src/irregular/2d_fft/2d_i6/2d_i6.cu:462-533) is
host code, compiled where it lies into oracle/_ref/libref_i6.so
(oracle/Makefile, target ref) with its default semi-axis fractions
ACTIVE_RX_FRAC = ACTIVE_RY_FRAC = 0.25.  Its active and inactive id lists must
equal, element for element and in order, the lists this library's geometry
builder gives for LLG_GEOM_ELLIPSE with the same fractions.
"""
import ctypes as C
import os

import numpy as np
import pytest

import llg
from conftest import REPO

REF_I6 = os.path.join(REPO, "oracle", "_ref", "libref_i6.so")


@pytest.mark.skipif(not os.path.exists(REF_I6), reason="reference i6 checker not built (needs the reference tree)")
@pytest.mark.parametrize("ng,ny", [(64, 48), (45, 27), (7, 5), (1, 1), (300, 2), (2048, 2048)])
def test_ellipse_lists_match_reference_builder(llg_lib, ng, ny):
    lib = C.CDLL(REF_I6)
    P = C.POINTER(C.c_int)
    lib.ref_i6_ellipse_lists.argtypes = [C.c_int, C.c_int, P, P, P, P]
    n = ng * ny
    a = np.zeros(n, np.int32)
    i = np.zeros(n, np.int32)
    na, ni = C.c_int(), C.c_int()
    assert lib.ref_i6_ellipse_lists(ng, ny, a.ctypes.data_as(P), C.byref(na), i.ctypes.data_as(P), C.byref(ni)) == 0
    assert na.value + ni.value == n
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_ELLIPSE, active_rx_frac=0.25, active_ry_frac=0.25)
    act = llg.build_geometry(g)["active"].astype(bool)
    ids = np.arange(n, dtype=np.int32)
    np.testing.assert_array_equal(ids[act], a[:na.value])
    np.testing.assert_array_equal(ids[~act], i[:ni.value])
