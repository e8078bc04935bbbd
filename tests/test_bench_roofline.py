"""bench.py's roofline numerator: algorithmic bytes per launch (CPU only).

For the 1536x512 bench film (N = 786,432 cells; open demag on a 3072x1024
padded grid, 1537 kept x-frequencies of 512 data rows) the per-launch bytes
of the roofline kernels are the documented per-cell figures times N: the
Arnoldi operator 169 B/cell (FP64 basis) and 109 B/cell (FP32 basis); the row
transforms an FP64 state pass plus the spectrum (FP32 complex in the mixed
chain, FP64 complex otherwise).
"""
import sys

from conftest import REPO

NG, NY = 1536, 512
N = NG * NY
DIMS = (3072, 1024, 1537, 512)


def _bench():
    sys.path.insert(0, REPO)
    import bench
    return bench


def test_arnoldi_operator_bytes_per_cell():
    b = _bench()
    assert b.algorithmic_bytes(2, NG, NY, DIMS) == 169 * N == 132_907_008
    assert b.algorithmic_bytes(2, NG, NY, DIMS, kf32=True) == 109 * N == 85_721_088


def test_demag_stage_bytes():
    b = _bench()
    s_mixed = 3 * 1537 * 512 * 8
    s_fp64 = 3 * 1537 * 512 * 16
    assert b.algorithmic_bytes(6, NG, NY, DIMS, mixed=True) == 24 * N + s_mixed == 37_761_024
    assert b.algorithmic_bytes(8, NG, NY, DIMS, mixed=True) == 24 * N + s_mixed
    assert b.algorithmic_bytes(6, NG, NY, DIMS) == 24 * N + s_fp64
    assert b.algorithmic_bytes(7, NG, NY, DIMS, mixed=True) == 2 * s_mixed + 1537 * 1024 * 20
    assert b.algorithmic_bytes(7, NG, NY, DIMS) == 2 * s_fp64 + 1537 * 1024 * 40
