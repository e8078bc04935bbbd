"""CPU checks of the text outputs and of checkpoint validation.

Frames, the frame cadence and the auxiliary files are compared byte for byte
with the reference's formats, restated here with Python's printf-style
formatting (correctly rounded, as the C library's):
  WriteFrame         src/irregular/2d_fft/2d_i2/2d_fft.cu:437-455
  final output.txt   src/irregular/2d_fft/2d_i2/2d_fft.cu:735-757
  ShouldWriteFrame   src/irregular/2d_fft/2d_i2/2d_fft.cu:457-463
  write_aux_files    src/irregular/2d_fft/2d_i3/2d_fft.cu:390-408
Checkpoint blobs can only be produced on a GPU; here the validator must
reject buffers that are not checkpoints.
"""
import numpy as np
import pytest

import llg


def _ref_frame(t, ng, ny, m3, final):
    n = ng * ny
    out = ["%f %d %d\n" % (t, 3 * ng, ny)]
    fmt = "%e %e %e\n" if final else "%f %f %f\n"
    for c in range(n):
        out.append(fmt % (m3[c], m3[n + c], m3[2 * n + c]))
    if not final:
        out.append("\n")
    return "".join(out)


@pytest.mark.parametrize("final", [False, True])
def test_frame_matches_reference_format(llg_lib, tmp_path, final):
    ng, ny = 13, 7
    rng = np.random.default_rng(3)
    m3 = rng.uniform(-1, 1, 3 * ng * ny)
    m3[0], m3[1], m3[2] = -0.0, 1e-9, -1e-9   # signed zeros and values that round to zero
    m3[3] = 0.9999995                           # rounds up in the last printed digit
    path = tmp_path / "output.txt"
    style = llg.FRAME_FINAL if final else llg.FRAME_TRAJECTORY
    llg.write_frame(str(path), 12.5, ng, ny, m3, append=False, style=style)
    assert path.read_text() == _ref_frame(12.5, ng, ny, m3, final)


def test_trajectory_appends_frames_and_reads_back(llg_lib, tmp_path):
    ng, ny = 8, 5
    rng = np.random.default_rng(4)
    path = tmp_path / "traj.txt"
    expect = ""
    frames = []
    for k in range(3):
        m3 = rng.uniform(-1, 1, 3 * ng * ny)
        frames.append(m3)
        llg.write_frame(str(path), 0.1 * k, ng, ny, m3, append=(k > 0))
        expect += _ref_frame(0.1 * k, ng, ny, m3, False)
    assert path.read_text() == expect
    back = llg.read_frames(str(path))
    assert len(back) == 3
    for (t, nx, nyy, m), m3 in zip(back, frames):
        assert (nx, nyy) == (3 * ng, ny)
        n = ng * ny
        assert np.abs(m - np.stack([m3[:n], m3[n:2 * n], m3[2 * n:]], axis=1)).max() <= 5e-7


def test_frame_cadence():
    # EARLY_SAVE_UNTIL 5.0, EARLY_SAVE_EVERY 1, LATE_SAVE_EVERY 10
    for iout, t in ((1, 0.1), (7, 5.0), (10, 5.1), (20, 80.0)):
        assert llg.should_write_frame(iout, t, 5.0, 1, 10)
    for iout, t in ((11, 5.1), (55, 60.0)):
        assert not llg.should_write_frame(iout, t, 5.0, 1, 10)
    with pytest.raises(llg.LLGError):
        llg.should_write_frame(1, 0.0, 5.0, 0, 10)


def test_aux_files_match_reference_format(llg_lib, tmp_path):
    g = llg.default_geom(48, 24, geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=12, grain_z_bias=1.0)
    geo = llg.build_geometry(g)
    llg.write_aux_files(str(tmp_path), 48, 24, geo["w"], geo["grain_id"])
    mask = "48 24\n" + "".join("%f\n" % v for v in geo["w"])
    gid = "48 24\n" + "".join("%d\n" % v for v in geo["grain_id"])
    assert (tmp_path / "mask.txt").read_text() == mask
    assert (tmp_path / "grain_id.txt").read_text() == gid
    (tmp_path / "none").mkdir()
    llg.write_aux_files(str(tmp_path / "none"), 48, 24)   # both arrays absent: nothing written
    assert not any((tmp_path / "none").iterdir())


def test_checkpoint_validator_rejects_non_checkpoints(llg_lib):
    for buf in (np.zeros(0, np.uint8), np.zeros(100, np.uint8), np.frombuffer(b"LLGCKPT1" + bytes(400), np.uint8)):
        with pytest.raises(llg.LLGError, match="checkpoint"):
            llg.checkpoint_inspect(buf)
