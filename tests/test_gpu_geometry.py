"""Device geometry builder (llg_build_geometry_device) against the host
builder (itself checked exactly against the oracle's restatement of the
reference builders): grain ids, active flags and per-cell axes identical,
the polycrystal window within 1e-14 (the two tanh implementations may
differ in the last bits)."""
import time

import numpy as np
import pytest

import llg

pytestmark = pytest.mark.gpu

KINDS = [
    (llg.GEOM_BULK, dict()),
    (llg.GEOM_HOLE_SQUARE, dict(hole_radius_frac_y=0.125)),
    (llg.GEOM_RING, dict()),
    (llg.GEOM_ELLIPSE, dict(active_rx_frac=0.3, active_ry_frac=0.2)),
    (llg.GEOM_ANNULUS, dict()),
    (llg.GEOM_SLIT, dict()),
    (llg.GEOM_POLYCRYSTAL, dict(num_grains=24, dead_grain_frac=0.10, grain_z_bias=1.0)),
    (llg.GEOM_POLYCRYSTAL, dict(num_grains=72, dead_grain_frac=0.16)),
    (llg.GEOM_POLYCRYSTAL, dict(num_grains=5, dead_grain_frac=0.0)),
]


def _compare(spec):
    import torch
    h = llg.build_geometry(spec, want=("active", "w", "msk3", "nsk3", "grain_id"))
    d = llg.build_geometry_device(spec)
    torch.cuda.synchronize()
    assert d["n_active"] == h["n_active"]
    assert np.array_equal(d["active"].cpu().numpy(), h["active"])
    assert np.array_equal(d["grain_id"].cpu().numpy(), h["grain_id"])
    assert np.array_equal(d["msk3"].cpu().numpy(), h["msk3"])
    assert np.array_equal(d["nsk3"].cpu().numpy(), h["nsk3"])
    assert np.abs(d["w"].cpu().numpy() - h["w"]).max() <= 1e-14
    return h, d


@pytest.mark.parametrize("kind,kw", KINDS)
@pytest.mark.parametrize("ng,ny", [(64, 40), (37, 23), (256, 128)])
def test_device_geometry_matches_host_builder(gpu, kind, kw, ng, ny):
    _compare(llg.default_geom(ng, ny, geometry_kind=kind, **kw))


def test_device_polycrystal_at_full_size(gpu):
    """1536x512, 72 grains, 16 % dead (the polycrystal workload's geometry)."""
    import torch
    spec = llg.default_geom(1536, 512, geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=72, dead_grain_frac=0.16,
                            grain_z_bias=1.0)
    t0 = time.perf_counter()
    llg.build_geometry(spec, want=("active", "w", "msk3", "nsk3", "grain_id"))
    th = time.perf_counter() - t0
    llg.build_geometry_device(spec)   # warm-up (module load)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    llg.build_geometry_device(spec)
    torch.cuda.synchronize()
    td = time.perf_counter() - t0
    print(f"polycrystal 1536x512/72 grains: host {th * 1e3:.1f} ms, device {td * 1e3:.1f} ms")
    _compare(spec)
