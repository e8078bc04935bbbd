"""CPU: the batched workload generator (seeded sizes, shapes, strengths and
initial states of the 64-instance mixed batch) and its geometry set-up."""
import llg


def test_config4_generator_is_seeded_and_covers_every_kind():
    a = llg.config4_instances(64, 12345)
    b = llg.config4_instances(64, 12345)
    assert [x["name"] for x in a] == [x["name"] for x in b]
    assert [x["params"].demag_strength for x in a] == [x["params"].demag_strength for x in b]
    assert {x["shape"] for x in a} == set(llg.CONFIG4_SHAPES)
    assert {(x["params"].ng, x["params"].ny) for x in a} == set(llg.CONFIG4_SIZES)
    for x in a:
        p = x["params"]
        assert 1.0 <= p.demag_strength <= 4.0 and p.demag_mode == llg.DEMAG_OPEN
        assert (p.windowed == 1) == (x["shape"] == "polycrystal")
        assert (p.exec_model == llg.EXEC_COMPACT) == (x["shape"] == "ellipse")
    assert [x["name"] for x in llg.config4_instances(64, 7)] != [x["name"] for x in a]


def test_config4_geometries_build_on_small_grids():
    small = ((64, 64), (96, 48), (64, 96), (128, 64))
    for inst in llg.config4_instances(12, 99, sizes=small):
        geo = llg.build_geometry(inst["geom"])
        p = inst["params"]
        assert geo["y0"].shape == (3 * p.ng * p.ny,)
        assert 0 < geo["active"].sum() < p.ng * p.ny + 1
