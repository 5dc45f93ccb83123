"""Host side of the pipeline-set ablations (no GPU): the comparator oracle
pinned to the reference's known-answer test, the set's validation rules,
and the ablation_stats.csv format."""

import ctypes as C
import math
import types

import numpy as np
import pytest

import kf_compare_oracle as kco
from kinectfusion_b200 import abi
from kinectfusion_b200.pipeline_set import (ABLATION_STATS_HEADER, AblationStats, PipelineComparison, PipelineSet,
                                            SurfaceMapsComparison, VolumeComparison, format_float)

NAN3 = [np.nan, np.nan, np.nan]


def _two_by_two():
    """tests.cpp:837-869: one compared pixel, one per side only."""
    pp = np.full((2, 2, 3), np.nan, np.float32)
    pn = np.full((2, 2, 3), np.nan, np.float32)
    rp = np.full((2, 2, 3), np.nan, np.float32)
    rn = np.full((2, 2, 3), np.nan, np.float32)
    pp[0, 0], pn[0, 0] = [0, 0, 1], [1, 0, 0]
    rp[0, 0], rn[0, 0] = [0.1, 0, 1], [0, 1, 0]
    pp[0, 1], pn[0, 1] = [0, 0, 1], [0, 0, -1]  # at(1, 0): x = 1, y = 0
    rp[1, 0], rn[1, 0] = [0, 0, 1], [0, 0, -1]  # at(0, 1)
    return pp, pn, rp, rn


def test_oracle_surface_known_answer():
    # tests.cpp:870-879
    c = kco.compare_surface_maps(*_two_by_two())
    assert c["compared_pixels"] == 1 and c["only_primary"] == 1 and c["only_reference"] == 1
    assert c["max_point_distance"] == pytest.approx(0.1) and c["mean_point_distance"] == pytest.approx(0.1)
    assert c["max_normal_angle"] == pytest.approx(math.pi / 2) and c["mean_normal_angle"] == pytest.approx(math.pi / 2)


def test_oracle_surface_rules():
    rng = np.random.default_rng(3)
    pp = rng.normal(size=(6, 7, 3)).astype(np.float32)
    pn = rng.normal(size=(6, 7, 3)).astype(np.float32)
    # identical maps: every valid pixel compared with zero deviation
    c = kco.compare_surface_maps(pp, pn, pp, pn)
    assert c["compared_pixels"] == 42 and c["max_point_distance"] == 0.0 and c["max_normal_angle"] == 0.0
    # a zero normal normalises to zero: angle atan2(0, 0) = 0, still compared
    rn = pn.copy()
    rn[0, 0] = 0.0
    assert kco.compare_surface_maps(pp, pn, pp, rn)["compared_pixels"] == 42
    # any non-finite component of a point or normal drops the pixel
    rp = pp.copy()
    rp[1, 1, 2] = np.inf
    rn[2, 2, 0] = np.nan
    c = kco.compare_surface_maps(pp, pn, rp, rn)
    assert c["compared_pixels"] == 40 and c["only_primary"] == 2 and c["only_reference"] == 0
    # opposite normals: pi
    assert kco.compare_surface_maps(pp[:1, :1], pn[:1, :1], pp[:1, :1], -pn[:1, :1])["max_normal_angle"] == \
        pytest.approx(math.pi)
    with pytest.raises(ValueError):
        kco.compare_surface_maps(pp, pn, pp[:, :3], pn[:, :3])


def test_oracle_volume_rules():
    pt = np.array([0.5, -0.25, 1.0, 0.0, 0.75], np.float32)
    pw = np.array([1.0, 2.0, 0.0, 3.0, 0.0], np.float32)
    rt = np.array([0.25, -0.25, 0.5, 1.0, 1.0], np.float32)
    rw = np.array([3.0, 2.0, 1.0, 0.0, 0.0], np.float32)
    c = kco.compare_volumes((pt, pw), (rt, rw))
    assert (c["compared_voxels"], c["only_primary"], c["only_reference"]) == (2, 1, 1)
    assert c["max_distance_delta"] == 0.25 and c["mean_distance_delta"] == 0.125 and c["max_weight_delta"] == 2.0
    empty = kco.compare_volumes((pt, np.zeros(5, np.float32)), (rt, np.zeros(5, np.float32)))
    assert empty == {"compared_voxels": 0, "only_primary": 0, "only_reference": 0, "max_distance_delta": 0.0,
                     "mean_distance_delta": 0.0, "max_weight_delta": 0.0}
    with pytest.raises(ValueError):
        kco.compare_volumes((pt, pw), (rt[:4], rw[:4]))


def test_oracle_mean_is_a_sequential_double_sum():
    # Deviation::add sums in double one value at a time: 1 + 1e-8 * n stays
    # visible where a float sum would lose it
    values = np.array([1.0] + [1e-8] * 1000, np.float32)
    assert kco._sequential_sum(values) == pytest.approx(1.0 + 1e-5, rel=1e-9)


@pytest.mark.parametrize("value,text", [(0.0, "0"), (1.0, "1"), (0.1, "0.1"), (2.5, "2.5"), (100.0, "100"),
                                        (1.5e-5, "1.5e-05"), (1e-4, "1e-04"), (0.001, "0.001"),
                                        (0.00012345, "0.00012345"), (3.1415927, "3.1415927"),
                                        (1e20, "1e+20"), (123456792.0, "123456792"), (65535.0, "65535"),
                                        (float("nan"), "nan"), (float("inf"), "inf"),
                                        (0.0012345678, "0.0012345678"), (1.0 / 3.0, "0.33333334")])
def test_csv_floats_follow_std_format(value, text):
    # std::format("{}", float): shortest round trip, fixed unless scientific is shorter
    assert format_float(value) == text
    if np.isfinite(value):
        assert np.float32(format_float(value)) == np.float32(value)


def _comparison(surface=True):
    v = VolumeComparison(120, 3, 4, 0.5, 0.0625, 2.0)
    s = SurfaceMapsComparison(300, 1, 2, 0.01, 0.005, 1.5707964, 0.25) if surface else None
    return PipelineComparison("classic", v, s)


def test_csv_rows_follow_logging_formatters():
    # logging.hpp:85-133: name, six volume fields, seven surface fields
    assert _comparison().csv() == "classic,120,3,4,0.5,0.0625,2,300,1,2,0.01,0.005,1.5707964,0.25"
    # surface absent: the seven surface columns stay empty
    row = _comparison(surface=False).csv()
    assert row == "classic,120,3,4,0.5,0.0625,2,,,,,,,"
    assert len(row.split(",")) == len(ABLATION_STATS_HEADER.strip().split(",")) - 1


def test_ablation_stats_file(tmp_path):
    # frame_output.cpp:215-242: truncated with a header by the first call,
    # appended afterwards, nothing written for an empty list
    stats = AblationStats(tmp_path / "out")
    stats.append(0, [])
    assert not stats.path.exists()
    (tmp_path / "out").mkdir()
    stats.path.write_text("stale\n")
    stats.append(0, [_comparison()])
    stats.append(5, [_comparison(), _comparison(surface=False)])
    lines = stats.path.read_text().splitlines()
    assert lines[0] + "\n" == ABLATION_STATS_HEADER
    assert lines[1].startswith("0,classic,120,") and lines[2].startswith("5,classic,")
    assert lines[3].endswith(",2,,,,,,,") and len(lines) == 4


def _fake(name, res=32, voxel=0.05):
    cfg = abi.PipelineConfig()
    cfg.volume.res_x = cfg.volume.res_y = cfg.volume.res_z = res
    cfg.volume.voxel_size = voxel
    # a set switches its members to concurrent frames (no device here)
    return types.SimpleNamespace(name=name, config=cfg, set_concurrent=lambda concurrent=True: None)


def test_pipeline_set_validation():
    # PipelineSet::create (pipeline_set.cpp:33-79), tests.cpp:651-664
    with pytest.raises(ValueError):
        PipelineSet([])
    with pytest.raises(ValueError):
        PipelineSet([_fake("a"), _fake("a")])
    with pytest.raises(ValueError):
        PipelineSet([_fake("a")], reference="missing")
    with pytest.raises(ValueError):
        PipelineSet([_fake("a"), _fake("b", res=64)])
    with pytest.raises(ValueError):
        PipelineSet([_fake("a"), _fake("b", voxel=0.02)])
    s = PipelineSet([_fake("a"), _fake("b"), _fake("c")], reference="b", compare_every_n_frames=3)
    assert s.size() == 3 and s.reference_index == 1 and s.reference.name == "b"
    assert [s.should_compare(i) for i in range(7)] == [True, False, False, True, False, False, True]
    assert PipelineSet([_fake("a"), _fake("b")]).reference_index == 0
    # a lone pipeline or a non-positive cadence never compares
    assert not PipelineSet([_fake("a")]).should_compare(0)
    assert not PipelineSet([_fake("a"), _fake("b")], compare_every_n_frames=0).should_compare(0)


def test_comparison_structs_match_header_layout():
    assert C.sizeof(abi.VolumeComparison) == 40
    assert C.sizeof(abi.SurfaceMapsComparison) == 40
