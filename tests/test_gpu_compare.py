"""GPU parity of the pipeline-set comparator (kf_compare_volumes,
kf_compare_surface_maps) and the ablation loop.

Bars: counts and maxima equal to the oracle's (restated Comparator::compare on
the downloaded host views) exactly; the means within one float ulp of the
oracle's sequential double sum (the device sums the same doubles in a fixed
tree order); the normal angles within one float ulp (the device evaluates
atan2 in double and rounds once, the oracle calls the C library's float
atan2).  The reference's own pipeline-set tests (test/tests.cpp:612-768) are
restated on their synthetic fixtures.
"""

import numpy as np
import pytest

import kf_compare_oracle as kco
import kf_oracle as ko
from fixtures import DEPTH_1M, DEPTH_1P4M, SYNTH_IMAGE, SYNTH_ORIGIN, SYNTH_RES, SYNTH_TRUNC, SYNTH_VOXEL, flat_depth, \
    synth_intrinsics
import kinectfusion_b200 as kf
from kinectfusion_b200 import abi, synthetic
from kinectfusion_b200.pipeline_set import (ABLATION_STATS_HEADER, PipelineSet, SetReconstruction,
                                            compare_surface_maps, compare_volumes)

pytestmark = pytest.mark.gpu

K640 = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
EYE = np.eye(4, dtype=np.float32)


@pytest.fixture(scope="module")
def seq():
    return synthetic.make_sequence(seed=1, frames=6)


def cfg1(**kw):
    half = 0.5 * 128 * 0.02
    return kf.pipeline_config(128, 0.02, (-half, -half, -0.5), 0.05, **kw)


def synth(**kw):
    return kf.pipeline_config(SYNTH_RES, SYNTH_VOXEL, SYNTH_ORIGIN, SYNTH_TRUNC, **kw)


def within_ulp(a, b, ulps=1):
    a, b = np.float32(a), np.float32(b)
    return abs(float(a) - float(b)) <= ulps * float(np.spacing(max(abs(a), abs(b))))


def assert_volume_parity(dev, primary, reference):
    o = kco.compare_volumes(primary.host_view(), reference.host_view())
    assert (dev.compared_voxels, dev.only_primary, dev.only_reference) == \
        (o["compared_voxels"], o["only_primary"], o["only_reference"])
    assert dev.max_distance_delta == o["max_distance_delta"]
    assert dev.max_weight_delta == o["max_weight_delta"]
    assert within_ulp(dev.mean_distance_delta, o["mean_distance_delta"]), (dev, o)
    return o


def assert_surface_parity(dev, p, r):
    o = kco.compare_surface_maps(p.points, p.normals, r.points, r.normals)
    assert (dev.compared_pixels, dev.only_primary, dev.only_reference) == \
        (o["compared_pixels"], o["only_primary"], o["only_reference"])
    assert dev.max_point_distance == o["max_point_distance"]
    assert within_ulp(dev.mean_point_distance, o["mean_point_distance"]), (dev, o)
    assert within_ulp(dev.max_normal_angle, o["max_normal_angle"]), (dev, o)
    assert within_ulp(dev.mean_normal_angle, o["mean_normal_angle"]), (dev, o)
    return o


def _feed(pipeline_set, seq, frames):
    for frame in range(frames):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K640, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        pipeline_set.integrate(raw, K640, w2c, normals=normals)


@pytest.fixture(scope="module")
def variants(seq):
    none = dict(color=abi.KF_COLOR_NONE)
    members = [kf.Pipeline(cfg1(**none), "baseline"),
               kf.Pipeline(cfg1(rule=abi.KF_RULE_CLASSIC, **none), "classic"),
               kf.Pipeline(cfg1(voxel=abi.KF_VOXEL_QUANTIZED, **none), "quantized"),
               kf.Pipeline(cfg1(voxel=abi.KF_VOXEL_BF16, **none), "bf16"),
               kf.Pipeline(cfg1(integration_mode=abi.KF_INTEGRATION_BAND, **none), "band"),
               kf.Pipeline(cfg1(integration_mode=abi.KF_INTEGRATION_BAND, storage=abi.KF_STORAGE_SPARSE,
                                voxel=abi.KF_VOXEL_BF16, **none), "sparse-bf16")]
    s = PipelineSet(members, reference="baseline")
    _feed(s, seq, 3)
    return s


def test_volume_comparator_matches_oracle(variants):
    comparisons = variants.compare()
    assert [c.name for c in comparisons] == ["classic", "quantized", "bf16", "band", "sparse-bf16"]
    for c, member in zip(comparisons, variants.members[1:]):
        o = assert_volume_parity(c.volume, member, variants.reference)
        assert o["compared_voxels"] > 0 and c.surface is None
    by_name = {c.name: c.volume for c in comparisons}
    # same observations, different storages (tests.cpp:684-696; the reference's
    # bounds hold for its single flat frame, test_reference_set_cases; over a
    # moving sequence the rounding of each fused average compounds)
    for name in ("quantized", "bf16"):
        v = by_name[name]
        assert v.only_primary == 0 and v.only_reference == 0 and 0.0 < v.max_distance_delta < 0.05
    # band: a subset of the full sweep's voxels (tests.cpp:713-719)
    assert by_name["band"].only_primary == 0 and by_name["band"].only_reference > 0
    # every pair both ways, and a volume against itself
    for member in variants.members:
        assert_volume_parity(compare_volumes(variants.reference, member), variants.reference, member)
    self_cmp = compare_volumes(variants.reference, variants.reference)
    assert self_cmp.compared_voxels == variants.reference.observed_voxel_count() > 0
    assert self_cmp.max_distance_delta == self_cmp.mean_distance_delta == self_cmp.max_weight_delta == 0.0


@pytest.mark.parametrize("storage", [abi.KF_STORAGE_DENSE, abi.KF_STORAGE_SPARSE])
def test_volume_comparator_fresh_volume(variants, storage):
    # a volume no integration touched: every observed voxel is the other side's
    mode = abi.KF_INTEGRATION_BAND if storage == abi.KF_STORAGE_SPARSE else abi.KF_INTEGRATION_FULL
    fresh = kf.Pipeline(cfg1(color=abi.KF_COLOR_NONE, storage=storage, integration_mode=mode))
    for primary, reference in ((fresh, variants.reference), (variants.reference, fresh), (fresh, fresh)):
        c = compare_volumes(primary, reference)
        assert_volume_parity(c, primary, reference)
        assert c.compared_voxels == 0 and c.max_distance_delta == 0.0 and c.mean_distance_delta == 0.0
    assert compare_volumes(fresh, variants.reference).only_reference == variants.reference.observed_voxel_count()


def test_volume_comparator_odd_resolution_all_pairs(seq):
    # resolutions that are not multiples of 8 (edge bricks padded), dense and
    # sparse on either side, every ordered pair against the oracle
    res, origin = (100, 92, 84), (-1.0, -0.92, -0.5)
    none = dict(color=abi.KF_COLOR_NONE)
    band = dict(integration_mode=abi.KF_INTEGRATION_BAND)
    members = [kf.Pipeline(kf.pipeline_config(res, 0.02, origin, 0.05, **none), "float"),
               kf.Pipeline(kf.pipeline_config(res, 0.02, origin, 0.05, voxel=abi.KF_VOXEL_QUANTIZED, **none), "q"),
               kf.Pipeline(kf.pipeline_config(res, 0.02, origin, 0.05, storage=abi.KF_STORAGE_SPARSE, **band,
                                              **none), "sparse"),
               kf.Pipeline(kf.pipeline_config(res, 0.02, origin, 0.05, storage=abi.KF_STORAGE_SPARSE,
                                              voxel=abi.KF_VOXEL_BF16, **band, **none), "sparse-bf16")]
    s = PipelineSet(members)
    _feed(s, seq, 2)
    for a in members:
        for b in members:
            c = compare_volumes(a, b)
            o = assert_volume_parity(c, a, b)
            assert o["compared_voxels"] > 0


def test_volume_comparator_rejects_other_geometry(variants):
    other = kf.Pipeline(kf.pipeline_config(64, 0.02, (-0.64, -0.64, -0.5), 0.05, color=abi.KF_COLOR_NONE))
    with pytest.raises(ValueError, match="matching geometry"):
        compare_volumes(other, variants.reference)


def test_surface_comparator_matches_oracle(variants, seq):
    outputs = variants.raycast_all(K640, 640, 480, seq.poses[2])
    comparisons = variants.compare(outputs)
    ref_host = outputs[0].maps.to_host()
    for c, out in zip(comparisons, outputs[1:]):
        host = out.maps.to_host()
        o = assert_surface_parity(c.surface, host, ref_host)
        assert o["compared_pixels"] > 1000
        # host maps take the staging path to the same kernel and result
        assert compare_surface_maps(host, ref_host) == c.surface
    # the device render equals the host render of Pipeline::raycast
    plain = variants.members[1].raycast(K640, 640, 480, seq.poses[2])
    assert np.array_equal(plain.points, outputs[1].maps.to_host().points, equal_nan=True)


def test_surface_comparator_known_answer():
    # tests.cpp:837-880 through the device kernel
    from test_compare_host import _two_by_two
    pp, pn, rp, rn = _two_by_two()
    c = compare_surface_maps(kf.SurfaceMaps(pp, pn, None), kf.SurfaceMaps(rp, rn, None))
    assert (c.compared_pixels, c.only_primary, c.only_reference) == (1, 1, 1)
    assert c.max_point_distance == pytest.approx(0.1) and c.mean_point_distance == pytest.approx(0.1)
    assert c.max_normal_angle == pytest.approx(np.pi / 2) and c.mean_normal_angle == pytest.approx(np.pi / 2)
    assert_surface_parity(c, kf.SurfaceMaps(pp, pn, None), kf.SurfaceMaps(rp, rn, None))
    # empty maps: nothing compared, zero means (Deviation::mean of no values)
    e = np.zeros((0, 4, 3), np.float32)
    z = compare_surface_maps(kf.SurfaceMaps(e, e, None), kf.SurfaceMaps(e, e, None))
    assert z.compared_pixels == 0 and z.mean_point_distance == 0.0
    with pytest.raises(ValueError, match="matching dimensions"):
        compare_surface_maps(kf.SurfaceMaps(pp, pn, None), kf.SurfaceMaps(rp[:1], rn[:1], None))


# ---- the reference's pipeline-set tests on their fixtures ------------------------------
def _flat(pipeline_set, raws, normals=None):
    for raw in raws:
        pipeline_set.integrate(flat_depth(raw), synth_intrinsics(), EYE, normals=normals)


def test_set_compares_variants_against_reference():
    # tests.cpp:612-649: angle-weighted baseline vs classic, two depths
    s = PipelineSet([kf.Pipeline(synth(), "baseline"), kf.Pipeline(synth(rule=abi.KF_RULE_CLASSIC), "classic")],
                    reference="baseline")
    assert s.size() == 2 and s.should_compare(0) and s.reference is s.members[0]
    normals = np.tile(np.array([0.0, 0.0, -1.0], np.float32), (SYNTH_IMAGE, SYNTH_IMAGE, 1))
    _flat(s, [DEPTH_1M, DEPTH_1P4M], normals)
    outputs = s.raycast_all(synth_intrinsics(), SYNTH_IMAGE, SYNTH_IMAGE, EYE)
    assert len(outputs) == 2
    comparisons = s.compare(outputs)
    assert len(comparisons) == 1 and comparisons[0].name == "classic"
    c = comparisons[0]
    assert c.volume.compared_voxels > 0 and c.volume.max_distance_delta > 0.0
    assert c.surface is not None and c.surface.compared_pixels > 0
    assert_volume_parity(c.volume, s.members[1], s.members[0])
    assert_surface_parity(c.surface, outputs[1].maps.to_host(), outputs[0].maps.to_host())
    with pytest.raises(ValueError):
        s.compare(outputs[:1])


@pytest.mark.parametrize("case", ["storages", "band", "sparse", "overflow"])
def test_reference_set_cases(case):
    band = dict(integration_mode=abi.KF_INTEGRATION_BAND)
    if case == "storages":  # tests.cpp:667-697
        members = [kf.Pipeline(synth(), "float"),
                   kf.Pipeline(synth(voxel=abi.KF_VOXEL_QUANTIZED, color=abi.KF_COLOR_NONE), "quantized"),
                   kf.Pipeline(synth(voxel=abi.KF_VOXEL_BF16, color=abi.KF_COLOR_NONE), "bf16")]
        reference = "float"
    elif case == "band":  # tests.cpp:698-720
        members = [kf.Pipeline(synth(), "full"), kf.Pipeline(synth(**band), "band")]
        reference = "full"
    elif case == "sparse":  # tests.cpp:722-744
        members = [kf.Pipeline(synth(**band), "dense-band"),
                   kf.Pipeline(synth(storage=abi.KF_STORAGE_SPARSE, **band), "sparse")]
        reference = "dense-band"
    else:  # tests.cpp:746-768
        members = [kf.Pipeline(synth(**band), "dense-band"),
                   kf.Pipeline(synth(storage=abi.KF_STORAGE_SPARSE, sparse_block_capacity=1, **band), "tiny")]
        reference = "dense-band"
    s = PipelineSet(members, reference=reference)
    _flat(s, [DEPTH_1M])
    comparisons = s.compare()
    assert len(comparisons) == len(members) - 1
    for c, member in zip(comparisons, members[1:]):
        v = c.volume
        assert_volume_parity(v, member, s.reference)
        if case == "storages":
            assert v.compared_voxels > 0 and v.only_primary == 0 and v.only_reference == 0
            assert v.max_distance_delta > 0.0
        elif case == "band":
            assert v.compared_voxels > 0 and v.max_distance_delta == 0.0
            assert v.only_reference > 0 and v.only_primary == 0
        elif case == "sparse":
            assert v.compared_voxels > 0 and v.max_distance_delta == 0.0
            assert v.only_primary == 0 and v.only_reference == 0
        else:
            assert v.max_distance_delta == 0.0 and v.only_primary == 0 and v.only_reference > 0
    if case == "storages":
        assert comparisons[0].volume.max_distance_delta < 1.0e-4
        assert comparisons[1].volume.max_distance_delta < 5.0e-3


# ---- the ablation loop -------------------------------------------------------------------
def test_set_reconstruction_writes_ablation_stats(seq, tmp_path):
    none = dict(color=abi.KF_COLOR_NONE)
    members = [kf.Pipeline(cfg1(**none), "baseline"),
               kf.Pipeline(cfg1(voxel=abi.KF_VOXEL_QUANTIZED, **none), "quantized"),
               kf.Pipeline(cfg1(rule=abi.KF_RULE_CLASSIC, **none), "classic")]
    loop = SetReconstruction(PipelineSet(members, reference="baseline", compare_every_n_frames=2), K640,
                             output_dir=tmp_path)
    for frame in range(6):
        results = loop.process(seq.depth[frame], seq.color[frame])
        assert len(results) == 3 and all(r.tracked for r in results)
    # frames 0, 2 and 4 compared, two rows each
    assert [f for f, _ in loop.comparisons] == [0, 2, 4]
    lines = (tmp_path / "ablation_stats.csv").read_text().splitlines()
    assert lines[0] + "\n" == ABLATION_STATS_HEADER and len(lines) == 7
    assert [ln.split(",")[:2] for ln in lines[1:3]] == [["0", "quantized"], ["0", "classic"]]
    for frame, comparisons in loop.comparisons:
        for c in comparisons:
            assert c.volume.compared_voxels > 0 and c.surface.compared_pixels > 0
    assert lines[5].startswith("4,quantized,") and lines[5] == "4," + loop.comparisons[2][1][0].csv()
    # each member runs alone: the reference member's trajectory is the one a
    # set of it alone produces, and close to the host-synchronous loop's
    alone = SetReconstruction(PipelineSet([kf.Pipeline(cfg1(**none), "baseline")]), K640)
    sync = kf.Reconstruction(kf.Pipeline(cfg1(**none)), K640)
    for frame in range(6):
        alone.process(seq.depth[frame], seq.color[frame])
        sync.process(seq.depth[frame], seq.color[frame])
    assert all(np.array_equal(a, b) for a, b in zip(alone.trajectories[0], loop.trajectories[0]))
    for a, b in zip(sync.trajectory, loop.trajectories[0]):
        assert np.abs(a - b).max() < 1e-4
    # volumes after the last frame, against the oracle
    for member in members[1:]:
        assert_volume_parity(compare_volumes(member, members[0]), member, members[0])
