"""The C-ABI library loads and exports every symbol include/kf_b200.h declares;
defaults mirror the reference's C++ default member values (CPU only)."""

import ctypes as C

import numpy as np
import pytest

from kinectfusion_b200 import abi
import kinectfusion_b200 as kf


def test_library_exports_every_declared_symbol():
    lib = abi.load()
    declared = abi.declared_functions()
    assert len(declared) >= 30
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing
    assert lib.kf_abi_version() == 1


def test_struct_sizes_match_header_layout():
    # field-by-field mirrors: sizes pin the padding the C compiler chose
    assert C.sizeof(abi.Rigid) == 48
    assert C.sizeof(abi.Intrinsics) == 16
    assert C.sizeof(abi.VolumeGeometry) == 32
    assert C.sizeof(abi.FrameView) == 8 * 3 + 8 + 16 + 48 + 4 + 4
    assert C.sizeof(abi.FrameResult) == 48 + 4 + 16 + 16 + 4 + 32 + 48  # 4 B of padding before the u64s


def test_defaults_mirror_reference():
    d = kf.default_depth_options()
    assert (d.levels, d.bilateral_radius) == (3, 2)
    assert np.isclose(d.bilateral_depth_sigma, 0.08) and np.isclose(d.max_normal_depth_jump, 0.1)
    i = kf.default_icp_options()
    assert i.min_correspondences == 64 and np.isclose(i.min_normal_dot, 0.9659258)
    assert np.isclose(i.max_update_translation, 0.15) and np.isclose(i.max_update_rotation, 0.35)
    c = kf.pipeline_config(512, 0.01, (-2.56, -2.56, -0.5), 0.05)
    assert c.voxel == abi.KF_VOXEL_FLOAT and c.color == abi.KF_COLOR_FLOAT
    assert c.tsdf_rule == abi.KF_RULE_ANGLE_WEIGHTED and c.raycast_backend == abi.KF_RAYCAST_MARCH
    assert np.isclose(c.integration.max_weight, 196.0) and np.isclose(c.raycast.max_depth, 8.0)


def test_no_device_fails_loudly():
    if kf.device_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        kf.Pipeline(kf.pipeline_config(32, 0.05, (-0.8, -0.8, 0.2), 0.05))
    with pytest.raises(RuntimeError):
        kf.PyramidSource()


def test_misconfiguration_rejected_before_device():
    # Pipeline::create validates before touching the device (pipeline.cpp:129-147)
    with pytest.raises(ValueError):
        kf.Pipeline(kf.pipeline_config(32, 0.05, (-0.8, -0.8, 0.2), 0.05, storage=abi.KF_STORAGE_SPARSE))
    with pytest.raises(ValueError):
        kf.Pipeline(kf.pipeline_config(0, 0.05, (-0.8, -0.8, 0.2), 0.05))
    with pytest.raises(ValueError):
        kf.Pipeline(kf.pipeline_config(32, 0.05, (-0.8, -0.8, 0.2), 0.0))
