"""ctypes binding of the C ABI in include/kf_b200.h.

The structures below mirror the header field by field.  Loading fails loudly
when the in-tree library (kinectfusion_b200/libkf_b200.so) is missing: there
is no CPU fallback behind this package.
"""

from __future__ import annotations

import ctypes as C
import pathlib

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libkf_b200.so"
HEADER = HERE.parent / "include" / "kf_b200.h"

KF_OK = 0
KF_ERR_INVALID_ARGUMENT = 1
KF_ERR_CUDA = 2
KF_ERR_NO_DEVICE = 3
KF_ERR_OUT_OF_MEMORY = 4
KF_ERR_DEVICE_TIMEOUT = 5
KF_ERR_UNSUPPORTED = 6
KF_ERR_IO = 7

KF_MEMORY_HOST = 0
KF_MEMORY_DEVICE = 1

KF_VOXEL_FLOAT, KF_VOXEL_QUANTIZED, KF_VOXEL_BF16 = 0, 1, 2
KF_COLOR_FLOAT, KF_COLOR_NONE = 0, 1
KF_STORAGE_DENSE, KF_STORAGE_SPARSE = 0, 1
KF_RULE_CLASSIC, KF_RULE_ANGLE_WEIGHTED = 0, 1
KF_INTEGRATION_FULL, KF_INTEGRATION_BAND = 0, 1
KF_RAYCAST_MARCH, KF_RAYCAST_BITMAP_MARCH, KF_RAYCAST_BAND_MARCH = 0, 1, 2
KF_CORNERS_SKIP_MISSING, KF_CORNERS_REQUIRE_ALL = 0, 1
KF_DAMPING_NONE, KF_DAMPING_IDENTITY, KF_DAMPING_DIAGONAL = 0, 1, 2

KF_ICP_MAX_ITERATIONS = 0
KF_ICP_CONVERGED = 1
KF_ICP_TOO_FEW_CORRESPONDENCES = 2
KF_ICP_SOLVE_FAILED = 3
KF_ICP_UPDATE_TOO_LARGE = 4
KF_ICP_UNCONSTRAINED_SYSTEM = 5
KF_ICP_INVALID_INPUT = 6
KF_ICP_NOT_RUN = 7

ICP_STATUS_NAMES = {
    0: "max_iterations", 1: "converged", 2: "too_few_correspondences", 3: "solve_failed",
    4: "update_too_large", 5: "unconstrained_system", 6: "invalid_input", 7: "not_run",
}


class Intrinsics(C.Structure):
    _fields_ = [("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float)]


class Rigid(C.Structure):
    _fields_ = [("r", C.c_float * 9), ("t", C.c_float * 3)]


class DepthOptions(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("depth_scale", C.c_float), ("min_depth", C.c_float),
                ("max_depth", C.c_float), ("max_normal_depth_jump", C.c_float),
                ("max_downsample_depth_jump", C.c_float), ("bilateral_filter", C.c_int32),
                ("bilateral_radius", C.c_int32), ("bilateral_spatial_sigma", C.c_float),
                ("bilateral_depth_sigma", C.c_float)]


class IntegrationOptions(C.Structure):
    _fields_ = [("depth_scale", C.c_float), ("observation_weight", C.c_float), ("max_weight", C.c_float),
                ("min_depth", C.c_float), ("max_depth", C.c_float), ("projective_distance", C.c_int32),
                ("distance_scaled_truncation", C.c_int32), ("truncation_distance_scale", C.c_float),
                ("mode", C.c_int32)]


class RaycastOptions(C.Structure):
    _fields_ = [("min_depth", C.c_float), ("max_depth", C.c_float), ("step_scale", C.c_float),
                ("corner_policy", C.c_int32), ("cell_gradient_normals", C.c_int32),
                ("seed_from_previous", C.c_int32)]


class VolumeGeometry(C.Structure):
    _fields_ = [("res_x", C.c_uint32), ("res_y", C.c_uint32), ("res_z", C.c_uint32), ("voxel_size", C.c_float),
                ("origin", C.c_float * 3), ("truncation_distance", C.c_float)]


class LaunchShapes(C.Structure):
    _fields_ = [("raycast_block_x", C.c_uint32), ("raycast_block_y", C.c_uint32), ("integrate_ctas", C.c_uint32),
                ("raycast_lanes", C.c_uint32 * 3)]


class PipelineConfig(C.Structure):
    _fields_ = [("volume", VolumeGeometry), ("voxel", C.c_int32), ("color", C.c_int32), ("storage", C.c_int32),
                ("sparse_block_capacity", C.c_uint64), ("tsdf_rule", C.c_int32),
                ("integration", IntegrationOptions), ("raycast", RaycastOptions), ("raycast_backend", C.c_int32)]


class FrameView(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("color", C.c_void_p), ("normals", C.c_void_p), ("width", C.c_uint32),
                ("height", C.c_uint32), ("intrinsics", Intrinsics), ("world_to_camera", Rigid),
                ("memory", C.c_int32)]


class RaycastCamera(C.Structure):
    _fields_ = [("intrinsics", Intrinsics), ("width", C.c_uint32), ("height", C.c_uint32),
                ("camera_to_world", Rigid)]


class SurfaceMapsView(C.Structure):
    _fields_ = [("points", C.c_void_p), ("normals", C.c_void_p), ("colors", C.c_void_p), ("width", C.c_uint32),
                ("height", C.c_uint32), ("memory", C.c_int32)]


class LevelView(C.Structure):
    _fields_ = [("depth", C.c_void_p), ("vertices", C.c_void_p), ("normals", C.c_void_p), ("width", C.c_uint32),
                ("height", C.c_uint32), ("intrinsics", Intrinsics)]


class IcpOptions(C.Structure):
    _fields_ = [("min_correspondences", C.c_uint64), ("max_point_distance", C.c_float),
                ("min_normal_dot", C.c_float), ("min_update_translation", C.c_float),
                ("min_update_rotation", C.c_float), ("max_update_translation", C.c_float),
                ("max_update_rotation", C.c_float), ("min_system_eigenvalue", C.c_float),
                ("max_condition_number", C.c_float), ("damping_mode", C.c_int32), ("damping_lambda", C.c_float),
                ("adaptive_damping", C.c_int32), ("lambda_increase", C.c_float), ("lambda_decrease", C.c_float),
                ("min_lambda", C.c_float), ("max_lambda", C.c_float)]


class IcpOutcome(C.Structure):
    _fields_ = [("pose", Rigid), ("pose_f64", C.c_double * 12), ("status", C.c_int32), ("iterations", C.c_int32),
                ("correspondences", C.c_uint64), ("mean_point_distance", C.c_float),
                ("mean_squared_residual", C.c_float), ("min_system_eigenvalue", C.c_float),
                ("condition_number", C.c_float), ("update_translation", C.c_float),
                ("update_rotation", C.c_float), ("damping_lambda", C.c_float), ("rejected_steps", C.c_uint64)]


class FrameResult(C.Structure):
    _fields_ = [("camera_to_world", Rigid), ("tracked", C.c_int32), ("status", C.c_int32 * 4),
                ("iterations", C.c_int32 * 4), ("correspondences", C.c_uint64 * 4),
                ("world_to_camera", Rigid)]


class Mesh(C.Structure):
    _fields_ = [("positions", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("colors", C.POINTER(C.c_float)), ("triangles", C.POINTER(C.c_uint32)),
                ("vertex_count", C.c_uint64), ("triangle_count", C.c_uint64)]


class WarmStartResult(C.Structure):
    _fields_ = [("start", Rigid), ("proposal", Rigid), ("twist", C.c_float * 6),
                ("cost_predicted", C.c_float), ("matches_predicted", C.c_float),
                ("cost_proposal", C.c_float), ("matches_proposal", C.c_float), ("used_proposal", C.c_int32)]


class VolumeComparison(C.Structure):
    _fields_ = [("compared_voxels", C.c_uint64), ("only_primary", C.c_uint64), ("only_reference", C.c_uint64),
                ("max_distance_delta", C.c_float), ("mean_distance_delta", C.c_float),
                ("max_weight_delta", C.c_float)]


class SurfaceMapsComparison(C.Structure):
    _fields_ = [("compared_pixels", C.c_uint64), ("only_primary", C.c_uint64), ("only_reference", C.c_uint64),
                ("max_point_distance", C.c_float), ("mean_point_distance", C.c_float),
                ("max_normal_angle", C.c_float), ("mean_normal_angle", C.c_float)]


WARM_START_TWIST_SCALE = 50.0  # KF_WARM_START_TWIST_SCALE

P = C.c_void_p
_PROTOTYPES = {
    "kf_last_error": (C.c_char_p, []),
    "kf_abi_version": (C.c_int, []),
    "kf_device_available": (C.c_int, [C.POINTER(C.c_int32)]),
    "kf_default_depth_options": (None, [C.POINTER(DepthOptions)]),
    "kf_default_integration_options": (None, [C.POINTER(IntegrationOptions)]),
    "kf_default_raycast_options": (None, [C.POINTER(RaycastOptions)]),
    "kf_default_icp_options": (None, [C.POINTER(IcpOptions)]),
    "kf_default_pipeline_config": (None, [C.POINTER(PipelineConfig)]),
    "kf_pyramid_create": (C.c_int, [C.POINTER(DepthOptions), C.POINTER(P)]),
    "kf_pyramid_destroy": (C.c_int, [P]),
    "kf_pyramid_build": (C.c_int, [P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32, C.POINTER(C.c_uint32)]),
    "kf_pyramid_level": (C.c_int, [P, C.c_uint32, C.POINTER(LevelView)]),
    "kf_pyramid_download_level": (C.c_int, [P, C.c_uint32, P, P, P]),
    "kf_pipeline_create": (C.c_int, [C.POINTER(PipelineConfig), C.POINTER(P)]),
    "kf_pipeline_destroy": (C.c_int, [P]),
    "kf_pipeline_reset": (C.c_int, [P]),
    "kf_pipeline_reset_async": (C.c_int, [P]),
    "kf_pipeline_integrate": (C.c_int, [P, C.POINTER(FrameView)]),
    "kf_pipeline_raycast": (C.c_int, [P, C.POINTER(RaycastCamera), C.POINTER(SurfaceMapsView)]),
    "kf_pipeline_observed_voxel_count": (C.c_int, [P, C.POINTER(C.c_uint64)]),
    "kf_pipeline_download_volume": (C.c_int, [P, P, P, P]),
    "kf_pipeline_download_raw": (C.c_int, [P, P, C.c_size_t, P, C.c_size_t]),
    "kf_pipeline_download_pool": (C.c_int, [P, P, C.c_size_t]),
    "kf_pyramid_raw_depth": (C.c_int, [P, C.POINTER(C.c_void_p)]),
    "kf_pipeline_render_model": (C.c_int, [P, C.POINTER(RaycastCamera), C.POINTER(SurfaceMapsView)]),
    "kf_icp_level": (C.c_int, [P, C.POINTER(LevelView), P, P, C.c_uint32, C.c_uint32, Intrinsics, C.POINTER(Rigid),
                               C.POINTER(Rigid), C.c_uint32, C.POINTER(IcpOutcome), P]),
    "kf_pipeline_extract_mesh": (C.c_int, [P, C.c_float, C.POINTER(Mesh)]),
    "kf_frame_kernel_count": (C.c_int, [P, C.POINTER(C.c_uint32)]),
    "kf_batch_create": (C.c_int, [P, P, P, C.c_uint32, C.POINTER(P)]),
    "kf_gemm_bf16": (C.c_int, [P, P, P, C.c_int32, C.c_int32, C.c_int32, P, C.c_int32, P]),
    "kf_pipeline_get_launch_shapes": (C.c_int, [P, C.POINTER(LaunchShapes)]),
    "kf_pipeline_set_launch_shapes": (C.c_int, [P, C.POINTER(LaunchShapes)]),
    "kf_pipeline_set_concurrent": (C.c_int, [P, C.c_int32]),
    "kf_pipeline_autotune": (C.c_int, [P, P, C.c_uint32, C.c_uint32, C.c_uint32, Intrinsics, C.POINTER(LaunchShapes),
                                       C.POINTER(C.c_float)]),
    "kf_batch_destroy": (C.c_int, [P]),
    "kf_batch_step": (C.c_int, [P, P, C.c_uint32, C.c_uint32, P, P, P, C.c_int32]),
    "kf_batch_stream": (C.c_int, [P, C.POINTER(P)]),
    "kf_batch_kernel_count": (C.c_int, [P, C.POINTER(C.c_uint32)]),
    "kf_pipeline_block_stats": (C.c_int, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "kf_pipeline_download_block_grid": (C.c_int, [P, P, C.c_size_t]),
    "kf_pipeline_download_skip_structures": (C.c_int, [P, P, P, P, C.c_size_t]),
    "kf_pipeline_download_band_bitmap": (C.c_int, [P, P, C.c_size_t]),
    "kf_pipeline_listed_blocks": (C.c_int, [P, C.POINTER(C.c_uint64)]),
    "kf_mesh_free": (None, [C.POINTER(Mesh)]),
    "kf_pipeline_synchronize": (C.c_int, [P]),
    "kf_pipeline_stream": (C.c_int, [P, C.POINTER(P)]),
    "kf_pipeline_set_kernel_events": (C.c_int, [P, P, P]),
    "kf_pipeline_update_counts": (C.c_int, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "kf_compare_volumes": (C.c_int, [P, P, C.POINTER(VolumeComparison)]),
    "kf_compare_surface_maps": (C.c_int, [C.POINTER(SurfaceMapsView), C.POINTER(SurfaceMapsView),
                                          C.POINTER(SurfaceMapsComparison)]),
    "kf_tracker_create": (C.c_int, [C.POINTER(IcpOptions), C.POINTER(P)]),
    "kf_tracker_destroy": (C.c_int, [P]),
    "kf_tracker_stall_next_level": (C.c_int, [P]),
    "kf_pipeline_track": (C.c_int, [P, P, C.POINTER(RaycastCamera), C.POINTER(LevelView), C.c_uint32,
                                    C.POINTER(IcpOutcome)]),
    "kf_icp_normal_equations": (C.c_int, [P, C.POINTER(LevelView), P, P, C.c_uint32, C.c_uint32, Intrinsics,
                                          C.POINTER(Rigid), C.POINTER(Rigid), P, C.POINTER(C.c_uint64)]),
    "kf_icp_normal_equations_static": (C.c_int, [C.POINTER(LevelView), P, P, C.c_uint32, C.c_uint32, Intrinsics,
                                                 C.POINTER(Rigid), C.POINTER(Rigid), C.c_float, C.c_float, P,
                                                 C.POINTER(C.c_uint64)]),
    "kf_frame_process": (C.c_int, [P, P, P, P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32, P, C.c_int32,
                                   C.POINTER(Rigid), C.POINTER(FrameResult)]),
    "kf_frame_enqueue": (C.c_int, [P, P, P, P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32, P, C.c_int32]),
    "kf_frame_submit": (C.c_int, [P, P, P, P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32, P, C.c_int32]),
    "kf_frame_result_next": (C.c_int, [P, C.POINTER(FrameResult)]),
    "kf_frame_result_fetch": (C.c_int, [P, C.POINTER(FrameResult)]),
    "kf_frame_set_pose": (C.c_int, [P, P, C.POINTER(Rigid)]),
    "kf_png_info": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_int32),
                              C.POINTER(C.c_int32)]),
    "kf_png_read_depth": (C.c_int, [C.c_char_p, P, C.c_uint32, C.c_uint32]),
    "kf_png_read_color": (C.c_int, [C.c_char_p, P, C.c_uint32, C.c_uint32]),
    "kf_png_write_depth": (C.c_int, [C.c_char_p, P, C.c_uint32, C.c_uint32]),
    "kf_png_write_color": (C.c_int, [C.c_char_p, P, C.c_uint32, C.c_uint32]),
    "kf_mesh_write_ply": (C.c_int, [C.c_char_p, C.POINTER(Mesh)]),
    "kf_maps_write_ply": (C.c_int, [C.c_char_p, P, P, P, C.c_uint32, C.c_uint32]),
    "kf_learner_create": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(P)]),
    "kf_learner_destroy": (C.c_int, [P]),
    "kf_learner_param_count": (C.c_int, [P, C.POINTER(C.c_uint64)]),
    "kf_learner_get_params": (C.c_int, [P, P]),
    "kf_learner_set_params": (C.c_int, [P, P]),
    "kf_learner_forward": (C.c_int, [P, P, C.c_uint32, P, P]),
    "kf_learner_gradients": (C.c_int, [P, P, P, C.c_uint32, P, P, P]),
    "kf_learner_train_step": (C.c_int, [P, P, P, C.c_uint32, C.c_float, P, P]),
    "kf_learner_error": (C.c_int, [P, C.POINTER(C.c_int32)]),
    "kf_warm_start_create": (C.c_int, [C.c_float, C.POINTER(P)]),
    "kf_warm_start_destroy": (C.c_int, [P]),
    "kf_warm_start_input": (C.c_int, [P, P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32, C.POINTER(Rigid), P]),
    "kf_warm_start_propose": (C.c_int, [P, P, P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32,
                                        C.POINTER(Rigid), C.POINTER(WarmStartResult)]),
    "kf_warm_start_reset": (C.c_int, [P]),
    "kf_warm_start_enqueue": (C.c_int, [P, P, P, P, P, C.c_uint32, C.c_uint32, Intrinsics, C.c_int32, C.c_int32]),
    "kf_warm_start_fetch": (C.c_int, [P, P, C.POINTER(WarmStartResult)]),
}

_lib = None


class KfError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"kf status {status}: {message}")
        self.status = status


def load() -> C.CDLL:
    """Loads libkf_b200.so and declares every prototype; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m kinectfusion_b200.build` "
                           "(the package has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (restype, argtypes) in _PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != KF_OK:
        msg = load().kf_last_error()
        raise KfError(status, msg.decode() if msg else "")


def declared_functions() -> list[str]:
    """Function names declared in include/kf_b200.h."""
    import re
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:kf_status|void|const char\*|int)\s+(kf_\w+)\s*\(", text, re.M)))


def rigid_from_matrix(m) -> Rigid:
    import numpy as np
    m = np.asarray(m, dtype=np.float64)
    r = Rigid()
    for i in range(3):
        for j in range(3):
            r.r[i * 3 + j] = float(np.float32(m[i, j]))
        r.t[i] = float(np.float32(m[i, 3]))
    return r


def matrix_from_rigid(r: Rigid):
    import numpy as np
    v = np.frombuffer(r, dtype=np.float32, count=12)  # r[9] then t[3], no padding
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = v[:9].reshape(3, 3)
    m[:3, 3] = v[9:]
    return m
