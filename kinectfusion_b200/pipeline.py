"""Python mirror of the reference's `--space cuda` interfaces over the C ABI.

Names and argument meanings follow include/kinectfusion/pipeline.hpp
(Pipeline), depth_processing.hpp (PyramidSource), icp_optimizer.hpp
(ProjectiveIcpTracker) and src/app/reconstruction.cpp (the frame loop).
Errors map like the reference's: misconfiguration raises ValueError
(std::invalid_argument), CUDA failures raise RuntimeError.  There is no host
fallback: without a CUDA device every constructor raises.
"""

from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import abi

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = abi.load()
    return _lib


def _check(status: int) -> None:
    if status == abi.KF_OK:
        return
    msg = (lib().kf_last_error() or b"").decode()
    if status in (abi.KF_ERR_INVALID_ARGUMENT, abi.KF_ERR_UNSUPPORTED):
        raise ValueError(msg)
    raise RuntimeError(f"kf status {status}: {msg}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def device_available() -> bool:
    out = C.c_int32()
    _check(lib().kf_device_available(C.byref(out)))
    return bool(out.value)


# ---- defaults -----------------------------------------------------------------------
def default_depth_options(**kw) -> abi.DepthOptions:
    o = abi.DepthOptions()
    lib().kf_default_depth_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_icp_options(**kw) -> abi.IcpOptions:
    o = abi.IcpOptions()
    lib().kf_default_icp_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def pipeline_config(resolution, voxel_size, origin, truncation, *, voxel=abi.KF_VOXEL_FLOAT,
                    color=abi.KF_COLOR_FLOAT, rule=abi.KF_RULE_ANGLE_WEIGHTED, storage=abi.KF_STORAGE_DENSE,
                    integration_mode=abi.KF_INTEGRATION_FULL, raycast_backend=abi.KF_RAYCAST_MARCH,
                    sparse_block_capacity=0, **options) -> abi.PipelineConfig:
    """PipelineConfig (pipeline.hpp:29-46); extra keywords set integration_*
    or raycast_* option fields, e.g. raycast_cell_gradient_normals=1."""
    c = abi.PipelineConfig()
    lib().kf_default_pipeline_config(C.byref(c))
    rx, ry, rz = (resolution,) * 3 if np.isscalar(resolution) else resolution
    c.volume = abi.VolumeGeometry(rx, ry, rz, voxel_size, (C.c_float * 3)(*origin), truncation)
    c.voxel, c.color, c.tsdf_rule, c.storage = voxel, color, rule, storage
    c.integration.mode = integration_mode
    c.raycast_backend = raycast_backend
    c.sparse_block_capacity = sparse_block_capacity
    for key, value in options.items():
        group, _, field = key.partition("_")
        setattr(getattr(c, group), field, value)
    return c


# ---- PyramidSource ------------------------------------------------------------------
class PyramidSource:
    """PyramidSource::create_device (depth_processing.hpp:422-463)."""

    def __init__(self, options: abi.DepthOptions | None = None):
        self.options = options if options is not None else default_depth_options()
        handle = C.c_void_p()
        _check(lib().kf_pyramid_create(C.byref(self.options), C.byref(handle)))
        self.handle = handle
        self.levels = 0

    def close(self):
        if getattr(self, "handle", None):
            lib().kf_pyramid_destroy(self.handle)
            self.handle = None

    __del__ = close

    def build(self, depth: np.ndarray, intrinsics: abi.Intrinsics) -> int:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        count = C.c_uint32()
        _check(lib().kf_pyramid_build(self.handle, _ptr(depth), depth.shape[1], depth.shape[0], intrinsics,
                                      abi.KF_MEMORY_HOST, C.byref(count)))
        self.levels = count.value
        return self.levels

    def level(self, index: int) -> abi.LevelView:
        v = abi.LevelView()
        _check(lib().kf_pyramid_level(self.handle, index, C.byref(v)))
        return v

    def download_level(self, index: int) -> dict:
        v = self.level(index)
        depth = np.empty((v.height, v.width), dtype=np.uint16)
        verts = np.empty((v.height, v.width, 3), dtype=np.float32)
        norms = np.empty((v.height, v.width, 3), dtype=np.float32)
        _check(lib().kf_pyramid_download_level(self.handle, index, _ptr(depth), _ptr(verts), _ptr(norms)))
        return {"depth": depth, "vertices": verts, "normals": norms, "intrinsics": v.intrinsics}


# ---- ProjectiveIcpTracker -----------------------------------------------------------
class ProjectiveIcpTracker:
    """ProjectiveIcpTracker with the device Gauss-Newton loop (icp_optimizer.hpp:107-196)."""

    def __init__(self, options: abi.IcpOptions | None = None):
        self.options = options if options is not None else default_icp_options()
        handle = C.c_void_p()
        _check(lib().kf_tracker_create(C.byref(self.options), C.byref(handle)))
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            lib().kf_tracker_destroy(self.handle)
            self.handle = None

    __del__ = close


@dataclasses.dataclass
class SurfaceMaps:
    points: np.ndarray
    normals: np.ndarray
    colors: np.ndarray


# ---- Pipeline -----------------------------------------------------------------------
class Pipeline:
    """Pipeline::create_device (pipeline.hpp:64-161) on one B200."""

    def __init__(self, config: abi.PipelineConfig, name: str = "baseline"):
        if not name:
            raise ValueError("Pipeline requires a non-empty name")  # pipeline.cpp:130
        self.name = name
        self.config = config
        handle = C.c_void_p()
        _check(lib().kf_pipeline_create(C.byref(config), C.byref(handle)))
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            lib().kf_pipeline_destroy(self.handle)
            self.handle = None

    __del__ = close

    @property
    def resolution(self):
        g = self.config.volume
        return g.res_x, g.res_y, g.res_z

    def reset(self, wait: bool = True):
        """Empty the volume; wait=False queues the refill on the pipeline's
        stream and returns at once (kf_pipeline_reset_async)."""
        _check(lib().kf_pipeline_reset(self.handle) if wait else lib().kf_pipeline_reset_async(self.handle))

    def integrate(self, depth, intrinsics, world_to_camera, color=None, normals=None):
        """Pipeline::integrate (pipeline.hpp:75-79); world_to_camera is a 4x4 or abi.Rigid."""
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        color = None if color is None else np.ascontiguousarray(color, dtype=np.uint32)
        normals = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32)
        w2c = world_to_camera if isinstance(world_to_camera, abi.Rigid) else abi.rigid_from_matrix(world_to_camera)
        f = abi.FrameView(_ptr(depth), _ptr(color), _ptr(normals), depth.shape[1], depth.shape[0], intrinsics, w2c,
                          abi.KF_MEMORY_HOST)
        _check(lib().kf_pipeline_integrate(self.handle, C.byref(f)))

    def raycast(self, intrinsics, width, height, camera_to_world, seed_points=None) -> SurfaceMaps:
        """Pipeline::raycast (pipeline.hpp:81)."""
        c2w = camera_to_world if isinstance(camera_to_world, abi.Rigid) else abi.rigid_from_matrix(camera_to_world)
        cam = abi.RaycastCamera(intrinsics, width, height, c2w)
        points = np.full((height, width, 3), np.nan, dtype=np.float32) if seed_points is None else \
            np.ascontiguousarray(seed_points, dtype=np.float32).copy()
        normals = np.empty((height, width, 3), dtype=np.float32)
        colors = np.empty((height, width), dtype=np.uint32)
        maps = abi.SurfaceMapsView(_ptr(points), _ptr(normals), _ptr(colors), width, height, abi.KF_MEMORY_HOST)
        _check(lib().kf_pipeline_raycast(self.handle, C.byref(cam), C.byref(maps)))
        return SurfaceMaps(points, normals, colors)

    def track(self, tracker: ProjectiveIcpTracker, intrinsics, width, height, camera_to_world,
              live: abi.LevelView, iterations: int) -> abi.IcpOutcome:
        """Pipeline::track + ProjectiveIcpTracker::estimate_pose (pipeline.hpp:84-85)."""
        c2w = camera_to_world if isinstance(camera_to_world, abi.Rigid) else abi.rigid_from_matrix(camera_to_world)
        cam = abi.RaycastCamera(intrinsics, width, height, c2w)
        out = abi.IcpOutcome()
        _check(lib().kf_pipeline_track(self.handle, tracker.handle, C.byref(cam), C.byref(live), iterations,
                                       C.byref(out)))
        return out

    def observed_voxel_count(self) -> int:
        n = C.c_uint64()
        _check(lib().kf_pipeline_observed_voxel_count(self.handle, C.byref(n)))
        return n.value

    def host_view(self, with_color=False):
        """Pipeline::host_view (pipeline.hpp:90): dense (tsdf, weight[, color]) shaped (z, y, x)."""
        rx, ry, rz = self.resolution
        tsdf = np.empty((rz, ry, rx), dtype=np.float32)
        weight = np.empty((rz, ry, rx), dtype=np.float32)
        color = np.empty((rz, ry, rx, 4), dtype=np.float32) if with_color else None
        _check(lib().kf_pipeline_download_volume(self.handle, _ptr(tsdf), _ptr(weight), _ptr(color)))
        return (tsdf, weight, color) if with_color else (tsdf, weight)

    def download_raw(self) -> np.ndarray:
        rx, ry, rz = self.resolution
        n = rx * ry * rz
        if self.config.voxel == abi.KF_VOXEL_FLOAT:
            raw = np.empty((n, 2), dtype=np.float32)
        else:
            raw = np.empty(n, dtype=np.uint32)
        _check(lib().kf_pipeline_download_raw(self.handle, _ptr(raw), raw.nbytes, None, 0))
        return raw

    def skip_structures(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """Dense storage: the march's skip structures (kf_pipeline_download_skip_structures):
        per-brick class and cube radius shaped (bz, by, bx), and the stencil records
        shaped (bz, by, bx, 8 layers, 4 words)."""
        rx, ry, rz = self.resolution
        shape = ((rz + 7) // 8, (ry + 7) // 8, (rx + 7) // 8)
        n = shape[0] * shape[1] * shape[2]
        cls, radius = np.empty(n, dtype=np.uint8), np.empty(n, dtype=np.uint8)
        records = np.empty(n * 32, dtype=np.uint32)
        _check(lib().kf_pipeline_download_skip_structures(self.handle, _ptr(cls), _ptr(radius), _ptr(records), n))
        return cls.reshape(shape), radius.reshape(shape), records.reshape(shape + (8, 4))

    def download_pool(self) -> np.ndarray:
        """Sparse storage: the raw block pool, (capacity, 512) voxels in slot
        order (kf_pipeline_download_pool)."""
        _, capacity = self.block_stats()
        if self.config.voxel == abi.KF_VOXEL_FLOAT:
            raw = np.empty((capacity, 512, 2), dtype=np.float32)
        else:
            raw = np.empty((capacity, 512), dtype=np.uint32)
        _check(lib().kf_pipeline_download_pool(self.handle, _ptr(raw), raw.nbytes))
        return raw

    def launch_shapes(self) -> abi.LaunchShapes:
        shapes = abi.LaunchShapes()
        _check(lib().kf_pipeline_get_launch_shapes(self.handle, C.byref(shapes)))
        return shapes

    def set_launch_shapes(self, raycast_block=(16, 4), integrate_ctas=148 * 48, raycast_lanes=None):
        """raycast_lanes: lanes per ray for renders of <= 20,000 rays, <=
        80,000 rays and more (each 1, 2 or 4); None keeps the current ones."""
        lanes = tuple(self.launch_shapes().raycast_lanes) if raycast_lanes is None else tuple(raycast_lanes)
        shapes = abi.LaunchShapes(raycast_block[0], raycast_block[1], integrate_ctas, (C.c_uint32 * 3)(*lanes))
        _check(lib().kf_pipeline_set_launch_shapes(self.handle, C.byref(shapes)))

    def set_concurrent(self, concurrent: bool = True):
        """Frames run beside other GPU work (kf_pipeline_set_concurrent): the
        ICP levels become per-step launches that can share the GPU."""
        _check(lib().kf_pipeline_set_concurrent(self.handle, 1 if concurrent else 0))

    def autotune(self, device_frames: int, count: int, intrinsics: abi.Intrinsics, width: int = 640,
                 height: int = 480) -> tuple[abi.LaunchShapes, float]:
        """kf_pipeline_autotune over `count` consecutive device-resident frames."""
        shapes, ms = abi.LaunchShapes(), C.c_float()
        _check(lib().kf_pipeline_autotune(self.handle, C.c_void_p(device_frames), count, width, height, intrinsics,
                                          C.byref(shapes), C.byref(ms)))
        return shapes, ms.value

    def block_stats(self) -> tuple[int, int]:
        """Sparse storage: (allocation attempts, capacity) of the block pool."""
        attempts, capacity = C.c_uint64(), C.c_uint64()
        _check(lib().kf_pipeline_block_stats(self.handle, C.byref(attempts), C.byref(capacity)))
        return attempts.value, capacity.value

    def block_grid(self) -> np.ndarray:
        """Sparse storage: the block-slot grid (0xFFFFFFFF = unallocated)."""
        rx, ry, rz = self.resolution
        grid = np.empty(((rx + 7) // 8) * ((ry + 7) // 8) * ((rz + 7) // 8), dtype=np.uint32)
        _check(lib().kf_pipeline_download_block_grid(self.handle, _ptr(grid), grid.size))
        return grid

    def listed_blocks(self) -> int:
        """8^3 blocks the last integration visited."""
        n = C.c_uint64()
        _check(lib().kf_pipeline_listed_blocks(self.handle, C.byref(n)))
        return n.value

    def band_bitmap(self) -> np.ndarray:
        """band-march backend: the dilated band bitmap (z-major block bits)."""
        rx, ry, rz = self.resolution
        blocks = ((rx + 7) // 8) * ((ry + 7) // 8) * ((rz + 7) // 8)
        words = np.empty((blocks + 31) // 32, dtype=np.uint32)
        _check(lib().kf_pipeline_download_band_bitmap(self.handle, _ptr(words), words.size))
        return words

    def extract_mesh(self, min_weight: float = 0.0) -> dict:
        """Pipeline::extract_mesh (pipeline.hpp:95) on the device."""
        mesh = abi.Mesh()
        _check(lib().kf_pipeline_extract_mesh(self.handle, min_weight, C.byref(mesh)))
        nv, nt = mesh.vertex_count, mesh.triangle_count
        try:
            return {
                "positions": np.ctypeslib.as_array(mesh.positions, (nv, 3)).copy() if nv else np.zeros((0, 3), np.float32),
                "normals": np.ctypeslib.as_array(mesh.normals, (nv, 3)).copy() if nv else np.zeros((0, 3), np.float32),
                "colors": np.ctypeslib.as_array(mesh.colors, (nv, 3)).copy() if nv else np.zeros((0, 3), np.float32),
                "triangles": np.ctypeslib.as_array(mesh.triangles, (nt, 3)).copy() if nt else np.zeros((0, 3), np.uint32),
            }
        finally:
            lib().kf_mesh_free(C.byref(mesh))


ICP_ITERATIONS = (10, 5, 4, 4)  # AppOptions::icp_iterations_for_level (app_options.cpp:147-158)


class Reconstruction:
    """The per-frame loop of src/app/reconstruction.cpp:143-277 over one
    pipeline: the first frame is fused at the start pose, every later frame is
    tracked level by level and fused when tracking succeeds, all inside one
    CUDA graph per frame (kf_frame_process)."""

    def __init__(self, pipeline: Pipeline, intrinsics: abi.Intrinsics, depth_options=None, icp_options=None,
                 iterations=ICP_ITERATIONS):
        self.pipeline = pipeline
        self.intrinsics = intrinsics
        self.pyramid = PyramidSource(depth_options)
        self.tracker = ProjectiveIcpTracker(icp_options)
        self.iterations = (C.c_uint32 * 4)(*iterations)
        self.pose = abi.rigid_from_matrix(np.eye(4))
        self.frames = 0
        self.trajectory = []
        self.results = []

    def process(self, depth, color=None) -> abi.FrameResult:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        color = None if color is None else np.ascontiguousarray(color, dtype=np.uint32)
        result = abi.FrameResult()
        _check(lib().kf_frame_process(self.pipeline.handle, self.pyramid.handle, self.tracker.handle, _ptr(depth),
                                      _ptr(color), depth.shape[1], depth.shape[0], self.intrinsics,
                                      abi.KF_MEMORY_HOST, self.iterations, 1 if self.frames == 0 else 0,
                                      C.byref(self.pose), C.byref(result)))
        self.frames += 1
        self.trajectory.append(abi.matrix_from_rigid(self.pose))
        self.results.append(result)
        return result


class PipelinedReconstruction(Reconstruction):
    """The same loop with frames in flight (kf_frame_submit /
    kf_frame_result_next): submit() returns once the frame is copied into the
    pipeline's staging and launched, so the host prepares the next frame
    while the device still works; results come back in submission order.
    The pose stays on the device between frames (FP64), where process()
    rounds it to float and sends it back each frame."""

    RESULTS_IN_FLIGHT = 8

    def submit(self, depth, color=None) -> None:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        color = None if color is None else np.ascontiguousarray(color, dtype=np.uint32)
        if self.frames == 0:
            _check(lib().kf_frame_set_pose(self.pipeline.handle, self.tracker.handle, C.byref(self.pose)))
        _check(lib().kf_frame_submit(self.pipeline.handle, self.pyramid.handle, self.tracker.handle, _ptr(depth),
                                     _ptr(color), depth.shape[1], depth.shape[0], self.intrinsics,
                                     abi.KF_MEMORY_HOST, self.iterations, 1 if self.frames == 0 else 0))
        self.frames += 1

    def next_result(self) -> abi.FrameResult:
        result = abi.FrameResult()
        _check(lib().kf_frame_result_next(self.pipeline.handle, C.byref(result)))
        self.pose = result.camera_to_world
        self.trajectory.append(abi.matrix_from_rigid(result.camera_to_world))
        self.results.append(result)
        return result


class Batch:
    """Independent sequences stepped together (kf_batch_*): one graph launch
    runs one frame of every member.  Each member is a Reconstruction-like
    triple (pipeline, pyramid, tracker) over its own volume."""

    def __init__(self, pipelines: list[Pipeline], intrinsics: abi.Intrinsics, depth_options=None, icp_options=None,
                 iterations=ICP_ITERATIONS):
        self.pipelines = list(pipelines)
        self.pyramids = [PyramidSource(depth_options) for _ in self.pipelines]
        self.trackers = [ProjectiveIcpTracker(icp_options) for _ in self.pipelines]
        n = len(self.pipelines)
        arr = C.c_void_p * n
        self.handle = C.c_void_p()
        _check(lib().kf_batch_create(arr(*[p.handle for p in self.pipelines]),
                                     arr(*[p.handle for p in self.pyramids]),
                                     arr(*[t.handle for t in self.trackers]), n, C.byref(self.handle)))
        self.intrinsics = (abi.Intrinsics * n)(*([intrinsics] * n))
        self.iterations = (C.c_uint32 * 4)(*iterations)
        self.frames = [0] * n

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value:
            lib().kf_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def step(self, device_depths: list, width: int = 640, height: int = 480):
        """device_depths[i]: device address of member i's u16 depth frame, or
        None when member i sits this step out."""
        n = len(self.pipelines)
        depths = (C.c_void_p * n)(*[d if d is not None else None for d in device_depths])
        first = (C.c_uint8 * n)(*[1 if (d is not None and self.frames[i] == 0) else 0
                                  for i, d in enumerate(device_depths)])
        _check(lib().kf_batch_step(self.handle, depths, width, height, self.intrinsics, self.iterations, first,
                                   abi.KF_MEMORY_DEVICE))
        for i, d in enumerate(device_depths):
            if d is not None:
                self.frames[i] += 1

    def stream(self) -> int:
        s = C.c_void_p()
        _check(lib().kf_batch_stream(self.handle, C.byref(s)))
        return s.value

    def kernel_count(self) -> int:
        k = C.c_uint32()
        _check(lib().kf_batch_kernel_count(self.handle, C.byref(k)))
        return k.value

    def result(self, i: int) -> abi.FrameResult:
        r = abi.FrameResult()
        _check(lib().kf_frame_result_fetch(self.pipelines[i].handle, C.byref(r)))
        return r
