"""ctypes binding of oracle/_ref/libkf_ref.so: the reference's own host
implementation, compiled from its sources by oracle/ref_build.sh.

TEST INFRASTRUCTURE ONLY.  The tests compare oracle/kf_oracle.c (the C
restatement the sm_100a kernels are checked against) with this library on
the same inputs; nothing in the product path loads it.  Array layouts match
kf_oracle.py: depth (h, w) uint16, vertex/normal/point maps (h, w, 3) float32,
raw voxels as the reference stores them (float voxel = (tsdf, weight) float
pair; int16/bf16 voxel = uint32 with the distance code in the low 16 bits and
the weight code in the high 16 bits; colour voxel = 4 floats).
"""

from __future__ import annotations

import ctypes as C
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
LIB = HERE / "_ref" / "libkf_ref.so"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from kinectfusion_b200 import abi  # noqa: E402  (POD structs shared with the C ABI header)

P = C.c_void_p
_lib = None


def available() -> bool:
    return LIB.exists()


def build() -> pathlib.Path:
    subprocess.run(["bash", str(HERE / "ref_build.sh")], check=True, capture_output=True)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB.exists():
        raise FileNotFoundError(f"{LIB} is not built (oracle/ref_build.sh needs the reference sources)")
    lib = C.CDLL(str(LIB))
    sig = {
        "kfr_last_error": (C.c_char_p, []),
        "kfr_pyramid": (C.c_int, [P, C.c_uint32, C.c_uint32, C.POINTER(abi.Intrinsics), C.POINTER(abi.DepthOptions),
                                  P, P, P, C.POINTER(C.c_uint32)]),
        "kfr_pipeline_create": (C.c_int, [C.POINTER(abi.PipelineConfig), C.POINTER(P)]),
        "kfr_pipeline_destroy": (None, [P]),
        "kfr_pipeline_integrate": (C.c_int, [P, P, P, P, C.c_uint32, C.c_uint32, C.POINTER(abi.Intrinsics),
                                             C.POINTER(abi.Rigid)]),
        "kfr_pipeline_raycast": (C.c_int, [P, C.POINTER(abi.Intrinsics), C.c_uint32, C.c_uint32, C.POINTER(abi.Rigid),
                                           P, P, P]),
        "kfr_pipeline_observed": (C.c_uint64, [P]),
        "kfr_pipeline_raw_bytes": (C.c_uint64, [P, C.c_int32]),
        "kfr_pipeline_copy_raw": (C.c_int, [P, C.c_int32, P]),
        "kfr_pipeline_overflowed": (C.c_int32, [P]),
        "kfr_pipeline_mesh": (C.c_int, [P, C.c_float, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
        "kfr_pipeline_mesh_copy": (C.c_int, [P, P, P, P, P]),
        "kfr_icp_equations": (C.c_int, [P, P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, C.c_uint32,
                                        C.POINTER(abi.Intrinsics), C.POINTER(abi.Rigid), C.POINTER(abi.Rigid),
                                        C.c_float, C.c_float, P, C.POINTER(C.c_uint64)]),
        "kfr_icp_estimate": (C.c_int, [P, P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, C.c_uint32,
                                       C.POINTER(abi.Intrinsics), C.POINTER(abi.Rigid), C.POINTER(abi.Rigid),
                                       C.c_uint32, C.POINTER(abi.IcpOptions), C.POINTER(abi.IcpOutcome)]),
        "kfr_track_frame": (C.c_int, [P, P, P, C.c_uint32, C.c_uint32, C.POINTER(abi.Intrinsics),
                                      C.POINTER(abi.DepthOptions), C.POINTER(abi.IcpOptions), P, C.c_int32,
                                      C.POINTER(abi.Rigid), C.POINTER(C.c_int32), P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib = lib
    return lib


def _check(rc: int):
    if rc != 0:
        raise RuntimeError("reference: " + load().kfr_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _rigid(m) -> abi.Rigid:
    return m if isinstance(m, abi.Rigid) else abi.rigid_from_matrix(m)


def pyramid(raw: np.ndarray, k: abi.Intrinsics, o: abi.DepthOptions) -> list[dict]:
    """DepthProcessor<kHost>::build_surface_pyramid (depth_processing.cpp:139-162)."""
    raw = np.ascontiguousarray(raw, dtype=np.uint16)
    h, w = raw.shape
    sizes = [((h >> lv), (w >> lv)) for lv in range(o.levels)]
    total = sum(a * b for a, b in sizes)
    depth = np.zeros(total, np.uint16)
    verts = np.zeros((total, 3), np.float32)
    norms = np.zeros((total, 3), np.float32)
    levels = C.c_uint32()
    _check(load().kfr_pyramid(_ptr(raw), w, h, C.byref(k), C.byref(o), _ptr(depth), _ptr(verts), _ptr(norms),
                              C.byref(levels)))
    out, off = [], 0
    for lv in range(levels.value):
        lh, lw = sizes[lv]
        n = lh * lw
        out.append({"depth": depth[off:off + n].reshape(lh, lw), "vertices": verts[off:off + n].reshape(lh, lw, 3),
                    "normals": norms[off:off + n].reshape(lh, lw, 3)})
        off += n
    return out


class RefPipeline:
    """The reference's host pipeline over one registered representation
    (BasicHostPipeline, pipeline.cpp:23-103) with its raw storage exposed."""

    def __init__(self, config: abi.PipelineConfig):
        self.config = config
        h = C.c_void_p()
        _check(load().kfr_pipeline_create(C.byref(config), C.byref(h)))
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value:
            load().kfr_pipeline_destroy(self.handle)
            self.handle = C.c_void_p()

    def integrate(self, depth, k, world_to_camera, color=None, normals=None):
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        color = None if color is None else np.ascontiguousarray(color, dtype=np.uint32)
        normals = None if normals is None else np.ascontiguousarray(normals, dtype=np.float32)
        w2c = _rigid(world_to_camera)
        _check(load().kfr_pipeline_integrate(self.handle, _ptr(depth), _ptr(color), _ptr(normals), depth.shape[1],
                                             depth.shape[0], C.byref(k), C.byref(w2c)))

    def raycast(self, k, width, height, camera_to_world):
        points = np.zeros((height, width, 3), np.float32)
        normals = np.zeros((height, width, 3), np.float32)
        colors = np.zeros((height, width), np.uint32)
        c2w = _rigid(camera_to_world)
        _check(load().kfr_pipeline_raycast(self.handle, C.byref(k), width, height, C.byref(c2w), _ptr(points),
                                           _ptr(normals), _ptr(colors)))
        return points, normals, colors

    def observed_voxel_count(self) -> int:
        return int(load().kfr_pipeline_observed(self.handle))

    def _raw(self, which: int, dtype) -> np.ndarray:
        n = int(load().kfr_pipeline_raw_bytes(self.handle, which))
        out = np.zeros(n // np.dtype(dtype).itemsize, dtype=dtype)
        if n:
            _check(load().kfr_pipeline_copy_raw(self.handle, which, _ptr(out)))
        return out

    def voxels(self) -> np.ndarray:
        """Raw geometric voxels (dense: x fastest; sparse: the block pool)."""
        if self.config.voxel == abi.KF_VOXEL_FLOAT:
            return self._raw(0, np.float32).reshape(-1, 2)
        return self._raw(0, np.uint32)

    def colors(self) -> np.ndarray:
        return self._raw(1, np.float32).reshape(-1, 4)

    def grid(self) -> np.ndarray:
        """Sparse block grid (block -> pool slot, 0xFFFFFFFF = unallocated)."""
        return self._raw(2, np.uint32)

    def overflowed(self) -> bool:
        return bool(load().kfr_pipeline_overflowed(self.handle))

    def mesh(self, min_weight: float = 0.0) -> dict:
        nv, nt = C.c_uint64(), C.c_uint64()
        _check(load().kfr_pipeline_mesh(self.handle, min_weight, C.byref(nv), C.byref(nt)))
        pos = np.zeros((nv.value, 3), np.float32)
        nor = np.zeros((nv.value, 3), np.float32)
        col = np.zeros((nv.value, 3), np.float32)
        tri = np.zeros((nt.value, 3), np.uint32)
        _check(load().kfr_pipeline_mesh_copy(self.handle, _ptr(pos), _ptr(nor), _ptr(col), _ptr(tri)))
        return {"positions": pos, "normals": nor, "colors": col, "triangles": tri}

    def track_frame(self, depth, k, pose, depth_options, icp_options, iterations=(10, 5, 4), first=False,
                    color=None):
        """One frame of Reconstruction::process_frame; returns (pose 4x4, tracked, level statuses)."""
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        color = None if color is None else np.ascontiguousarray(color, dtype=np.uint32)
        its = np.array(list(iterations) + [4] * (4 - len(iterations)), dtype=np.uint32)
        r = _rigid(pose)
        tracked = C.c_int32()
        status = np.zeros(4, np.int32)
        _check(load().kfr_track_frame(self.handle, _ptr(depth), _ptr(color), depth.shape[1], depth.shape[0],
                                      C.byref(k), C.byref(depth_options), C.byref(icp_options), _ptr(its),
                                      1 if first else 0, C.byref(r), C.byref(tracked), _ptr(status)))
        return abi.matrix_from_rigid(r), bool(tracked.value), status


def icp_equations(live_v, live_n, model_p, model_n, k, camera, model, max_d=0.05, min_dot=0.9659258):
    """HostCorrespondenceSearch::match + IcpNormalEquations::accumulate over the
    live image in pixel order (sums[29], count)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (live_v, live_n, model_p, model_n)]
    lh, lw = arrs[0].shape[:2]
    mh, mw = arrs[2].shape[:2]
    sums = np.zeros(29, np.float32)
    count = C.c_uint64()
    _check(load().kfr_icp_equations(_ptr(arrs[0]), _ptr(arrs[1]), lw, lh, _ptr(arrs[2]), _ptr(arrs[3]), mw, mh,
                                    C.byref(k), C.byref(_rigid(camera)), C.byref(_rigid(model)), max_d, min_dot,
                                    _ptr(sums), C.byref(count)))
    return sums, count.value


def icp_estimate(live_v, live_n, model_p, model_n, k, model_camera_to_world, initial, iterations,
                 options: abi.IcpOptions) -> abi.IcpOutcome:
    """ProjectiveIcpTracker::estimate_pose(TrackingRequest) (icp_optimizer.cpp:46-56)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (live_v, live_n, model_p, model_n)]
    lh, lw = arrs[0].shape[:2]
    mh, mw = arrs[2].shape[:2]
    out = abi.IcpOutcome()
    _check(load().kfr_icp_estimate(_ptr(arrs[0]), _ptr(arrs[1]), lw, lh, _ptr(arrs[2]), _ptr(arrs[3]), mw, mh,
                                   C.byref(k), C.byref(_rigid(model_camera_to_world)), C.byref(_rigid(initial)),
                                   iterations, C.byref(options), C.byref(out)))
    return out


# ---- the reference's CUDA pipeline (libkf_ref_cuda.so) --------------------------------------
LIB_CUDA = HERE / "_ref" / "libkf_ref_cuda.so"
# the reference's host code with its device seams taken by
# kinectfusion_b200/glue/b200_backend.cpp over this project's library
LIB_GLUE = HERE / "_ref" / "libkf_ref_b200.so"
_lib_cuda = {}


def cuda_available(backend: str = "cuda") -> bool:
    return (LIB_CUDA if backend == "cuda" else LIB_GLUE).exists()


def load_cuda(backend: str = "cuda") -> C.CDLL:
    """backend "cuda": the reference built with its own CUDA path
    (src/kinectfusion/cuda/*.cu for sm_100a); "glue": the reference's host
    code over this project's library through the drop-in glue.  Each is
    loaded into its own handle."""
    if backend in _lib_cuda:
        return _lib_cuda[backend]
    path = LIB_CUDA if backend == "cuda" else LIB_GLUE
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built")
    lib = C.CDLL(str(path))
    sig = {
        "kfr_last_error": (C.c_char_p, []),
        "kfr_dev_available": (C.c_int, []),
        "kfr_dev_create": (C.c_int, [C.POINTER(abi.PipelineConfig), C.POINTER(abi.DepthOptions),
                                     C.POINTER(abi.IcpOptions), C.c_int32, C.c_int32, C.POINTER(P)]),
        "kfr_dev_destroy": (None, [P]),
        "kfr_dev_frame": (C.c_int, [P, P, P, C.c_uint32, C.c_uint32, C.POINTER(abi.Intrinsics), P, C.c_int32,
                                    C.POINTER(abi.Rigid), C.POINTER(C.c_int32), P]),
        "kfr_dev_raycast": (C.c_int, [P, C.POINTER(abi.Intrinsics), C.c_uint32, C.c_uint32, C.POINTER(abi.Rigid),
                                      P, P, P]),
        "kfr_dev_host_view": (C.c_int, [P, P]),
        "kfr_dev_observed": (C.c_uint64, [P]),
        "kfr_dev_synchronize": (C.c_int, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib_cuda[backend] = lib
    return lib


class RefDevicePipeline:
    """The reference's --space cuda pipeline (Pipeline::create with
    MemorySpace::kDevice, the device PyramidSource, ProjectiveIcpTracker) run
    frame by frame as Reconstruction::process_frame does.  device_solve and
    capture_graph are its --icp-device-solve / --icp-capture-graph switches."""

    def __init__(self, config: abi.PipelineConfig, depth_options: abi.DepthOptions, icp_options: abi.IcpOptions,
                 device_solve: bool = False, capture_graph: bool = False, iterations=(10, 5, 4),
                 backend: str = "cuda"):
        self.lib = load_cuda(backend)
        h = C.c_void_p()
        self._check(self.lib.kfr_dev_create(C.byref(config), C.byref(depth_options), C.byref(icp_options),
                                            int(device_solve), int(capture_graph), C.byref(h)))
        self.handle = h
        self.config = config
        self.iterations = np.array(list(iterations) + [4] * (4 - len(iterations)), dtype=np.uint32)
        self.pose = abi.rigid_from_matrix(np.eye(4))
        self.frames = 0
        self.trajectory = []

    def _check(self, rc: int):
        if rc != 0:
            raise RuntimeError("reference (device): " + self.lib.kfr_last_error().decode())

    def __del__(self):
        if getattr(self, "handle", None) and self.handle.value:
            self.lib.kfr_dev_destroy(self.handle)
            self.handle = C.c_void_p()

    def process(self, depth, intrinsics, color=None):
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        color = None if color is None else np.ascontiguousarray(color, dtype=np.uint32)
        tracked = C.c_int32()
        status = np.zeros(4, np.int32)
        self._check(self.lib.kfr_dev_frame(self.handle, _ptr(depth), _ptr(color), depth.shape[1], depth.shape[0],
                                              C.byref(intrinsics), _ptr(self.iterations), 1 if self.frames == 0 else 0,
                                              C.byref(self.pose), C.byref(tracked), _ptr(status)))
        self.frames += 1
        self.trajectory.append(abi.matrix_from_rigid(self.pose))
        return bool(tracked.value), status

    def raycast(self, k, width, height, camera_to_world):
        points = np.zeros((height, width, 3), np.float32)
        normals = np.zeros((height, width, 3), np.float32)
        colors = np.zeros((height, width), np.uint32)
        self._check(self.lib.kfr_dev_raycast(self.handle, C.byref(k), width, height,
                                                C.byref(_rigid(camera_to_world)), _ptr(points), _ptr(normals),
                                                _ptr(colors)))
        return points, normals, colors

    def host_view(self) -> np.ndarray:
        g = self.config.volume
        out = np.zeros((g.res_x * g.res_y * g.res_z, 2), np.float32)
        self._check(self.lib.kfr_dev_host_view(self.handle, _ptr(out)))
        return out

    def observed_voxel_count(self) -> int:
        return int(self.lib.kfr_dev_observed(self.handle))

    def synchronize(self):
        self._check(self.lib.kfr_dev_synchronize())
