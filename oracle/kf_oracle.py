"""Python binding of the CPU oracle (oracle/libkf_oracle.so).

TEST INFRASTRUCTURE ONLY: the parity checker of the CUDA path, used by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the product.
"""

from __future__ import annotations

import ctypes as C
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libkf_oracle.so"
sys.path.insert(0, str(HERE.parent))

from kinectfusion_b200 import abi  # noqa: E402  (structures only; the GPU library is not loaded)

_lib = None


class Volume(C.Structure):
    _fields_ = [("geometry", abi.VolumeGeometry), ("voxel", C.c_int32), ("voxels", C.c_void_p),
                ("colors", C.c_void_p), ("grid", C.c_void_p), ("marked_frame", C.c_void_p),
                ("work_list", C.c_void_p), ("capacity", C.c_uint64), ("allocated", C.c_uint64),
                ("work_count", C.c_uint64), ("frame_stamp", C.c_uint32)]


def build() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    P = C.c_void_p
    proto = {
        "kfo_volume_clear": (None, [C.POINTER(Volume)]),
        "kfo_observed_voxel_count": (C.c_uint64, [C.POINTER(Volume)]),
        "kfo_bilateral": (None, [P, C.c_uint32, C.c_uint32, C.POINTER(abi.DepthOptions), P]),
        "kfo_downsample": (None, [P, C.c_uint32, C.c_uint32, C.POINTER(abi.DepthOptions), P]),
        "kfo_vertices": (None, [P, C.c_uint32, C.c_uint32, abi.Intrinsics, C.POINTER(abi.DepthOptions), P]),
        "kfo_normals": (None, [P, C.c_uint32, C.c_uint32, C.POINTER(abi.DepthOptions), P]),
        "kfo_scaled_intrinsics": (abi.Intrinsics, [abi.Intrinsics, C.c_uint32]),
        "kfo_integrate": (None, [C.POINTER(Volume), C.POINTER(abi.FrameView), C.POINTER(abi.IntegrationOptions),
                                 C.c_int32, C.c_int32]),
        "kfo_integrate_band": (None, [C.POINTER(Volume), C.POINTER(abi.FrameView),
                                      C.POINTER(abi.IntegrationOptions), C.c_int32]),
        "kfo_integrate_band_device": (None, [C.POINTER(Volume), C.POINTER(abi.FrameView),
                                             C.POINTER(abi.IntegrationOptions), C.c_int32]),
        "kfo_integrate_f64": (None, [P, C.POINTER(abi.VolumeGeometry), C.POINTER(abi.FrameView),
                                     C.POINTER(abi.IntegrationOptions), C.c_int32, C.c_int32]),
        "kfo_integrate_sparse": (None, [C.POINTER(Volume), C.POINTER(abi.FrameView),
                                        C.POINTER(abi.IntegrationOptions), C.c_int32]),
        "kfo_raycast": (None, [C.POINTER(Volume), C.POINTER(abi.RaycastCamera), C.POINTER(abi.RaycastOptions),
                               P, P, P, C.c_int32]),
        "kfo_band_word_count": (C.c_uint64, [C.POINTER(Volume)]),
        "kfo_band_bitmap": (None, [C.POINTER(Volume), P, P]),
        "kfo_raycast_band": (None, [C.POINTER(Volume), P, C.POINTER(abi.RaycastCamera),
                                    C.POINTER(abi.RaycastOptions), P, P, P, C.c_int32]),
        "kfo_icp_equations": (None, [P, P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, C.c_uint32, abi.Intrinsics,
                                     C.POINTER(abi.Rigid), C.POINTER(abi.Rigid), C.c_float, C.c_float, P,
                                     C.POINTER(C.c_uint64)]),
        "kfo_icp_equations_f64": (None, [P, P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, C.c_uint32,
                                         abi.Intrinsics, C.POINTER(abi.Rigid), C.POINTER(abi.Rigid), C.c_float,
                                         C.c_float, P, C.POINTER(C.c_uint64)]),
        "kfo_icp_estimate": (None, [P, P, C.c_uint32, C.c_uint32, P, P, C.c_uint32, C.c_uint32, abi.Intrinsics,
                                    C.POINTER(abi.Rigid), C.POINTER(abi.Rigid), C.c_uint32,
                                    C.POINTER(abi.IcpOptions), C.POINTER(abi.IcpOutcome)]),
        "kfo_rigid_inverse": (None, [C.POINTER(abi.Rigid), C.POINTER(abi.Rigid)]),
        "kfo_rigid_compose": (None, [C.POINTER(abi.Rigid), C.POINTER(abi.Rigid), C.POINTER(abi.Rigid)]),
        "kfo_marching_cubes": (C.c_int, [C.POINTER(Volume), C.c_float, C.POINTER(abi.Mesh)]),
        "kfo_mesh_free": (None, [C.POINTER(abi.Mesh)]),
        "kfo_mc_case_triangle_counts": (None, [P]),
    }
    for name, (res, args) in proto.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


# ---- option defaults (the reference's default member values) ---------------------
def depth_options(**kw) -> abi.DepthOptions:
    o = abi.DepthOptions(levels=3, depth_scale=5000.0, min_depth=0.4, max_depth=8.0, max_normal_depth_jump=0.1,
                         max_downsample_depth_jump=0.1, bilateral_filter=1, bilateral_radius=2,
                         bilateral_spatial_sigma=2.0, bilateral_depth_sigma=0.08)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def integration_options(**kw) -> abi.IntegrationOptions:
    o = abi.IntegrationOptions(depth_scale=5000.0, observation_weight=1.0, max_weight=196.0, min_depth=0.4,
                               max_depth=8.0, projective_distance=1, distance_scaled_truncation=0,
                               truncation_distance_scale=0.01, mode=abi.KF_INTEGRATION_FULL)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def raycast_options(**kw) -> abi.RaycastOptions:
    o = abi.RaycastOptions(min_depth=0.4, max_depth=8.0, step_scale=1.0, corner_policy=0, cell_gradient_normals=0,
                           seed_from_previous=0)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def icp_options(**kw) -> abi.IcpOptions:
    o = abi.IcpOptions(min_correspondences=64, max_point_distance=0.05, min_normal_dot=0.9659258,
                       min_update_translation=1e-5, min_update_rotation=1e-5, max_update_translation=0.15,
                       max_update_rotation=0.35, min_system_eigenvalue=1e-6, max_condition_number=1e6,
                       damping_mode=0, damping_lambda=1e-3, adaptive_damping=0, lambda_increase=10.0,
                       lambda_decrease=0.1, min_lambda=1e-9, max_lambda=1e6)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def intrinsics(fx, fy, cx, cy) -> abi.Intrinsics:
    return abi.Intrinsics(fx, fy, cx, cy)


def scaled(k: abi.Intrinsics, level: int) -> abi.Intrinsics:
    return load().kfo_scaled_intrinsics(k, level)


# ---- depth processing -------------------------------------------------------------
def bilateral(depth: np.ndarray, o: abi.DepthOptions) -> np.ndarray:
    depth = np.ascontiguousarray(depth, dtype=np.uint16)
    out = np.empty_like(depth)
    load().kfo_bilateral(ptr(depth), depth.shape[1], depth.shape[0], C.byref(o), ptr(out))
    return out


def downsample(depth: np.ndarray, o: abi.DepthOptions) -> np.ndarray:
    depth = np.ascontiguousarray(depth, dtype=np.uint16)
    out = np.empty((depth.shape[0] // 2, depth.shape[1] // 2), dtype=np.uint16)
    load().kfo_downsample(ptr(depth), depth.shape[1], depth.shape[0], C.byref(o), ptr(out))
    return out


def vertices(depth: np.ndarray, k: abi.Intrinsics, o: abi.DepthOptions) -> np.ndarray:
    depth = np.ascontiguousarray(depth, dtype=np.uint16)
    out = np.empty(depth.shape + (3,), dtype=np.float32)
    load().kfo_vertices(ptr(depth), depth.shape[1], depth.shape[0], k, C.byref(o), ptr(out))
    return out


def normals(verts: np.ndarray, o: abi.DepthOptions) -> np.ndarray:
    verts = np.ascontiguousarray(verts, dtype=np.float32)
    out = np.empty_like(verts)
    load().kfo_normals(ptr(verts), verts.shape[1], verts.shape[0], C.byref(o), ptr(out))
    return out


def pyramid(raw: np.ndarray, k: abi.Intrinsics, o: abi.DepthOptions) -> list[dict]:
    """DepthProcessor<kHost>::build_surface_pyramid (depth_processing.cpp:139-162)."""
    levels = []
    current = bilateral(raw, o)
    for level in range(o.levels):
        if current.shape[0] == 0 or current.shape[1] == 0:
            break
        kl = scaled(k, level)
        v = vertices(current, kl, o)
        n = normals(v, o)
        nxt = downsample(current, o) if level + 1 < o.levels else None
        levels.append({"depth": current, "vertices": v, "normals": n, "intrinsics": kl})
        if nxt is None:
            break
        current = nxt
    return levels


# ---- volumes ----------------------------------------------------------------------
class OracleVolume:
    """Dense or sparse volume storage in the oracle's raw layout."""

    def __init__(self, res, voxel_size, origin, truncation, voxel=abi.KF_VOXEL_FLOAT, color=False,
                 sparse=False, capacity=0):
        rx, ry, rz = (res, res, res) if np.isscalar(res) else res
        self.geometry = abi.VolumeGeometry(rx, ry, rz, voxel_size, (C.c_float * 3)(*origin), truncation)
        self.voxel = voxel
        blocks = ((rx + 7) // 8) * ((ry + 7) // 8) * ((rz + 7) // 8)
        self.sparse = sparse
        if sparse:
            self.capacity = capacity if capacity else blocks // 4
            n = self.capacity * 512
            self.grid = np.full(blocks, 0xFFFFFFFF, dtype=np.uint32)
            self.marked = np.zeros(blocks, dtype=np.uint32)
            self.work = np.zeros(max(blocks, 1), dtype=np.uint32)
        else:
            self.capacity = 0
            n = rx * ry * rz
            self.grid = self.marked = self.work = None
        self.count = n
        if voxel == abi.KF_VOXEL_FLOAT:
            self.voxels = np.zeros((n, 2), dtype=np.float32)
        else:
            self.voxels = np.zeros(n, dtype=np.uint32)
        self.colors = np.zeros((n, 4), dtype=np.float32) if color else None
        self.struct = Volume(self.geometry, voxel, ptr(self.voxels), ptr(self.colors), ptr(self.grid),
                             ptr(self.marked), ptr(self.work), self.capacity, 0, 0, 1)
        load().kfo_volume_clear(C.byref(self.struct))

    @property
    def res(self):
        g = self.geometry
        return g.res_x, g.res_y, g.res_z

    def observed_voxel_count(self) -> int:
        return int(load().kfo_observed_voxel_count(C.byref(self.struct)))

    def decoded(self):
        """(tsdf, weight) float arrays in storage order."""
        if self.voxel == abi.KF_VOXEL_FLOAT:
            return self.voxels[:, 0].copy(), self.voxels[:, 1].copy()
        d = (self.voxels & 0xFFFF).astype(np.uint16)
        w = (self.voxels >> 16).astype(np.float32) * np.float32(1.0 / 256.0)
        if self.voxel == abi.KF_VOXEL_QUANTIZED:
            t = d.view(np.int16).astype(np.float32) * np.float32(1.0 / 32767.0)
        else:
            t = (d.astype(np.uint32) << 16).view(np.float32)
        return t, w

    def dense(self):
        """Dense (tsdf, weight) arrays shaped (z, y, x); unallocated = (1, 0)."""
        rx, ry, rz = self.res
        t, w = self.decoded()
        if not self.sparse:
            return t.reshape(rz, ry, rx), w.reshape(rz, ry, rx)
        tsdf = np.ones((rz, ry, rx), dtype=np.float32)
        weight = np.zeros((rz, ry, rx), dtype=np.float32)
        bx, by, bz = (rx + 7) // 8, (ry + 7) // 8, (rz + 7) // 8
        for block in np.nonzero(self.grid != 0xFFFFFFFF)[0]:
            slot = int(self.grid[block])
            x0, y0, z0 = (block % bx) * 8, ((block // bx) % by) * 8, (block // (bx * by)) * 8
            tb = t[slot * 512:(slot + 1) * 512].reshape(8, 8, 8)
            wb = w[slot * 512:(slot + 1) * 512].reshape(8, 8, 8)
            ex, ey, ez = min(8, rx - x0), min(8, ry - y0), min(8, rz - z0)
            tsdf[z0:z0 + ez, y0:y0 + ey, x0:x0 + ex] = tb[:ez, :ey, :ex]
            weight[z0:z0 + ez, y0:y0 + ey, x0:x0 + ex] = wb[:ez, :ey, :ex]
        return tsdf, weight


def frame_view(depth, k, world_to_camera, color=None, normals_map=None) -> tuple[abi.FrameView, list]:
    depth = np.ascontiguousarray(depth, dtype=np.uint16)
    keep = [depth]
    if color is not None:
        color = np.ascontiguousarray(color, dtype=np.uint32)
        keep.append(color)
    if normals_map is not None:
        normals_map = np.ascontiguousarray(normals_map, dtype=np.float32)
        keep.append(normals_map)
    w2c = world_to_camera if isinstance(world_to_camera, abi.Rigid) else abi.rigid_from_matrix(world_to_camera)
    f = abi.FrameView(ptr(depth), ptr(color), ptr(normals_map), depth.shape[1], depth.shape[0], k, w2c,
                      abi.KF_MEMORY_HOST)
    return f, keep


def integrate(vol: OracleVolume, depth, k, world_to_camera, o: abi.IntegrationOptions,
              rule=abi.KF_RULE_ANGLE_WEIGHTED, color=None, normals_map=None, threads=1, band_walk="host"):
    """band_walk: "host" walks the band at voxel steps (BandIntegrationSweep<kHost>),
    "device" at half-block steps (BandIntegrationSweep<kDevice>)."""
    f, keep = frame_view(depth, k, world_to_camera, color, normals_map)
    if vol.sparse:
        load().kfo_integrate_sparse(C.byref(vol.struct), C.byref(f), C.byref(o), rule)
    elif o.mode == abi.KF_INTEGRATION_BAND:
        fn = load().kfo_integrate_band_device if band_walk == "device" else load().kfo_integrate_band
        fn(C.byref(vol.struct), C.byref(f), C.byref(o), rule)
    else:
        load().kfo_integrate(C.byref(vol.struct), C.byref(f), C.byref(o), rule, threads)
    del keep


class OracleVolumeF64:
    """FP64 (tsdf, weight) volume for the error statements of the stored volumes."""

    def __init__(self, res, voxel_size, origin, truncation):
        rx, ry, rz = (res, res, res) if np.isscalar(res) else res
        self.geometry = abi.VolumeGeometry(rx, ry, rz, voxel_size, (C.c_float * 3)(*origin), truncation)
        self.voxels = np.zeros((rx * ry * rz, 2), dtype=np.float64)
        self.voxels[:, 0] = 1.0

    def dense(self):
        g = self.geometry
        shape = (g.res_z, g.res_y, g.res_x)
        return self.voxels[:, 0].reshape(shape), self.voxels[:, 1].reshape(shape)


def integrate_f64(vol: OracleVolumeF64, depth, k, world_to_camera, o: abi.IntegrationOptions,
                  rule=abi.KF_RULE_ANGLE_WEIGHTED, normals_map=None, threads=1):
    f, keep = frame_view(depth, k, world_to_camera, None, normals_map)
    load().kfo_integrate_f64(ptr(vol.voxels), C.byref(vol.geometry), C.byref(f), C.byref(o), rule, threads)
    del keep


def raycast(vol: OracleVolume, k, width, height, camera_to_world, o: abi.RaycastOptions, threads=1,
            seed_points=None):
    cam = abi.RaycastCamera(k, width, height,
                            camera_to_world if isinstance(camera_to_world, abi.Rigid)
                            else abi.rigid_from_matrix(camera_to_world))
    points = np.full((height, width, 3), np.nan, dtype=np.float32) if seed_points is None else \
        np.ascontiguousarray(seed_points, dtype=np.float32).copy()
    nrm = np.empty((height, width, 3), dtype=np.float32)
    colors = np.empty((height, width), dtype=np.uint32)
    load().kfo_raycast(C.byref(vol.struct), C.byref(cam), C.byref(o), ptr(points), ptr(nrm), ptr(colors), threads)
    return points, nrm, colors


def band_bitmap(vol: OracleVolume):
    """(raw, dilated) band words of a dense volume (BandRebuild<kHost>)."""
    n = int(load().kfo_band_word_count(C.byref(vol.struct)))
    raw = np.zeros(n, dtype=np.uint32)
    dilated = np.zeros(n, dtype=np.uint32)
    load().kfo_band_bitmap(C.byref(vol.struct), ptr(raw), ptr(dilated))
    return raw, dilated


def raycast_band(vol: OracleVolume, band_words, k, width, height, camera_to_world, o: abi.RaycastOptions,
                 threads=1, seed_points=None):
    """The band-march raycast (BandSkip over the dilated band words)."""
    cam = abi.RaycastCamera(k, width, height,
                            camera_to_world if isinstance(camera_to_world, abi.Rigid)
                            else abi.rigid_from_matrix(camera_to_world))
    points = np.full((height, width, 3), np.nan, dtype=np.float32) if seed_points is None else \
        np.ascontiguousarray(seed_points, dtype=np.float32).copy()
    nrm = np.empty((height, width, 3), dtype=np.float32)
    colors = np.empty((height, width), dtype=np.uint32)
    words = np.ascontiguousarray(band_words, dtype=np.uint32)
    load().kfo_raycast_band(C.byref(vol.struct), ptr(words), C.byref(cam), C.byref(o), ptr(points), ptr(nrm),
                            ptr(colors), threads)
    return points, nrm, colors


def icp_equations(live_v, live_n, model_p, model_n, k, camera, model, max_d=0.05, min_dot=0.9659258, f64=False):
    lv = np.ascontiguousarray(live_v, dtype=np.float32)
    ln = np.ascontiguousarray(live_n, dtype=np.float32)
    mp = np.ascontiguousarray(model_p, dtype=np.float32)
    mn = np.ascontiguousarray(model_n, dtype=np.float32)
    cam = camera if isinstance(camera, abi.Rigid) else abi.rigid_from_matrix(camera)
    mod = model if isinstance(model, abi.Rigid) else abi.rigid_from_matrix(model)
    count = C.c_uint64()
    if f64:
        sums = np.zeros(29, dtype=np.float64)
        load().kfo_icp_equations_f64(ptr(lv), ptr(ln), lv.shape[1], lv.shape[0], ptr(mp), ptr(mn), mp.shape[1],
                                     mp.shape[0], k, C.byref(cam), C.byref(mod), max_d, min_dot, ptr(sums),
                                     C.byref(count))
    else:
        sums = np.zeros(29, dtype=np.float32)
        load().kfo_icp_equations(ptr(lv), ptr(ln), lv.shape[1], lv.shape[0], ptr(mp), ptr(mn), mp.shape[1],
                                 mp.shape[0], k, C.byref(cam), C.byref(mod), max_d, min_dot, ptr(sums),
                                 C.byref(count))
    return sums, int(count.value)


def icp_estimate(live_v, live_n, model_p, model_n, k, model_camera_to_world, initial, iterations,
                 o: abi.IcpOptions) -> abi.IcpOutcome:
    lv = np.ascontiguousarray(live_v, dtype=np.float32)
    ln = np.ascontiguousarray(live_n, dtype=np.float32)
    mp = np.ascontiguousarray(model_p, dtype=np.float32)
    mn = np.ascontiguousarray(model_n, dtype=np.float32)
    mc = model_camera_to_world if isinstance(model_camera_to_world, abi.Rigid) else \
        abi.rigid_from_matrix(model_camera_to_world)
    ini = initial if isinstance(initial, abi.Rigid) else abi.rigid_from_matrix(initial)
    out = abi.IcpOutcome()
    load().kfo_icp_estimate(ptr(lv), ptr(ln), lv.shape[1], lv.shape[0], ptr(mp), ptr(mn), mp.shape[1], mp.shape[0],
                            k, C.byref(mc), C.byref(ini), iterations, C.byref(o), C.byref(out))
    return out


def rigid_inverse(r: abi.Rigid) -> abi.Rigid:
    out = abi.Rigid()
    load().kfo_rigid_inverse(C.byref(r), C.byref(out))
    return out


def marching_cubes(vol: OracleVolume, min_weight: float = 0.0):
    mesh = abi.Mesh()
    status = load().kfo_marching_cubes(C.byref(vol.struct), min_weight, C.byref(mesh))
    if status != 0:
        raise RuntimeError(f"oracle marching cubes failed with status {status}")
    nv, nt = mesh.vertex_count, mesh.triangle_count
    out = {
        "positions": np.ctypeslib.as_array(mesh.positions, shape=(nv, 3)).copy() if nv else np.zeros((0, 3), np.float32),
        "normals": np.ctypeslib.as_array(mesh.normals, shape=(nv, 3)).copy() if nv else np.zeros((0, 3), np.float32),
        "colors": np.ctypeslib.as_array(mesh.colors, shape=(nv, 3)).copy() if nv else np.zeros((0, 3), np.float32),
        "triangles": np.ctypeslib.as_array(mesh.triangles, shape=(nt, 3)).copy() if nt else np.zeros((0, 3), np.uint32),
    }
    load().kfo_mesh_free(C.byref(mesh))
    return out


def mc_case_triangle_counts() -> np.ndarray:
    counts = np.zeros(256, dtype=np.int32)
    load().kfo_mc_case_triangle_counts(ptr(counts))
    return counts


# ---- the per-frame loop (Reconstruction::process_frame, reconstruction.cpp:184-277) ----
ICP_ITERATIONS = {0: 10, 1: 5, 2: 4}


def track(vol: OracleVolume, levels, raw_shape, pose, ray_opts, icp_opts, threads=1):
    """The tracking half of a frame of the reference loop (track_pose,
    reconstruction.cpp:218-250): levels 2, 1, 0 against renders of `vol` at
    the current estimate; returns (pose, tracked, per-level outcomes)."""
    outcomes = {}
    tracked_pose = pose
    for level in range(len(levels) - 1, -1, -1):
        lv = levels[level]
        h, w = raw_shape[0] >> level, raw_shape[1] >> level
        mp, mn, _ = raycast(vol, lv["intrinsics"], w, h, tracked_pose, ray_opts, threads=threads)
        out = icp_estimate(lv["vertices"], lv["normals"], mp, mn, lv["intrinsics"], tracked_pose, tracked_pose,
                           ICP_ITERATIONS.get(level, 4), icp_opts)
        outcomes[level] = out
        tracked_pose = abi.matrix_from_rigid(out.pose)
        if out.status not in (abi.KF_ICP_MAX_ITERATIONS, abi.KF_ICP_CONVERGED):
            return tracked_pose, False, outcomes
    return tracked_pose, True, outcomes


def track_frame(vol: OracleVolume, raw_depth, k, pose, depth_opts, integ_opts, ray_opts, icp_opts,
                rule=abi.KF_RULE_ANGLE_WEIGHTED, color=None, threads=1, first=False, band_walk="host"):
    """One frame of the reference loop on the oracle; returns (pose, tracked, per-level outcomes)."""
    levels = pyramid(raw_depth, k, depth_opts)
    outcomes = {}
    tracked_pose = pose
    ok = True
    if not first:
        tracked_pose, ok, outcomes = track(vol, levels, raw_depth.shape, pose, ray_opts, icp_opts, threads=threads)
    if ok:
        w2c = rigid_inverse(abi.rigid_from_matrix(tracked_pose))
        integrate(vol, raw_depth, k, w2c, integ_opts, rule, color=color, normals_map=levels[0]["normals"],
                  threads=threads, band_walk=band_walk)
    return tracked_pose, ok, outcomes
