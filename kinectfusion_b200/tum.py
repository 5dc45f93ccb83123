"""Real-data frames and output files: TUM RGB-D sequences and PLY / PNG /
trajectory writers.

TumSequence mirrors the reference's VirtualSensor
(src/kinectfusion/virtual_sensor.cpp:41-147): `depth.txt` and `rgb.txt`
list "timestamp relative_path" after three header lines, depth and colour
frames pair by index, the depth intrinsics follow the camera family named in
the dataset directory (freiburg2 / freiburg3, else freiburg1), and frames are
decoded a few ahead on worker threads (or all up front with preload).  The
PNG decoding and the PLY writing run in libkf_b200.so (kf_png_*, kf_*_ply);
the ctypes calls release the interpreter lock, so the prefetch threads decode
in parallel.
"""

from __future__ import annotations

import concurrent.futures
import ctypes as C
import dataclasses
import math
import os
import pathlib

import numpy as np

from . import abi
from .pipeline import _check, lib

# Calibrated depth intrinsics of the TUM RGB-D camera families (fx, fy, cx, cy),
# as the reference selects them (virtual_sensor.cpp:18-37).
TUM_DEPTH_INTRINSICS = {
    "freiburg1": (517.3, 516.5, 318.6, 255.3),
    "freiburg2": (520.9, 521.0, 325.1, 249.7),
    "freiburg3": (535.4, 539.2, 320.1, 247.6),
}
PREFETCH_DEPTH = 4


def tum_depth_intrinsics(dataset_dir) -> abi.Intrinsics:
    name = str(dataset_dir)
    for family in ("freiburg2", "freiburg3"):
        if family in name:
            return abi.Intrinsics(*TUM_DEPTH_INTRINSICS[family])
    return abi.Intrinsics(*TUM_DEPTH_INTRINSICS["freiburg1"])


def read_index(path) -> tuple[list[float], list[str]]:
    """VirtualSensor::read_index (virtual_sensor.cpp:171-191): skip three
    header lines, then read "timestamp path" pairs."""
    with open(path) as f:
        lines = f.read().split("\n")
    tokens = " ".join(lines[3:]).split()
    stamps, files = [], []
    for i in range(0, len(tokens) - 1, 2):
        try:
            stamps.append(float(tokens[i]))
        except ValueError:
            break
        files.append(tokens[i + 1])
    return stamps, files


def _bytes(path) -> bytes:
    return os.fsencode(os.fspath(path))


def png_info(path) -> tuple[int, int, int, int]:
    """(width, height, colour type, bit depth) of a PNG file."""
    w, h, ct, bd = C.c_uint32(), C.c_uint32(), C.c_int32(), C.c_int32()
    _check(lib().kf_png_info(_bytes(path), C.byref(w), C.byref(h), C.byref(ct), C.byref(bd)))
    return w.value, h.value, ct.value, bd.value


def read_depth_png(path) -> np.ndarray:
    """A 16-bit grayscale depth PNG as uint16 HxW (raw sensor units)."""
    w, h, _, _ = png_info(path)
    out = np.empty((h, w), dtype=np.uint16)
    _check(lib().kf_png_read_depth(_bytes(path), out.ctypes.data_as(C.c_void_p), w, h))
    return out


def read_color_png(path) -> np.ndarray:
    """A colour PNG as uint32 HxW RGBA8 (R | G << 8 | B << 16 | A << 24)."""
    w, h, _, _ = png_info(path)
    out = np.empty((h, w), dtype=np.uint32)
    _check(lib().kf_png_read_color(_bytes(path), out.ctypes.data_as(C.c_void_p), w, h))
    return out


def write_depth_png(path, depth) -> None:
    d = np.ascontiguousarray(depth, dtype=np.uint16)
    _check(lib().kf_png_write_depth(_bytes(path), d.ctypes.data_as(C.c_void_p), d.shape[1], d.shape[0]))


def write_color_png(path, rgba) -> None:
    c = np.ascontiguousarray(rgba, dtype=np.uint32)
    _check(lib().kf_png_write_color(_bytes(path), c.ctypes.data_as(C.c_void_p), c.shape[1], c.shape[0]))


@dataclasses.dataclass
class Frame:
    index: int
    timestamp: float
    depth: np.ndarray  # uint16 HxW
    color: np.ndarray  # uint32 HxW RGBA8


class TumSequence:
    """The frames of one TUM RGB-D dataset directory, in order."""

    def __init__(self, dataset_dir, preload: bool = False, prefetch: int = PREFETCH_DEPTH):
        self.dir = pathlib.Path(dataset_dir)
        self.depth_timestamps, self.depth_files = read_index(self.dir / "depth.txt")
        _, self.color_files = read_index(self.dir / "rgb.txt")
        if not self.depth_files or not self.color_files:
            raise ValueError(f"no frames listed in {self.dir}")
        self.intrinsics = tum_depth_intrinsics(self.dir)
        self.prefetch = max(1, prefetch)
        self._preloaded = None
        if preload:
            with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as pool:
                self._preloaded = list(pool.map(self._decode, range(len(self))))

    def __len__(self) -> int:
        return min(len(self.depth_files), len(self.color_files))

    def _decode(self, index: int) -> Frame:
        return Frame(index, self.depth_timestamps[index], read_depth_png(self.dir / self.depth_files[index]),
                     read_color_png(self.dir / self.color_files[index]))

    def __iter__(self):
        if self._preloaded is not None:
            yield from self._preloaded
            return
        with concurrent.futures.ThreadPoolExecutor(max_workers=self.prefetch) as pool:
            pending = [pool.submit(self._decode, i) for i in range(min(self.prefetch, len(self)))]
            following = len(pending)
            while pending:
                frame = pending.pop(0).result()
                if following < len(self):
                    pending.append(pool.submit(self._decode, following))
                    following += 1
                yield frame


def write_sequence(dataset_dir, depth_frames, color_frames, fps: float = 30.0) -> None:
    """Stores frames as a TUM RGB-D directory (depth/, rgb/, the two index
    files), e.g. to replay synthetic frames through TumSequence."""
    root = pathlib.Path(dataset_dir)
    (root / "depth").mkdir(parents=True, exist_ok=True)
    (root / "rgb").mkdir(parents=True, exist_ok=True)
    header = "# {} maps\n# file: 'sequence'\n# timestamp filename\n"
    with open(root / "depth.txt", "w") as fd, open(root / "rgb.txt", "w") as fc:
        fd.write(header.format("depth"))
        fc.write(header.format("color"))
        for i, (d, c) in enumerate(zip(depth_frames, color_frames)):
            stamp = f"{i / fps:.6f}"
            write_depth_png(root / "depth" / f"{stamp}.png", d)
            write_color_png(root / "rgb" / f"{stamp}.png", c)
            fd.write(f"{stamp} depth/{stamp}.png\n")
            fc.write(f"{stamp} rgb/{stamp}.png\n")


def write_mesh_ply(path, mesh: dict) -> None:
    """A mesh from Pipeline.extract_mesh as FrameOutput::write_mesh stores it."""
    pos = np.ascontiguousarray(mesh["positions"], dtype=np.float32)
    nrm = np.ascontiguousarray(mesh["normals"], dtype=np.float32)
    col = np.ascontiguousarray(mesh["colors"], dtype=np.float32)
    tri = np.ascontiguousarray(mesh["triangles"], dtype=np.uint32)
    m = abi.Mesh(pos.ctypes.data_as(C.POINTER(C.c_float)), nrm.ctypes.data_as(C.POINTER(C.c_float)),
                 col.ctypes.data_as(C.POINTER(C.c_float)), tri.ctypes.data_as(C.POINTER(C.c_uint32)),
                 len(pos), len(tri))
    _check(lib().kf_mesh_write_ply(_bytes(path), C.byref(m)))


def write_point_cloud_ply(path, points, normals, colors) -> None:
    """Raycast maps (HxWx3 points and normals, HxW RGBA8) as
    FrameOutput::write_raycast_point_cloud stores them."""
    p = np.ascontiguousarray(points, dtype=np.float32)
    n = np.ascontiguousarray(normals, dtype=np.float32)
    c = np.ascontiguousarray(colors, dtype=np.uint32)
    h, w = c.shape
    _check(lib().kf_maps_write_ply(_bytes(path), p.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p),
                                   c.ctypes.data_as(C.c_void_p), w, h))


def write_trajectory(path, poses, timestamps) -> None:
    """Camera poses in the TUM trajectory format "timestamp tx ty tz qx qy qz
    qw" (Reconstruction's trajectory output, reconstruction.cpp:362-391)."""
    with open(path, "w") as f:
        for stamp, pose in zip(timestamps, poses):
            m = np.asarray(pose, dtype=np.float64)
            q = _quaternion(m[:3, :3])
            t = m[:3, 3]
            f.write(f"{stamp:.9f} {t[0]:.9f} {t[1]:.9f} {t[2]:.9f} {q[0]:.9f} {q[1]:.9f} {q[2]:.9f} {q[3]:.9f}\n")


def _quaternion(r: np.ndarray):
    tr = np.trace(r)
    if tr > 0:
        s = math.sqrt(tr + 1.0) * 2
        return ((r[2, 1] - r[1, 2]) / s, (r[0, 2] - r[2, 0]) / s, (r[1, 0] - r[0, 1]) / s, 0.25 * s)
    i = int(np.argmax(np.diag(r)))
    j, k = (i + 1) % 3, (i + 2) % 3
    s = math.sqrt(1.0 + r[i, i] - r[j, j] - r[k, k]) * 2
    q = [0.0, 0.0, 0.0, 0.0]
    q[i] = 0.25 * s
    q[j] = (r[j, i] + r[i, j]) / s
    q[k] = (r[k, i] + r[i, k]) / s
    q[3] = (r[k, j] - r[j, k]) / s
    return tuple(q)


class FrameOutput:
    """FrameOutput (src/app/frame_output.cpp:34-213): per-frame raycast
    outputs written by worker threads, at most MAX_PENDING_WRITES in flight
    (the oldest is waited for first), and mesh.ply.  Frames go to
    `output_dir`, or `output_dir/subdirectory` for a pipeline-set member
    other than the reference.  write_frame takes host maps (SurfaceMaps, or
    anything with to_host(), such as pipeline_set.DeviceSurfaceMaps)."""

    MAX_PENDING_WRITES = 16

    def __init__(self, output_dir, write_raycast_images: bool = False, write_point_clouds: bool = False):
        self.output_dir = pathlib.Path(output_dir)
        self.write_raycast_images = write_raycast_images
        self.write_point_clouds = write_point_clouds
        self._pool = concurrent.futures.ThreadPoolExecutor(max_workers=4)
        self._pending: list[concurrent.futures.Future] = []

    def writes_frames(self) -> bool:
        return self.write_raycast_images or self.write_point_clouds

    @staticmethod
    def frame_prefix(frame_index: int) -> str:
        return f"frame_{frame_index:06d}"

    def write_frame(self, maps, frame_index: int, subdirectory: str = "") -> None:
        if not self.writes_frames():
            return
        if hasattr(maps, "to_host"):
            maps = maps.to_host()
        while len(self._pending) >= self.MAX_PENDING_WRITES:
            self._pending.pop(0).result()
        directory = self.output_dir / subdirectory if subdirectory else self.output_dir
        directory.mkdir(parents=True, exist_ok=True)
        prefix = directory / self.frame_prefix(frame_index)
        if self.write_raycast_images:
            self._pending.append(self._pool.submit(write_color_png, f"{prefix}_raycast.png", maps.colors))
        if self.write_point_clouds:
            self._pending.append(self._pool.submit(write_point_cloud_ply, f"{prefix}_raycast_point_cloud.ply",
                                                   maps.points, maps.normals, maps.colors))

    def write_mesh(self, mesh: dict, subdirectory: str = "") -> None:
        directory = self.output_dir / subdirectory if subdirectory else self.output_dir
        directory.mkdir(parents=True, exist_ok=True)
        write_mesh_ply(directory / "mesh.ply", mesh)

    def finish_pending_writes(self) -> None:
        pending, self._pending = self._pending, []
        for future in pending:
            future.result()

    def close(self) -> None:
        try:
            self.finish_pending_writes()
        finally:
            self._pool.shutdown(wait=True)
