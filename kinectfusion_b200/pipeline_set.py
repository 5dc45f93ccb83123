"""Pipeline sets and their ablation statistics.

PipelineSet mirrors the reference's PipelineSet
(include/kinectfusion/pipeline_set.hpp, src/kinectfusion/pipeline_set.cpp):
several pipelines of one volume geometry fed the same frames, compared
against a reference member.  The comparisons (Comparator::compare,
src/kinectfusion/comparison.cpp:12-81) run on the device through
kf_compare_volumes / kf_compare_surface_maps, so no volume leaves HBM.

SetReconstruction is the app's frame loop over a set
(src/app/reconstruction.cpp:143-334): each member tracks against its own
model and integrates at its own pose, and every `compare_every_n_frames`
frames all members are raycast from the reference member's pose, compared,
and the rows appended to ablation_stats.csv in the format of
FrameOutput::append_ablation_stats (src/app/frame_output.cpp:215-242, fields
of src/app/logging.hpp:85-143).
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import os
import pathlib

import numpy as np

from . import abi
from .pipeline import (ICP_ITERATIONS, Pipeline, ProjectiveIcpTracker, PyramidSource, SurfaceMaps, _check, _ptr,
                       lib)


def format_float(x) -> str:
    """A float as std::format("{}") prints it: the shortest digits that read
    back to the same float, in fixed or scientific notation, whichever is
    shorter (fixed on a tie), scientific exponents signed with two or more
    digits (std::to_chars)."""
    v = np.float32(x)
    if np.isnan(v):
        return "-nan" if np.signbit(v) else "nan"
    if np.isinf(v):
        return "-inf" if v < 0 else "inf"
    if v == 0:
        return "-0" if np.signbit(v) else "0"
    mantissa, exponent = np.format_float_scientific(v, unique=True, trim="-").split("e")
    sign = "-" if mantissa.startswith("-") else ""
    digits = mantissa.lstrip("-").replace(".", "")
    e = int(exponent)
    scientific = (sign + digits[0] + ("." + digits[1:] if len(digits) > 1 else "") + "e" + ("-" if e < 0 else "+")
                  + f"{abs(e):02d}")
    if e >= len(digits) - 1:
        fixed = sign + str(int(abs(float(v))))  # an integer: printed exactly
    elif e >= 0:
        fixed = sign + digits[:e + 1] + "." + digits[e + 1:]
    else:
        fixed = sign + "0." + "0" * (-e - 1) + digits
    return fixed if len(fixed) <= len(scientific) else scientific


@dataclasses.dataclass
class VolumeComparison:
    """VolumeComparison (comparison.hpp:21-28)."""
    compared_voxels: int
    only_primary: int
    only_reference: int
    max_distance_delta: float
    mean_distance_delta: float
    max_weight_delta: float

    def csv(self) -> str:
        return ",".join([str(self.compared_voxels), str(self.only_primary), str(self.only_reference),
                         format_float(self.max_distance_delta), format_float(self.mean_distance_delta),
                         format_float(self.max_weight_delta)])


@dataclasses.dataclass
class SurfaceMapsComparison:
    """SurfaceMapsComparison (comparison.hpp:11-19)."""
    compared_pixels: int
    only_primary: int
    only_reference: int
    max_point_distance: float
    mean_point_distance: float
    max_normal_angle: float
    mean_normal_angle: float

    def csv(self) -> str:
        return ",".join([str(self.compared_pixels), str(self.only_primary), str(self.only_reference),
                         format_float(self.max_point_distance), format_float(self.mean_point_distance),
                         format_float(self.max_normal_angle), format_float(self.mean_normal_angle)])


@dataclasses.dataclass
class PipelineComparison:
    """PipelineComparison (pipeline_set.hpp:24-28)."""
    name: str
    volume: VolumeComparison
    surface: SurfaceMapsComparison | None = None

    def csv(self) -> str:
        """The "{:csv}" form (logging.hpp:122-133): the surface fields are
        left empty when no maps were compared."""
        tail = self.surface.csv() if self.surface is not None else ",,,,,,"
        return f"{self.name},{self.volume.csv()},{tail}"


def _fields(struct) -> dict:
    return {name: getattr(struct, name) for name, _ in struct._fields_}


def compare_volumes(primary: Pipeline, reference: Pipeline) -> VolumeComparison:
    """Comparator::compare of two pipelines' volumes, on the device."""
    out = abi.VolumeComparison()
    _check(lib().kf_compare_volumes(primary.handle, reference.handle, C.byref(out)))
    return VolumeComparison(**_fields(out))


class DeviceSurfaceMaps:
    """SurfaceMaps held in device memory (torch tensors on the current CUDA
    device): points / normals HxWx3 float32, colors HxW RGBA8."""

    def __init__(self, width: int, height: int):
        import torch
        self.width, self.height = width, height
        self.points = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
        self.normals = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
        self.colors = torch.empty((height, width), dtype=torch.int32, device="cuda")

    def view(self) -> abi.SurfaceMapsView:
        return abi.SurfaceMapsView(self.points.data_ptr(), self.normals.data_ptr(), self.colors.data_ptr(),
                                   self.width, self.height, abi.KF_MEMORY_DEVICE)

    def to_host(self) -> SurfaceMaps:
        return SurfaceMaps(self.points.cpu().numpy(), self.normals.cpu().numpy(),
                           self.colors.cpu().numpy().view(np.uint32))


def _maps_view(maps) -> abi.SurfaceMapsView:
    if isinstance(maps, DeviceSurfaceMaps):
        return maps.view()
    points = np.ascontiguousarray(maps.points, dtype=np.float32)
    normals = np.ascontiguousarray(maps.normals, dtype=np.float32)
    h, w = points.shape[:2]
    view = abi.SurfaceMapsView(_ptr(points), _ptr(normals), None, w, h, abi.KF_MEMORY_HOST)
    view._keep = (points, normals)
    return view


def compare_surface_maps(primary, reference) -> SurfaceMapsComparison:
    """Comparator::compare of two sets of surface maps (host SurfaceMaps or
    DeviceSurfaceMaps), on the device."""
    pv, rv = _maps_view(primary), _maps_view(reference)
    out = abi.SurfaceMapsComparison()
    _check(lib().kf_compare_surface_maps(C.byref(pv), C.byref(rv), C.byref(out)))
    return SurfaceMapsComparison(**_fields(out))


@dataclasses.dataclass
class PipelineOutput:
    """PipelineOutput (pipeline_set.hpp:30-33)."""
    name: str
    maps: object  # SurfaceMaps or DeviceSurfaceMaps


def _same_geometry(a: abi.PipelineConfig, b: abi.PipelineConfig) -> bool:
    ga, gb = a.volume, b.volume
    return ((ga.res_x, ga.res_y, ga.res_z, ga.voxel_size, tuple(ga.origin), ga.truncation_distance)
            == (gb.res_x, gb.res_y, gb.res_z, gb.voxel_size, tuple(gb.origin), gb.truncation_distance))


class PipelineSet:
    """PipelineSet (pipeline_set.hpp:35-129) over device pipelines."""

    def __init__(self, pipelines: list[Pipeline], reference: str = "", compare_every_n_frames: int = 1):
        # PipelineSet::create (pipeline_set.cpp:33-79)
        if not pipelines:
            raise ValueError("Pipeline set requires at least one pipeline")
        names = [p.name for p in pipelines]
        if len(set(names)) != len(names):
            raise ValueError("Pipeline set requires unique pipeline names")
        if any(not _same_geometry(p.config, pipelines[0].config) for p in pipelines):
            raise ValueError("Pipeline set requires matching volume geometries")
        self.reference_index = 0
        if reference:
            if reference not in names:
                raise ValueError("Pipeline set reference must name a configured pipeline")
            self.reference_index = names.index(reference)
        self.members = list(pipelines)
        # the members' frames run side by side on their own streams
        if len(self.members) > 1:
            for member in self.members:
                member.set_concurrent(True)
        self.compare_every_n_frames = compare_every_n_frames
        self._maps: dict[tuple[int, int, int], DeviceSurfaceMaps] = {}

    def size(self) -> int:
        return len(self.members)

    @property
    def reference(self) -> Pipeline:
        return self.members[self.reference_index]

    def should_compare(self, frame_index: int) -> bool:
        return (len(self.members) > 1 and self.compare_every_n_frames > 0
                and frame_index % self.compare_every_n_frames == 0)

    def integrate(self, depth, intrinsics, world_to_camera, color=None, normals=None) -> None:
        for member in self.members:
            member.integrate(depth, intrinsics, world_to_camera, color, normals)

    def integrate_member(self, index: int, depth, intrinsics, world_to_camera, color=None, normals=None) -> None:
        self.members[index].integrate(depth, intrinsics, world_to_camera, color, normals)

    def raycast_member(self, index: int, intrinsics, width, height, camera_to_world) -> SurfaceMaps:
        return self.members[index].raycast(intrinsics, width, height, camera_to_world)

    def raycast_reference(self, intrinsics, width, height, camera_to_world) -> SurfaceMaps:
        return self.reference.raycast(intrinsics, width, height, camera_to_world)

    def raycast_all(self, intrinsics, width, height, camera_to_world, device: bool = True) -> list[PipelineOutput]:
        """Every member rendered from one camera, in member order.  With
        device=True the maps stay in HBM (reused per member and extent) for
        compare(); to_host() reads one back."""
        if not device:
            return [PipelineOutput(m.name, m.raycast(intrinsics, width, height, camera_to_world))
                    for m in self.members]
        c2w = camera_to_world if isinstance(camera_to_world, abi.Rigid) else abi.rigid_from_matrix(camera_to_world)
        cam = abi.RaycastCamera(intrinsics, width, height, c2w)
        outputs = []
        for i, member in enumerate(self.members):
            maps = self._maps.get((i, width, height))
            if maps is None:
                maps = self._maps[(i, width, height)] = DeviceSurfaceMaps(width, height)
            if member.config.raycast.seed_from_previous:
                maps.points.fill_(float("nan"))
            view = maps.view()
            _check(lib().kf_pipeline_raycast(member.handle, C.byref(cam), C.byref(view)))
            outputs.append(PipelineOutput(member.name, maps))
        return outputs

    def compare(self, outputs: list[PipelineOutput] | None = None) -> list[PipelineComparison]:
        """PipelineSet::compare (pipeline_set.cpp:136-181): every member but
        the reference against the reference; surfaces too when `outputs`
        (from raycast_all) are given."""
        if outputs is not None and len(outputs) != len(self.members):
            raise ValueError("Pipeline comparison requires one raycast output per pipeline")
        comparisons = []
        for i, member in enumerate(self.members):
            if i == self.reference_index:
                continue
            volume = compare_volumes(member, self.reference)
            surface = None
            if outputs is not None:
                surface = compare_surface_maps(outputs[i].maps, outputs[self.reference_index].maps)
            comparisons.append(PipelineComparison(member.name, volume, surface))
        return comparisons


ABLATION_STATS_HEADER = ("frame,pipeline,compared_voxels,volume_only_pipeline,volume_only_reference,"
                         "max_distance_delta,mean_distance_delta,max_weight_delta,compared_pixels,"
                         "surface_only_pipeline,surface_only_reference,max_point_distance,mean_point_distance,"
                         "max_normal_angle,mean_normal_angle\n")


class AblationStats:
    """FrameOutput::append_ablation_stats (frame_output.cpp:215-242): the
    first call truncates output_dir/ablation_stats.csv and writes the
    header; every call appends one row per comparison."""

    def __init__(self, output_dir):
        self.path = pathlib.Path(output_dir) / "ablation_stats.csv"
        self.started = False

    def append(self, frame_index: int, comparisons: list[PipelineComparison]) -> None:
        if not comparisons:
            return
        os.makedirs(self.path.parent, exist_ok=True)
        try:
            with open(self.path, "w" if not self.started else "a") as out:
                if not self.started:
                    out.write(ABLATION_STATS_HEADER)
                self.started = True
                for comparison in comparisons:
                    out.write(f"{frame_index},{comparison.csv()}\n")
        except OSError as error:
            raise RuntimeError(f"Failed to open ablation stats output: {self.path}") from error


class SetReconstruction:
    """The app's loop over a pipeline set (reconstruction.cpp:143-334).

    Per frame the depth (and colour) is uploaded once to HBM and every member
    runs its own whole-frame graph from it (kf_frame_enqueue on the member's
    stream, so members overlap on the GPU): a pyramid, tracking against the
    member's own model and, when tracking holds, integration at the member's
    own pose; a rejected member keeps its last good pose.  On comparison
    frames every member is raycast from the reference member's pose at full
    resolution and compared with the reference on the device; the rows go to
    `comparisons` and, with an output directory, to ablation_stats.csv."""

    def __init__(self, pipeline_set: PipelineSet, intrinsics: abi.Intrinsics, output_dir=None, depth_options=None,
                 icp_options=None, iterations=ICP_ITERATIONS, frame_output=None):
        self.set = pipeline_set
        self.frame_output = frame_output  # tum.FrameOutput: per-frame raycast images / point clouds
        self.intrinsics = intrinsics
        self.pyramids = [PyramidSource(depth_options) for _ in pipeline_set.members]
        self.trackers = [ProjectiveIcpTracker(icp_options) for _ in pipeline_set.members]
        self.iterations = (C.c_uint32 * 4)(*iterations)
        self.stats = AblationStats(output_dir) if output_dir is not None else None
        self.frames = 0
        self.trajectories: list[list[np.ndarray]] = [[] for _ in pipeline_set.members]
        self.results: list[list[abi.FrameResult]] = [[] for _ in pipeline_set.members]
        self.comparisons: list[tuple[int, list[PipelineComparison]]] = []
        self._upload = None

    def _stage(self, depth, color):
        import torch
        h, w = depth.shape
        if self._upload is None or self._upload[0].shape != (h, w):
            self._upload = (torch.empty((h, w), dtype=torch.int16, device="cuda"),
                            torch.empty((h, w), dtype=torch.int32, device="cuda"))
        d, c = self._upload
        d.copy_(torch.from_numpy(np.ascontiguousarray(depth, dtype=np.uint16).view(np.int16)))
        if color is not None:
            c.copy_(torch.from_numpy(np.ascontiguousarray(color, dtype=np.uint32).view(np.int32)))
        torch.cuda.current_stream().synchronize()  # the members' streams read the upload next
        return C.c_void_p(d.data_ptr()), (C.c_void_p(c.data_ptr()) if color is not None else None)

    def process(self, depth, color=None) -> list[abi.FrameResult]:
        depth = np.asarray(depth)
        h, w = depth.shape
        d_ptr, c_ptr = self._stage(depth, color)
        first = 1 if self.frames == 0 else 0
        for i, member in enumerate(self.set.members):
            _check(lib().kf_frame_enqueue(member.handle, self.pyramids[i].handle, self.trackers[i].handle, d_ptr,
                                          c_ptr, w, h, self.intrinsics, abi.KF_MEMORY_DEVICE, self.iterations,
                                          first))
        results = []
        for i, member in enumerate(self.set.members):
            r = abi.FrameResult()
            _check(lib().kf_frame_result_fetch(member.handle, C.byref(r)))
            results.append(r)
            self.results[i].append(r)
            self.trajectories[i].append(abi.matrix_from_rigid(r.camera_to_world))
        frame_index = self.frames
        self.frames += 1
        # render_model_outputs (reconstruction.cpp:303-334): one viewpoint,
        # the reference member's pose
        writes = self.frame_output is not None and self.frame_output.writes_frames()
        pose = results[self.set.reference_index].camera_to_world
        if self.set.should_compare(frame_index):
            outputs = self.set.raycast_all(self.intrinsics, w, h, pose)
            comparisons = self.set.compare(outputs)
            self.comparisons.append((frame_index, comparisons))
            if self.stats is not None:
                self.stats.append(frame_index, comparisons)
            if writes:
                for i, output in enumerate(outputs):
                    subdirectory = "" if i == self.set.reference_index else output.name
                    self.frame_output.write_frame(output.maps, frame_index, subdirectory)
        elif writes:
            self.frame_output.write_frame(self.set.raycast_reference(self.intrinsics, w, h, pose), frame_index)
        return results
