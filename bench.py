"""Benchmark of the per-frame pipeline: frames/s at 640x480 into a 512^3 volume.

One step = one frame of the reference's per-frame loop (Reconstruction::
process_frame, src/app/reconstruction.cpp:184-216): bilateral + 3-level
pyramid, per level a model raycast at the current pose estimate and the
ICP iterations [10, 5, 4], then TSDF integration at the tracked pose.

Workload: the 640x480 synthetic scene (seeded box room + spheres + boxes,
kinectfusion_b200/synthetic.py) through a dense 512^3 float volume at 1 cm
(8 B/voxel, 1 GiB, colour off), angle-weighted TSDF, truncation 5 cm.
The timed steps are first passes through fresh 30-frame seeded sequences:
step s is frame s mod 30 of pass s div 30, every pass starts from an emptied
volume (the refill is queued on the stream inside the timed region) and
fuses its first frame without tracking, as a new reconstruction does.  The
1 GiB volume is larger than L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

The default 120 steps are four passes over four seeds.

Multi-GPU: replicas only (each rank tracks its own seeded sequence; the
path has no exchange step).  Timing is CUDA events on the pipeline's stream,
barrier + synchronize on both sides, max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "frames/s (640x480, 512^3) and ICP iters/frame, learned vs plain at equal ATE"
RES, VOXEL, TRUNC = 512, 0.01, 0.05
ORIGIN = (-0.5 * RES * VOXEL, -0.5 * RES * VOXEL, -0.5)
SEQ_FRAMES = 30


def frame_schedule(step: int) -> int:
    """Triangle wave over the sequence: 0..29, 28..1, 0..29, ... (the
    ablation and comparison runs, which replay one sequence)."""
    period = 2 * (SEQ_FRAMES - 1)
    s = step % period
    return s if s < SEQ_FRAMES else period - s


def workload_config() -> dict:
    return {"workload": "640x480 synthetic RGB-D frames tracked and fused into a dense 512^3 float volume "
                        "(0.01 m voxels, 8 B/voxel, colour off), angle-weighted TSDF, ICP [10,5,4]",
            "frame": [640, 480], "volume": [RES, RES, RES], "voxel_size_m": VOXEL, "truncation_m": TRUNC,
            "voxel_bytes": 8, "sequence_frames": SEQ_FRAMES,
            "l2": "inputs larger than L2 (1 GiB volume re-read every step), no flush"}


# ---- clocks ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons sampled DURING the timed region.

    NVML (read-only queries) every 2 ms when it is available, so that a timed
    region of a few tens of milliseconds still gets samples; otherwise
    nvidia-smi at its 100 ms floor.  Nothing here changes a GPU setting."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int, period_s: float = 0.002):
        self.index = index
        self.period_s = period_s
        self.proc = None
        self.nvml = None
        self.lines: list[str] = []
        self.samples: list[tuple[float, float | None, int]] = []
        self.skip = 0
        self._stop = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.index)
        uuid = str(getattr(props, "uuid", "") or "")
        if uuid:
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except pynvml.NVMLError:
                pass
        bus = "%08x:%02x:%02x.0" % (getattr(props, "pci_domain_id", 0), getattr(props, "pci_bus_id", 0),
                                    getattr(props, "pci_device_id", 0))
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except pynvml.NVMLError:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def __enter__(self):
        try:
            nv, handle = self._nvml_handle()
            self.nvml = (nv, handle)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(handle, nv.NVML_CLOCK_SM))
            self.masks = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                          nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:  # no NVML binding or no device handle: nvidia-smi
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _poll(self):
        nv, handle = self.nvml
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(handle, nv.NVML_CLOCK_SM))
                reasons = int(nv.nvmlDeviceGetCurrentClocksEventReasons(handle))
                self.samples.append((time.perf_counter(), sm, reasons))
            except Exception:
                pass
            self._stop.wait(self.period_s)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_started(self, timeout: float = 5.0):
        # nvidia-smi needs a moment before its first sample; the timed region
        # starts once it reports
        t0 = time.time()
        if self.nvml is not None:
            while not self.samples and time.time() - t0 < timeout:
                time.sleep(0.001)
            self.skip = len(self.samples)
            return
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)
        self.skip = len(self.lines)

    def __exit__(self, *exc):
        self._stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=2)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        if self.nvml is not None:
            for _, mhz, bits in self.samples[self.skip:]:
                sm.append(mhz)
                for name, mask in zip(self.NAMES, self.masks):
                    if bits & mask:
                        reasons.add(name)
            mx = self.max_mhz
            source = f"nvml every {self.period_s * 1e3:g} ms"
        else:
            for line in self.lines[self.skip:]:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for name, flag in zip(self.NAMES, parts[5:9]):
                    if flag.lower().startswith("active"):
                        reasons.add(name)
            source = "nvidia-smi every 100 ms"
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": source}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"hbm_gbs": 6650.0, "fallback": True}


def profile_traffic() -> float | None:
    """DRAM bytes per integrate launch from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "integrate_dense512_cfg2.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---- ranks ------------------------------------------------------------------------------
def max_over_ranks(times_ms: list[float], dist, device: str) -> list[float]:
    """Each timing as the slowest rank's (every rank runs its own replica over
    the same timed region, between barriers)."""
    import torch
    t = torch.tensor(times_ms, dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_throughput(steps: int, world: int, elapsed_ms: float) -> float:
    """Whole-job frames/s: every rank processed `steps` frames of its own
    sequence in at most `elapsed_ms`."""
    return steps * world / (elapsed_ms / 1e3)


# ---- our arm ------------------------------------------------------------------------------
def pass_of(step: int) -> tuple[int, int]:
    """(pass, frame) of a timed step: the steps play fresh 30-frame sequences
    one after another, each from an emptied volume."""
    return divmod(step, SEQ_FRAMES)


def percentiles(values: list[float]) -> dict:
    a = np.asarray(values, dtype=np.float64)
    return {"mean": round(float(a.mean()), 4), "p50": round(float(np.percentile(a, 50)), 4),
            "p90": round(float(np.percentile(a, 90)), 4), "p99": round(float(np.percentile(a, 99)), 4),
            "max": round(float(a.max()), 4), "min": round(float(a.min()), 4)}


def run_ours(args, rank: int, world: int, dist) -> dict | None:
    import torch

    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    lib = abi.load()
    # the timed steps are consecutive first passes through fresh sequences
    # (at most four distinct seeds, cycled); every pass starts from an empty
    # volume, as a new reconstruction does
    passes = (args.steps + SEQ_FRAMES - 1) // SEQ_FRAMES
    n_seq = max(1, min(passes, 4))
    seqs = [synthetic.make_sequence(seed=1000 + 100 * rank, frames=SEQ_FRAMES)]
    for i in range(1, n_seq):
        seqs.append(synthetic.make_sequence_device(seed=1000 + 100 * rank + i, frames=SEQ_FRAMES))
    seq = seqs[0]
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED)
    pipe = kf.Pipeline(cfg)
    pyr = kf.PyramidSource()
    tracker = kf.ProjectiveIcpTracker()
    iters = (C.c_uint32 * 4)(10, 5, 4, 4)
    stream_ptr = C.c_void_p()
    abi.check(lib.kf_pipeline_stream(pipe.handle, C.byref(stream_ptr)))
    stream = torch.cuda.ExternalStream(stream_ptr.value)
    depth_dev = [torch.from_numpy(q.depth.view(np.int16)).cuda() for q in seqs]
    frame_bytes = 640 * 480 * 2
    identity = abi.rigid_from_matrix(np.eye(4))
    kcount = C.c_uint32()

    def enqueue(step: int) -> int:
        """Queue timed step `step`; returns the kernels it launched."""
        p, f = pass_of(step)
        launched = 0
        if f == 0:
            abi.check(lib.kf_pipeline_reset_async(pipe.handle))  # fill kernel + memsets
            abi.check(lib.kf_frame_set_pose(pipe.handle, tracker.handle, C.byref(identity)))
            launched += 2
        base = depth_dev[p % n_seq].data_ptr()
        abi.check(lib.kf_frame_enqueue(pipe.handle, pyr.handle, tracker.handle, C.c_void_p(base + f * frame_bytes),
                                       None, 640, 480, k, abi.KF_MEMORY_DEVICE, iters, 1 if f == 0 else 0))
        abi.check(lib.kf_frame_kernel_count(pipe.handle, C.byref(kcount)))
        return launched + int(kcount.value)

    def barrier():
        if dist is not None:
            dist.barrier()

    # warm-up: W frames of the first sequence (captures the first-frame and
    # tracking graphs), then the timed region starts from an empty volume
    for s in range(max(args.warmup, 3)):
        enqueue(s)
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs ------------------------------------
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_events = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    barrier()
    torch.cuda.synchronize()
    launches = 0
    with ClockSampler(torch.cuda.current_device()) as clocks:
        clocks.wait_started()
        start.record(stream)
        for s in range(args.steps):
            launches += enqueue(s)
            step_events[s].record(stream)
        stop.record(stream)
        stop.synchronize()
    torch.cuda.synchronize()
    barrier()
    elapsed_ms = start.elapsed_time(stop)
    step_ms = [start.elapsed_time(step_events[0])] + [step_events[i - 1].elapsed_time(step_events[i])
                                                      for i in range(1, args.steps)]
    last = abi.FrameResult()
    abi.check(lib.kf_frame_result_fetch(pipe.handle, C.byref(last)))

    # ---- end to end through the public API: host depth in, pose out ----------------
    # Frames in flight (kf_frame_submit / kf_frame_result_next): every step
    # copies its depth frame from pinned host memory into the pipeline's
    # staging and up to the device, and reads its result (the frame's tracker
    # state, 736 B) back to the host; up to two frames run ahead of the
    # results read.  Same fresh passes as above.  The host-synchronous loop
    # (kf_frame_process per frame, the reference's loop shape) is reported
    # beside it.
    result_bytes = 2 * 736  # the frame graph's own result copy + the queued copy
    pipe2 = kf.Pipeline(cfg)
    loop = kf.PipelinedReconstruction(pipe2, k)
    pinned = [torch.from_numpy(q.depth.view(np.int16)).pin_memory().numpy().view(np.uint16) for q in seqs]

    def submit(step: int):
        p, f = pass_of(step)
        if f == 0:
            pipe2.reset(wait=False)
            loop.frames, loop.pose = 0, identity  # the next submit sets the start pose
        loop.submit(pinned[p % n_seq][f])

    for s in range(max(args.warmup, 3)):
        submit(s)
        loop.next_result()
    loop.results.clear()
    loop.trajectory.clear()
    stream2_ptr = C.c_void_p()
    abi.check(lib.kf_pipeline_stream(pipe2.handle, C.byref(stream2_ptr)))
    stream2 = torch.cuda.ExternalStream(stream2_ptr.value)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    ahead = 2
    e0.record(stream2)
    for s in range(args.steps):
        submit(s)
        if s >= ahead:
            loop.next_result()
    while len(loop.results) < args.steps:
        loop.next_result()
    e1.record(stream2)
    e1.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)

    sync_pipe = kf.Pipeline(cfg)
    sync_loop = kf.Reconstruction(sync_pipe, k)

    def process(step: int):
        p, f = pass_of(step)
        if f == 0:
            sync_pipe.reset(wait=False)
            sync_loop.frames, sync_loop.pose = 0, abi.rigid_from_matrix(np.eye(4))
        sync_loop.process(pinned[p % n_seq][f])

    for s in range(max(args.warmup, 3)):
        process(s)
    sync_steps = min(args.steps, 400)
    sync_stream_ptr = C.c_void_p()
    abi.check(lib.kf_pipeline_stream(sync_pipe.handle, C.byref(sync_stream_ptr)))
    sync_stream = torch.cuda.ExternalStream(sync_stream_ptr.value)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    f0.record(sync_stream)
    for s in range(sync_steps):
        process(s)
    f1.record(sync_stream)
    f1.synchronize()
    e2e_sync_fps = sync_steps / (f0.elapsed_time(f1) / 1e3)
    del sync_loop, sync_pipe

    # accuracy of the e2e trajectory over the first pass of the first sequence
    ate = None
    n = min(len(loop.trajectory), SEQ_FRAMES)
    if n >= 3:
        est = np.stack(loop.trajectory[:n]).astype(np.float64)
        ate = synthetic.ate_rmse(est, seq.poses[:n])["rmse"]
    tracked_iters = [sum(r.iterations[:3]) for i, r in enumerate(loop.results) if pass_of(i)[1] != 0]
    iters_per_frame = float(np.mean(tracked_iters)) if tracked_iters else None

    # ---- dominant kernel: integration, timed alone with events on its stream -------
    # integrate_blocks_kernel (one CTA per listed 8^3 block) of a fresh pass
    # over the first sequence at its ground-truth poses: the events bracket
    # that kernel alone (the depth tiles and block culling before it, and the
    # stencil-bit rebuild after it, fall outside)
    pipe2.reset()
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev_a.record(stream2)  # torch creates the CUDA events lazily, on first record
    ev_b.record(stream2)
    abi.check(lib.kf_pipeline_set_kernel_events(pipe2.handle, C.c_void_p(ev_a.cuda_event), C.c_void_p(ev_b.cuda_event)))
    kernel_ms, kernel_updates = [], []
    pyr_probe = kf.PyramidSource()
    for idx in range(min(args.steps, SEQ_FRAMES)):
        pyr_probe.build(seq.depth[idx], k)
        normals = pyr_probe.download_level(0)["normals"]
        w2c = np.linalg.inv(seq.poses[idx])
        u0 = C.c_uint64()
        abi.check(lib.kf_pipeline_update_counts(pipe2.handle, C.byref(u0), None))
        pipe2.integrate(seq.depth[idx], k, w2c, normals=normals)
        u1 = C.c_uint64()
        abi.check(lib.kf_pipeline_update_counts(pipe2.handle, C.byref(u1), None))
        kernel_ms.append(ev_a.elapsed_time(ev_b))
        kernel_updates.append(u1.value - u0.value)
    abi.check(lib.kf_pipeline_set_kernel_events(pipe2.handle, None, None))

    # ---- secondary figures: the march alone, and the colour-on volume ---------------
    # one 640x480 render of the model (the fresh pass above, 30 frames fused)
    # at the last tracked pose into device maps, timed with events on the
    # pipeline's stream (the call syncs after them)
    rays = 640 * 480
    d_points = torch.empty(rays * 3, device="cuda")
    d_normals = torch.empty(rays * 3, device="cuda")
    d_colors = torch.empty(rays, dtype=torch.int32, device="cuda")
    maps = abi.SurfaceMapsView(d_points.data_ptr(), d_normals.data_ptr(), d_colors.data_ptr(), 640, 480,
                               abi.KF_MEMORY_DEVICE)
    cam = abi.RaycastCamera(k, 640, 480, abi.rigid_from_matrix(seq.poses[min(args.steps, SEQ_FRAMES) - 1]))
    torch.cuda.synchronize()
    rc_ms = []
    for i in range(13):
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record(stream2)
        abi.check(lib.kf_pipeline_raycast(pipe2.handle, C.byref(cam), C.byref(maps)))
        r1.record(stream2)
        r1.synchronize()
        if i >= 3:
            rc_ms.append(r0.elapsed_time(r1))
    raycast_ms = float(np.median(rc_ms))
    hits = int(torch.isfinite(d_points.view(-1, 3)).all(1).sum())
    colour = None
    if rank == 0:
        cfg_c = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_FLOAT,
                                   rule=abi.KF_RULE_ANGLE_WEIGHTED)
        pipe_c = kf.Pipeline(cfg_c)
        pyr_c, tracker_c = kf.PyramidSource(), kf.ProjectiveIcpTracker()
        sc_ptr = C.c_void_p()
        abi.check(lib.kf_pipeline_stream(pipe_c.handle, C.byref(sc_ptr)))
        stream_c = torch.cuda.ExternalStream(sc_ptr.value)
        color_dev = torch.from_numpy(seq.color.view(np.int32)).cuda()
        base0 = depth_dev[0].data_ptr()

        def enqueue_c(f: int):
            if f == 0:
                abi.check(lib.kf_pipeline_reset_async(pipe_c.handle))
                abi.check(lib.kf_frame_set_pose(pipe_c.handle, tracker_c.handle, C.byref(identity)))
            abi.check(lib.kf_frame_enqueue(pipe_c.handle, pyr_c.handle, tracker_c.handle,
                                           C.c_void_p(base0 + f * frame_bytes),
                                           C.c_void_p(color_dev.data_ptr() + f * 640 * 480 * 4), 640, 480, k,
                                           abi.KF_MEMORY_DEVICE, iters, 1 if f == 0 else 0))

        for f in range(3):
            enqueue_c(f)
        torch.cuda.synchronize()
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(stream_c)
        for f in range(SEQ_FRAMES):
            enqueue_c(f)
        c1.record(stream_c)
        c1.synchronize()
        colour = {"value": round(SEQ_FRAMES / (c0.elapsed_time(c1) / 1e3), 2), "unit": "frames/s",
                  "steps": SEQ_FRAMES, "voxel_bytes": 24, "volume_gib": 3.0,
                  "note": "one fresh 30-frame pass of the first sequence, colour frames fused"}
        del pipe_c

    elapsed_ms, e2e_ms = max_over_ranks([elapsed_ms, e2e_ms], dist, "cuda")
    if rank != 0:
        return None

    fps = replica_throughput(args.steps, world, elapsed_ms)
    e2e_fps = replica_throughput(args.steps, world, e2e_ms)
    # voxel updates per frame of a fresh pass (the counters restart with each
    # pass's refill, so they come from the kernel probe's pass at the
    # ground-truth poses)
    voxel_updates_per_step = float(np.mean(kernel_updates))
    peaks = measured_peaks()
    # algorithmic bytes of one integrate launch: read+write 8 B per fused voxel
    # plus the frame inputs it reads (depth 2 B + normals 12 B per pixel).
    frame_inputs = 640 * 480 * (2 + 12)
    alg_bytes = float(np.mean(kernel_updates)) * 16 + frame_inputs
    kernel_s = float(np.mean(kernel_ms)) / 1e3
    achieved = alg_bytes / kernel_s / 1e9
    traffic = profile_traffic()
    line = {
        "metric": METRIC, "value": round(fps, 2), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded analytic RGB-D scene)",
        "config": {**workload_config(), "parallelism": f"replicas{world}",
                   "passes": passes, "sequences": [1000 + 100 * rank + i for i in range(n_seq)]},
        "step_ms": percentiles(step_ms),
        "e2e": {"value": round(e2e_fps, 2), "unit": "frames/s", "h2d_bytes_per_step": frame_bytes,
                "d2h_bytes_per_step": result_bytes,
                "api": "PipelinedReconstruction.submit / next_result (kf_frame_submit, kf_frame_result_next), "
                       "two frames in flight, pinned host depth, fresh volume per 30-frame pass"},
        "e2e_synchronous": {"value": round(e2e_sync_fps * world, 2), "unit": "frames/s",
                            "h2d_bytes_per_step": frame_bytes, "d2h_bytes_per_step": 736, "steps": sync_steps,
                            "api": "Reconstruction.process (kf_frame_process, host sync per frame)"},
        "gpu_launches": launches,
        "gpu_launches_note": "kernel nodes of every frame graph launched in the timed region, plus the volume "
                             "fill and start-pose kernels of each new pass",
        "voxel_updates_per_s": round(voxel_updates_per_step * fps, 1),
        "icp_iters_per_frame": iters_per_frame,
        "ate_rmse_m": ate,
        "tracked_last_step": bool(last.tracked),
        "roofline": {"bound": "hbm", "kernel": "integrate_blocks_kernel<float, no colour> (block culling "
                                               "and stencil-bit rebuild outside the events)",
                     "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                     "frac": round(achieved / peaks.get("hbm_gbs", 6650.0), 4),
                     "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                     "launch_ms": round(kernel_s * 1e3, 4), "launches": len(kernel_ms),
                     "peak_source": "measured (burst copy)" if not peaks.get("fallback") else "fallback",
                     # the reference's full sweep visits every voxel: 512^3 x 16 B per launch
                     "full_grid_equivalent_gbs": round(RES ** 3 * 16 / kernel_s / 1e9, 1)},
        "raycast_640x480": {"ms": round(raycast_ms, 4), "rays_per_s": round(rays / (raycast_ms / 1e3), 1),
                            "surface_pixels": hits, "note": "march + surface kernels, one render, device maps"},
        "colour_on": colour,
        "clocks": clocks.summary(),
    }
    if args.cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(seq)
    return line


# ---- batched sequences (16 independent sequences, one graph launch per step) --------------
def batch_members(count: int = 16) -> list[dict]:
    """Seeded members: resolution from {128,192,256,384,512}, frames U[20,200],
    storage alternating int16 / bf16; the volume covers the 5.12 m scene cube."""
    rng = np.random.default_rng(4)
    from kinectfusion_b200 import abi
    members = []
    for i in range(count):
        res = int(rng.choice([128, 192, 256, 384, 512]))
        vs = 5.12 / res
        members.append({"seed": 2000 + i, "resolution": res, "voxel_size_m": vs,
                        "truncation_m": max(0.05, 3.0 * vs), "frames": int(rng.integers(20, 201)),
                        "voxel": abi.KF_VOXEL_QUANTIZED if i % 2 == 0 else abi.KF_VOXEL_BF16})
    return members


def run_batch(args) -> dict:
    import torch

    sys.path.insert(0, str(ROOT / "oracle"))
    import kf_oracle as ko
    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    members = batch_members()
    seqs = [synthetic.make_sequence(seed=m["seed"], frames=m["frames"]) for m in members]
    frames = [torch.from_numpy(s.depth.view(np.int16)).cuda() for s in seqs]

    def config(m):
        half = 0.5 * m["resolution"] * m["voxel_size_m"]
        return kf.pipeline_config(m["resolution"], m["voxel_size_m"], (-half, -half, -0.5), m["truncation_m"],
                                  voxel=m["voxel"], color=abi.KF_COLOR_NONE)

    pipelines = [kf.Pipeline(config(m)) for m in members]
    tuned = []
    for p, f in zip(pipelines, frames):
        shapes, _ = p.autotune(f.data_ptr(), 4, k)
        tuned.append([shapes.raycast_block_x, shapes.raycast_block_y, shapes.integrate_ctas])
    batch = kf.Batch(pipelines, k)
    stream = torch.cuda.ExternalStream(batch.stream())
    steps = max(m["frames"] for m in members)
    frame_bytes = 640 * 480 * 2
    total_frames = sum(m["frames"] for m in members)
    identity = abi.rigid_from_matrix(np.eye(4))

    def run_pass() -> float:
        for p, t in zip(pipelines, batch.trackers):
            p.reset()
            abi.check(abi.load().kf_frame_set_pose(p.handle, t.handle, C.byref(identity)))
        batch.frames = [0] * len(members)
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for step in range(steps):
            batch.step([f.data_ptr() + step * frame_bytes if step < m["frames"] else None
                        for f, m in zip(frames, members)])
        stop.record(stream)
        stop.synchronize()
        return start.elapsed_time(stop)

    run_pass()  # captures every member's frame graphs and the step graphs
    with ClockSampler(torch.cuda.current_device()) as clocks:
        clocks.wait_started()
        elapsed_ms = run_pass()
    kernels = batch.kernel_count()

    # precision: the first 3 frames of each member against the FP64 oracle
    # integration at the device's own poses, and one normal-equation sweep
    # against the FP64 reduction
    precision = []
    for m, seq in zip(members, seqs):
        loop = kf.Reconstruction(kf.Pipeline(config(m)), k)
        ref = ko.OracleVolumeF64(m["resolution"], m["voxel_size_m"],
                                 (-0.5 * m["resolution"] * m["voxel_size_m"],) * 2 + (-0.5,), m["truncation_m"])
        for f in range(3):
            loop.process(seq.depth[f])
            if loop.results[-1].tracked:
                normals = ko.pyramid(seq.depth[f], k, ko.depth_options())[0]["normals"]
                w2c = ko.rigid_inverse(abi.rigid_from_matrix(loop.trajectory[-1]))
                ko.integrate_f64(ref, seq.depth[f], k, w2c, ko.integration_options(), normals_map=normals,
                                 threads=os.cpu_count() or 1)
        tsdf, weight = loop.pipeline.host_view()
        rt, rw = ref.dense()
        both = (weight > 0) & (rw > 0)
        err = np.abs(tsdf[both].astype(np.float64) - rt[both]) * m["truncation_m"]
        quantum = 1.0 / 32767.0 if m["voxel"] == abi.KF_VOXEL_QUANTIZED else 1.0 / 256.0
        within = float(np.mean(np.abs(tsdf[both].astype(np.float64) - rt[both]) <= quantum)) if both.any() else None
        precision.append({"resolution": m["resolution"], "storage": "int16" if m["voxel"] == abi.KF_VOXEL_QUANTIZED
                          else "bf16", "voxels_compared": int(both.sum()),
                          "tsdf_err_m_median": float(np.median(err)) if both.any() else None,
                          "tsdf_err_m_p999": float(np.percentile(err, 99.9)) if both.any() else None,
                          "tsdf_err_m_max": float(err.max()) if both.any() else None,
                          "within_one_code": within})
    # ICP: one level-2 sweep of member 0 against the FP64 reduction
    m, seq = members[0], seqs[0]
    probe = kf.Reconstruction(kf.Pipeline(config(m)), k)
    for f in range(3):
        probe.process(seq.depth[f])
    pyr = kf.PyramidSource()
    pyr.build(seq.depth[3], k)
    kl = ko.scaled(k, 2)
    maps = probe.pipeline.raycast(kl, 160, 120, probe.trajectory[-1])
    live = pyr.download_level(2)
    camera = abi.rigid_from_matrix(probe.trajectory[-1])
    model = ko.rigid_inverse(camera)
    s64, c64 = ko.icp_equations(live["vertices"], live["normals"], maps.points, maps.normals, kl, camera, model,
                                f64=True)
    d_points = torch.from_numpy(np.ascontiguousarray(maps.points).view(np.uint8).reshape(-1)).cuda()
    d_normals = torch.from_numpy(np.ascontiguousarray(maps.normals).view(np.uint8).reshape(-1)).cuda()
    sums, count = np.zeros(29, dtype=np.float32), C.c_uint64()
    tr = kf.ProjectiveIcpTracker()
    torch.cuda.synchronize()
    abi.check(abi.load().kf_icp_normal_equations(tr.handle, C.byref(pyr.level(2)), C.c_void_p(d_points.data_ptr()),
                                                 C.c_void_p(d_normals.data_ptr()), 160, 120, kl, C.byref(camera),
                                                 C.byref(model), sums.ctypes.data_as(C.c_void_p), C.byref(count)))
    icp_rel = float(np.abs(sums.astype(np.float64) - s64).max() / max(np.abs(s64).max(), 1e-30))

    fps = total_frames / (elapsed_ms / 1e3)
    return {"metric": "frames/s, 16 independent sequences in one graph launch per step", "value": round(fps, 2),
            "unit": "frames/s", "n_gpus": 1, "steps": steps, "warmup": steps, "ms_per_step": round(elapsed_ms / steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (int16/bf16 storage)",
            "data": "synthetic (seeded analytic RGB-D scenes)",
            "config": {"workload": "16 seeded sequences of 640x480 frames, dense volumes of uneven resolution, "
                                   "int16/bf16 alternating, angle-weighted TSDF, ICP [10,5,4], all members "
                                   "stepped in one graph launch", "members": [
                                       {k2: (v if k2 != "voxel" else ("int16" if v == abi.KF_VOXEL_QUANTIZED else "bf16"))
                                        for k2, v in m.items()} for m in members],
                       "autotuned_shapes": tuned, "total_frames": total_frames,
                       "l2": "volumes and frames larger than L2 in total, no flush"},
            "gpu_launches": kernels, "gpu_launches_note": "kernel nodes of the last step graph",
            "precision_vs_fp64": {"tsdf": precision, "icp_sums_max_rel_err": icp_rel, "icp_pixels": int(c64)},
            "clocks": clocks.summary()}


# ---- CPU baseline (the reference's own host code, bounded sample) ----------------------------
def cpu_baseline(seq, frames: int = 2) -> dict:
    """The reference's host path on one core (oracle/_ref/libkf_ref.so, its
    own sources compiled here; single-threaded by construction) over a
    bounded sample: the first frame fused, then `frames` tracked frames of
    the same 512^3 workload.  Falls back to the oracle port, also on one
    core, when the library was not built."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import kf_oracle as ko
    import kf_ref as kr
    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    pose = np.eye(4, dtype=np.float32)
    if kr.available():
        model = kr.RefPipeline(kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE,
                                                  rule=abi.KF_RULE_ANGLE_WEIGHTED))

        def frame(i, first=False):
            return model.track_frame(seq.depth[i], k, pose, ko.depth_options(), ko.icp_options(), first=first)[0]
        kind, what = "reference", "the reference's own host code (oracle/_ref/libkf_ref.so), 1 thread"
    else:
        vol = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC)
        opts = (ko.depth_options(), ko.integration_options(), ko.raycast_options(), ko.icp_options())

        def frame(i, first=False):
            return ko.track_frame(vol, seq.depth[i], k, pose, *opts, threads=1, first=first)[0]
        kind, what = "port", "the CPU oracle port, 1 thread (oracle/_ref was not built)"
    pose = frame(0, True)
    t0 = time.perf_counter()
    for f in range(1, 1 + frames):
        pose = frame(f)
    dt = time.perf_counter() - t0
    return {"value": round(frames / dt, 4), "unit": "frames/s", "cores": 1, "kind": kind,
            "host_cores": os.cpu_count(),
            "sample": f"{frames} tracked frames of the same 512^3 workload (after one fused first frame), {what}"}


# ---- reference arm -----------------------------------------------------------------------------
def run_reference(args, rank: int) -> dict | None:
    """The reference's CPU implementation of the path: its own host code
    (src/kinectfusion/*.cpp compiled from source into oracle/_ref/libkf_ref.so
    by oracle/ref_build.sh), driven frame by frame as
    Reconstruction::process_frame does, on the same fresh 30-frame sequence
    and 512^3 workload as our arm.  The reference's host path is
    single-threaded by construction (plain loops, README.md:109-111), so it
    runs on one core.  Each step is one frame (about 3.5 s); the run is
    bounded to KF_REFERENCE_MAX_FRAMES frames in total (default 30).  Falls
    back to the oracle port (kf_oracle.c) when the library was not built."""
    if rank != 0:
        return None
    sys.path.insert(0, str(ROOT / "oracle"))
    import kf_oracle as ko
    import kf_ref as kr
    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    seq = synthetic.make_sequence(seed=1000, frames=SEQ_FRAMES)
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    steps, warmup = args.steps, max(1, args.warmup)
    budget = int(os.environ.get("KF_REFERENCE_MAX_FRAMES", "30"))
    if steps + warmup > budget:
        warmup = min(warmup, 2)
        steps = max(1, budget - warmup)
    pose = np.eye(4, dtype=np.float32)
    if kr.available():
        kind, cores = "reference", 1
        cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED)
        model = kr.RefPipeline(cfg)

        def frame(i: int, first: bool):
            nonlocal pose
            pose, _, _ = model.track_frame(seq.depth[i], k, pose, ko.depth_options(), ko.icp_options(), first=first)
        what = "the reference's own host code (oracle/_ref/libkf_ref.so, compiled from its sources), 1 thread"
    else:
        kind, cores = "port", os.cpu_count() or 1
        vol = ko.OracleVolume(RES, VOXEL, ORIGIN, TRUNC)
        opts = (ko.depth_options(), ko.integration_options(), ko.raycast_options(), ko.icp_options())

        def frame(i: int, first: bool):
            nonlocal pose
            pose, _, _ = ko.track_frame(vol, seq.depth[i], k, pose, *opts, threads=cores, first=first)
        what = f"the CPU oracle port ({cores} OpenMP threads; oracle/_ref was not built)"
    frame(0, True)  # the first frame is fused without tracking
    for s in range(1, 1 + warmup):
        frame(s, False)
    t0 = time.perf_counter()
    for s in range(steps):
        frame((1 + warmup + s) % SEQ_FRAMES, False)
    dt = time.perf_counter() - t0
    fps = steps / dt
    return {"impl": "reference", "metric": METRIC, "value": round(fps, 4), "unit": "frames/s", "n_gpus": 0,
            "steps": steps, "warmup": warmup, "ms_per_step": round(dt / steps * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded analytic RGB-D scene)",
            "config": {**workload_config(), "parallelism": f"cpu{cores}"},
            "cpu_baseline": {"value": round(fps, 4), "unit": "frames/s", "cores": cores, "kind": kind,
                             "host_cores": os.cpu_count(),
                             "sample": f"frames 1..{warmup + steps} of the first 30-frame sequence after its fused "
                                       f"first frame ({warmup} untimed), {what}"},
            "e2e": {"value": round(fps, 4), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_cuda(args) -> dict:
    """The reference's own CUDA pipeline on this GPU: src/kinectfusion/cuda/*.cu
    built for sm_100a from its sources (oracle/_ref/libkf_ref_cuda.so), run as
    its app's frame loop (Reconstruction::process_frame with --space cuda
    --preload: host frames uploaded by its device pyramid source, its device
    model renders, its device correspondence sweeps).  Beside it, on the same
    frames and clock: the same reference loop with its device seams taken by
    this project's drop-in glue (kinectfusion_b200/glue/b200_backend.cpp over
    libkf_b200.so, oracle/_ref/libkf_ref_b200.so) and this project's own
    host-frame loop (kf_frame_process).  Timed by the host clock around each
    fresh 30-frame pass, as the reference's own fps line is
    (reconstruction.cpp:117-138)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import kf_oracle as ko
    import kf_ref as kr
    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    passes = max(1, args.steps // SEQ_FRAMES)
    seqs = [synthetic.make_sequence(seed=1000 + i, frames=SEQ_FRAMES) for i in range(min(passes, 4))]

    class Ours:
        def __init__(self, cfg):
            self.loop = kf.Reconstruction(kf.Pipeline(cfg), k)

        def process(self, depth, color):
            return bool(self.loop.process(depth, color).tracked)

        def synchronize(self):
            pass  # process() returns after the frame's result is on the host

    class Reference:
        def __init__(self, cfg, backend, device_solve):
            self.loop = kr.RefDevicePipeline(cfg, ko.depth_options(), ko.icp_options(), device_solve=device_solve,
                                             backend=backend)

        def process(self, depth, color):
            return self.loop.process(depth, k, color)[0]

        def synchronize(self):
            self.loop.synchronize()

    rows = []
    for name, color, device_solve in (("default (colour float, host solve)", abi.KF_COLOR_FLOAT, False),
                                      ("--color none", abi.KF_COLOR_NONE, False),
                                      ("--color none --icp-device-solve", abi.KF_COLOR_NONE, True)):
        cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=color, rule=abi.KF_RULE_ANGLE_WEIGHTED)
        makers = {"reference_cuda": lambda: Reference(cfg, "cuda", device_solve),
                  "reference_over_glue": lambda: Reference(cfg, "glue", device_solve),
                  "ours": lambda: Ours(cfg)}
        timings = {}
        for impl, make in makers.items():
            if impl == "reference_over_glue" and not kr.cuda_available("glue"):
                continue
            warm = make()  # warm-up pass of three frames on a throwaway instance
            for f in range(3):
                warm.process(seqs[0].depth[f], seqs[0].color[f] if color == abi.KF_COLOR_FLOAT else None)
            warm.synchronize()
            del warm
            total, frames, tracked = 0.0, 0, 0
            for p in range(passes):
                q = seqs[p % len(seqs)]
                loop = make()
                loop.synchronize()
                t0 = time.perf_counter()
                for f in range(SEQ_FRAMES):
                    tracked += int(loop.process(q.depth[f], q.color[f] if color == abi.KF_COLOR_FLOAT else None))
                loop.synchronize()
                total += time.perf_counter() - t0
                frames += SEQ_FRAMES
                del loop
            timings[impl] = {"fps": round(frames / total, 1), "tracked": tracked}
        row = {"flags": name, "frames": frames,
               **{f"{impl}_fps": t["fps"] for impl, t in timings.items()},
               "tracked": {impl: t["tracked"] for impl, t in timings.items()},
               "ours_over_reference_cuda": round(timings["ours"]["fps"] / timings["reference_cuda"]["fps"], 2)}
        if "reference_over_glue" in timings:
            row["glue_over_reference_cuda"] = round(timings["reference_over_glue"]["fps"] /
                                                    timings["reference_cuda"]["fps"], 2)
        rows.append(row)
    return {"metric": "frames/s, the reference's own CUDA pipeline on this B200 (640x480, 512^3)",
            "value": rows[1]["reference_cuda_fps"], "unit": "frames/s", "n_gpus": 1, "steps": passes * SEQ_FRAMES,
            "warmup": 3, "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded analytic RGB-D scene)",
            "config": {**workload_config(), "timing": "host clock around each fresh 30-frame pass (the reference's "
                                                     "own fps line), host frames in, every implementation"},
            "rows": rows}


# The reference's published ablation rows (README.md:199-214, RTX 5080, TUM
# freiburg1_desk, 512^3 at 0.01 m, colour on): flag -> (config keywords, fps).
ABLATIONS = [
    ("baseline", {}, 545),
    ("--cell-normals", {"raycast_cell_gradient_normals": 1}, 840),
    ("--integration band", {"integration_mode": 1}, 680),
    ("--icp-device-solve", {}, 570),
    ("--tsdf-variant classic", {"rule": 0}, 565),
    ("--color none", {"color": 0}, 560),
    ("--distance-scaled-truncation", {"integration_distance_scaled_truncation": 1}, 550),
    ("--no-projective-tsdf-distance", {"integration_projective_distance": 0}, 550),
    ("--voxel bf16", {"voxel": 2}, 550),
    ("--voxel quantized", {"voxel": 1}, 545),
    ("--icp-capture-graph", {}, 540),
    ("--raycast-seed-previous", {"raycast_seed_from_previous": 1}, 540),
    ("--raycast-tsdf-from-valid-corners", {"raycast_corner_policy": 1}, 515),
    ("--storage sparse --integration band", {"storage": 1, "integration_mode": 1}, 505),
    ("--raycast bitmap-march", {"raycast_backend": 1}, 140),
    ("--raycast band-march", {"raycast_backend": 2}, 135),
]


def run_ablations(args) -> dict:
    """The reference's ablation table on this pipeline: the cfg2 sequence
    (512^3 at 0.01 m, angle-weighted, colour on unless the row turns it off)
    under each of the reference's flags, frames/s over device-resident frames.
    Rows whose flag selects what this pipeline always does (the device solve,
    the captured graph) run the baseline configuration."""
    import torch

    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    lib = abi.load()
    seq = synthetic.make_sequence(seed=1000, frames=SEQ_FRAMES)
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    depth_dev = torch.from_numpy(seq.depth.view(np.int16)).cuda()
    color_dev = torch.from_numpy(seq.color.view(np.int32)).cuda()
    iters = (C.c_uint32 * 4)(10, 5, 4, 4)
    steps = min(args.steps, 300)
    rows = []
    for flag, kw, ref_fps in ABLATIONS:
        kw = dict(kw)
        color = kw.pop("color", abi.KF_COLOR_FLOAT)
        rule = kw.pop("rule", abi.KF_RULE_ANGLE_WEIGHTED)
        cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=color, rule=rule, **kw)
        pipe = kf.Pipeline(cfg)
        pyr, tracker = kf.PyramidSource(), kf.ProjectiveIcpTracker()
        sp = C.c_void_p()
        abi.check(lib.kf_pipeline_stream(pipe.handle, C.byref(sp)))
        stream = torch.cuda.ExternalStream(sp.value)

        def enqueue(step: int):
            idx = frame_schedule(step)
            col = C.c_void_p(color_dev.data_ptr() + idx * 640 * 480 * 4) if color == abi.KF_COLOR_FLOAT else None
            abi.check(lib.kf_frame_enqueue(pipe.handle, pyr.handle, tracker.handle,
                                           C.c_void_p(depth_dev.data_ptr() + idx * 640 * 480 * 2), col, 640, 480,
                                           k, abi.KF_MEMORY_DEVICE, iters, 1 if step == 0 else 0))

        for st in range(3):
            enqueue(st)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for st in range(steps):
            enqueue(3 + st)
        b.record(stream)
        b.synchronize()
        fps = steps / (a.elapsed_time(b) / 1e3)
        last = abi.FrameResult()
        abi.check(lib.kf_frame_result_fetch(pipe.handle, C.byref(last)))
        rows.append({"flag": flag, "fps": round(fps, 1), "reference_rtx5080_fps": ref_fps,
                     "tracked_last_frame": bool(last.tracked)})
        del pipe, pyr, tracker
        torch.cuda.synchronize()
    base = rows[0]["fps"]
    return {
        "metric": "frames/s per reference ablation flag (640x480, 512^3)", "value": base, "unit": "frames/s",
        "n_gpus": 1, "steps": steps, "warmup": 3, "higher_is_better": True, "scaling": "none", "vs_baseline": None,
        "dtype": "per row", "data": "synthetic (seeded analytic RGB-D scene)",
        "config": {"workload": "cfg2 sequence, 512^3 at 0.01 m, colour on unless the row turns it off, "
                               "ICP [10,5,4]; the reference's figures are from README.md on an RTX 5080 with "
                               "TUM freiburg1_desk (another scene and GPU)"},
        "rows": rows,
    }


def _live_bricks(a, b) -> int:
    """8^3 bricks where either volume holds a voxel of weight > 0 (from the
    dense host views): the bricks the volume comparator must read."""
    counts = []
    for p in (a, b):
        _, w = p.host_view()
        rz, ry, rx = w.shape
        counts.append((w > 0).reshape(rz // 8, 8, ry // 8, 8, rx // 8, 8).any(axis=(1, 3, 5)))
    return int((counts[0] | counts[1]).sum())


def run_compare(args) -> dict:
    """The pipeline-set ablation run with a comparison every frame
    (--pipelines ... with compare_every_n_frames 1): three 512^3 members
    (baseline float + colour, classic float, bf16) each track and integrate
    the cfg2 frames, then all are raycast at 640x480 from the baseline's pose
    and compared with it on the device.  `value` is set frames/s; the
    roofline is the volume comparator's kernel (one read of both volumes)."""
    import torch

    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic
    from kinectfusion_b200.pipeline_set import PipelineSet, compare_volumes

    lib = abi.load()
    seq = synthetic.make_sequence(seed=1000, frames=SEQ_FRAMES)
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    depth_dev = torch.from_numpy(seq.depth.view(np.int16)).cuda()
    color_dev = torch.from_numpy(seq.color.view(np.int32)).cuda()
    iters = (C.c_uint32 * 4)(10, 5, 4, 4)
    res = args.compare_res
    origin = (-0.5 * res * VOXEL, -0.5 * res * VOXEL, -0.5)
    members = [kf.Pipeline(kf.pipeline_config(res, VOXEL, origin, TRUNC), "baseline"),
               kf.Pipeline(kf.pipeline_config(res, VOXEL, origin, TRUNC, rule=abi.KF_RULE_CLASSIC,
                                              color=abi.KF_COLOR_NONE), "classic"),
               kf.Pipeline(kf.pipeline_config(res, VOXEL, origin, TRUNC, voxel=abi.KF_VOXEL_BF16,
                                              color=abi.KF_COLOR_NONE), "bf16")]
    pset = PipelineSet(members, reference="baseline")
    pyramids = [kf.PyramidSource() for _ in members]
    trackers = [kf.ProjectiveIcpTracker() for _ in members]
    sp = C.c_void_p()
    abi.check(lib.kf_pipeline_stream(members[1].handle, C.byref(sp)))
    classic_stream = torch.cuda.ExternalStream(sp.value)

    def step(s: int, compare: bool = True):
        idx = frame_schedule(s)
        d = C.c_void_p(depth_dev.data_ptr() + idx * 640 * 480 * 2)
        for i, m in enumerate(members):
            col = C.c_void_p(color_dev.data_ptr() + idx * 640 * 480 * 4) if i == 0 else None
            abi.check(lib.kf_frame_enqueue(m.handle, pyramids[i].handle, trackers[i].handle, d, col, 640, 480, k,
                                           abi.KF_MEMORY_DEVICE, iters, 1 if s == 0 else 0))
        r = abi.FrameResult()
        for m in members:
            abi.check(lib.kf_frame_result_fetch(m.handle, C.byref(r)))
        if compare:
            abi.check(lib.kf_frame_result_fetch(members[0].handle, C.byref(r)))
            outputs = pset.raycast_all(k, 640, 480, r.camera_to_world)
            return pset.compare(outputs)
        return None

    warm = max(args.warmup, 3)
    for s in range(warm):
        step(s)
    torch.cuda.synchronize()
    steps = min(args.steps, 100)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        clocks.wait_started()
        t0 = time.perf_counter()
        for s in range(steps):
            last = step(warm + s)
        torch.cuda.synchronize()
        set_s = time.perf_counter() - t0
        # the same frames without the comparisons, for the comparison's share
        t0 = time.perf_counter()
        for s in range(steps):
            step(warm + steps + s, compare=False)
        torch.cuda.synchronize()
        plain_s = time.perf_counter() - t0
        # the volume comparator alone (classic vs baseline: two float volumes),
        # CUDA events on the primary's stream around the whole call
        times = []
        for _ in range(20):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(classic_stream)
            compare_volumes(members[1], members[0])
            e1.record(classic_stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    compare_ms = float(np.median(times))
    # algorithmic bytes: the observed bits of both volumes (64 B per brick
    # each) and both float bricks wherever either volume observed a voxel
    blocks = (res // 8) ** 3
    live = _live_bricks(members[1], members[0])
    traffic_bytes = blocks * 2 * 64 + live * 2 * 4096
    gbs = traffic_bytes / (compare_ms / 1e3) / 1e9
    peaks = measured_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    # CPU baseline: the oracle's Comparator on the two downloaded host views
    # (the reference's path: host_view of both volumes, then a host loop)
    cpu = None
    if args.cpu_baseline:
        sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent / "oracle"))
        import kf_compare_oracle as kco
        t0 = time.perf_counter()
        views = (members[1].host_view(), members[0].host_view())
        download_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        kco.compare_volumes(*views)
        cpu_s = time.perf_counter() - t0
        cpu = {"value": round(1000.0 * (cpu_s + download_s), 1), "unit": "ms per volume comparison", "cores": 1,
               "kind": "port", "sample": "one 512^3 float-vs-float comparison: host_view download of both volumes "
                                         f"({round(1000 * download_s, 1)} ms) + numpy Comparator"}
    return {
        "metric": f"pipeline-set frames/s, 3 members at {res}^3, compared every frame", "value": round(steps / set_s, 1),
        "unit": "frames/s", "n_gpus": 1, "steps": steps, "warmup": warm, "ms_per_step": round(1000 * set_s / steps, 3),
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32 / bf16 voxels, f64 sums",
        "data": "synthetic (seeded analytic RGB-D scene)",
        "config": {"workload": "members baseline (float + colour), classic (float), bf16; 640x480 cfg2 frames from "
                               "HBM; per frame: every member tracks and integrates, all raycast at 640x480 from the "
                               "baseline's pose, kf_compare_volumes + kf_compare_surface_maps per member; inputs "
                               "larger than L2"},
        "frames_per_s_without_comparison": round(steps / plain_s, 1),
        "compare_volumes_ms": round(compare_ms, 4),
        "compare_live_bricks": {"live": int(live), "of": int(blocks), "algorithmic_bytes": int(traffic_bytes),
                                "full_read_bytes": int(res ** 3 * 16)},
        "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(gbs / peak, 4), "traffic": None,
                     "peak_source": "measured" if not peaks.get("fallback") else "fallback",
                     "kernel": "kf_compare_volumes, float vs float: live-block passes (mask, scan, list), "
                               "compare_volumes_kernel, finish kernel and result copy, event to event"},
        "last_comparisons": [c.csv() for c in last],
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }


def run_integrate(args) -> dict:
    """The integration kernel alone on the headline geometry: one fresh dense
    512^3 float volume (1 GiB, larger than L2; about 1.1 GB on the device in
    all), the first 30-frame sequence integrated at its ground-truth poses
    (pixel table, depth tiles, block culling, integrate_blocks_kernel,
    stencil bits per frame), CUDA events around integrate_blocks_kernel only.
    The small, single-pipeline entry point that ncu captures target."""
    import torch

    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    lib = abi.load()
    seq = synthetic.make_sequence(seed=1000, frames=SEQ_FRAMES)
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    cfg = kf.pipeline_config(RES, VOXEL, ORIGIN, TRUNC, color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED)
    pipe = kf.Pipeline(cfg)
    sp = C.c_void_p()
    abi.check(lib.kf_pipeline_stream(pipe.handle, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    pyr = kf.PyramidSource()
    normals = []
    for f in range(SEQ_FRAMES):
        pyr.build(seq.depth[f], k)
        normals.append(pyr.download_level(0)["normals"])
    ev_a, ev_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev_a.record(stream)
    ev_b.record(stream)
    abi.check(lib.kf_pipeline_set_kernel_events(pipe.handle, C.c_void_p(ev_a.cuda_event), C.c_void_p(ev_b.cuda_event)))
    frames = min(max(args.steps, 1), SEQ_FRAMES)
    ms, updates = [], []
    for f in range(frames):
        u0 = C.c_uint64()
        abi.check(lib.kf_pipeline_update_counts(pipe.handle, C.byref(u0), None))
        pipe.integrate(seq.depth[f], k, np.linalg.inv(seq.poses[f]), normals=normals[f])
        u1 = C.c_uint64()
        abi.check(lib.kf_pipeline_update_counts(pipe.handle, C.byref(u1), None))
        ms.append(ev_a.elapsed_time(ev_b))
        updates.append(u1.value - u0.value)
    abi.check(lib.kf_pipeline_set_kernel_events(pipe.handle, None, None))
    listed = C.c_uint64()
    abi.check(lib.kf_pipeline_listed_blocks(pipe.handle, C.byref(listed)))
    timed = slice(1, None) if frames > 1 else slice(None)
    alg = float(np.mean(updates[timed])) * 16 + 640 * 480 * 14
    kernel_s = float(np.mean(ms[timed])) / 1e3
    peaks = measured_peaks()
    achieved = alg / kernel_s / 1e9
    return {"metric": "integrate_blocks_kernel GB/s of algorithmic traffic (640x480 into 512^3 float)",
            "value": round(achieved, 1), "unit": "GB/s", "n_gpus": 1, "steps": frames, "warmup": 1,
            "ms_per_step": round(kernel_s * 1e3, 4), "higher_is_better": True, "scaling": "none",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded analytic RGB-D scene)",
            "config": {"workload": "one fresh dense 512^3 float volume, frames 0..N-1 of the first sequence "
                                   "integrated at ground-truth poses, angle-weighted, colour off"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                         "frac": round(achieved / peaks.get("hbm_gbs", 6650.0), 4),
                         "alg_bytes_per_launch": alg, "launch_ms": round(kernel_s * 1e3, 4)},
            "per_frame_ms": [round(m, 4) for m in ms], "voxel_updates": updates,
            "listed_blocks_last_frame": int(listed.value)}


def run_gemm(args) -> dict:
    """The tensor-core kernel alone (kf_gemm_bf16, the learned warm start's
    matrix engine): a square 8192^3 bf16 product with FP32 accumulation,
    device-resident operands, against the measured cuBLAS bf16 peak."""
    import torch

    from kinectfusion_b200 import abi

    lib = abi.load()
    m = n = k = args.gemm_size
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    a = torch.randn(m, k, device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn(n, k, device="cuda", generator=g).to(torch.bfloat16)
    c = torch.empty(m, n, device="cuda")
    stream = torch.cuda.current_stream()

    def run():
        abi.check(lib.kf_gemm_bf16(C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), C.c_void_p(c.data_ptr()),
                                   m, n, k, None, 0, C.c_void_p(stream.cuda_stream)))

    for _ in range(max(args.warmup, 3)):
        run()
    torch.cuda.synchronize()
    steps = min(args.steps, 50)
    times = []
    with ClockSampler(torch.cuda.current_device()) as clocks:
        clocks.wait_started()
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    tflops = 2.0 * m * n * k / (ms / 1e3) / 1e12
    # accuracy against an FP32 product of the same bf16 operands (a slice)
    ref = a[:256].float() @ b.float().T
    err = float((c[:256] - ref).abs().max() / (ref.abs().max() + 1.0))
    peaks = measured_peaks()
    peak = peaks.get("bf16_tflops", 1590.0)
    return {
        "metric": f"bf16 GEMM TFLOP/s (tcgen05, {m}x{n}x{k})", "value": round(tflops, 1), "unit": "TFLOP/s",
        "n_gpus": 1, "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "bf16 in, f32 accumulate",
        "data": "synthetic (seeded normal operands)",
        "config": {"workload": f"C = A B^T, A {m}x{k}, B {n}x{k} bf16 row-major, C fp32; 128 x 128 tiles, "
                               "4-stage TMA ring, kf_gemm_bf16 (includes its call overhead)"},
        "roofline": {"bound": "tensor", "achieved": round(tflops, 1), "peak": peak, "unit": "TFLOP/s",
                     "frac": round(tflops / peak, 4), "traffic": None,
                     "peak_source": "measured" if not peaks.get("fallback") else "fallback"},
        "max_rel_error_vs_fp32": err,
        "clocks": clocks.summary(),
    }


def run_sparse(args) -> dict:
    """cfg3: one sequence of 300 frames (steps up to 2 cm / 1 deg) tracked and
    fused into a sparse 8^3-block hash over a 2048^3 domain of 5 mm voxels
    (bf16 voxels, band integration, angle-weighted TSDF, plain march), then
    the block-wise mesh with min weight 2."""
    import torch

    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, synthetic

    lib = abi.load()
    frames = args.sparse_frames
    seq = synthetic.make_sequence_device(seed=3000, frames=frames, max_step_m=0.02, max_step_deg=1.0)
    k = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
    res, vs = 2048, 0.005
    cfg = kf.pipeline_config(res, vs, (-0.5 * res * vs, -0.5 * res * vs, -0.5), 0.05, voxel=abi.KF_VOXEL_BF16,
                             color=abi.KF_COLOR_NONE, rule=abi.KF_RULE_ANGLE_WEIGHTED,
                             storage=abi.KF_STORAGE_SPARSE, integration_mode=abi.KF_INTEGRATION_BAND)
    pipe = kf.Pipeline(cfg)
    pyr, tracker = kf.PyramidSource(), kf.ProjectiveIcpTracker()
    iters = (C.c_uint32 * 4)(10, 5, 4, 4)
    sp = C.c_void_p()
    abi.check(lib.kf_pipeline_stream(pipe.handle, C.byref(sp)))
    stream = torch.cuda.ExternalStream(sp.value)
    depth_dev = torch.from_numpy(seq.depth.view(np.int16)).cuda()
    frame_bytes = 640 * 480 * 2

    def enqueue(f: int):
        abi.check(lib.kf_frame_enqueue(pipe.handle, pyr.handle, tracker.handle,
                                       C.c_void_p(depth_dev.data_ptr() + f * frame_bytes), None, 640, 480, k,
                                       abi.KF_MEMORY_DEVICE, iters, 1 if f == 0 else 0))

    warm = max(args.warmup, 3)
    for f in range(warm):
        enqueue(f)
    torch.cuda.synchronize()
    u0 = C.c_uint64()
    abi.check(lib.kf_pipeline_update_counts(pipe.handle, C.byref(u0), None))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        clocks.wait_started()
        e0.record(stream)
        for f in range(warm, frames):
            enqueue(f)
        e1.record(stream)
        e1.synchronize()
    ms = e0.elapsed_time(e1)
    u1 = C.c_uint64()
    abi.check(lib.kf_pipeline_update_counts(pipe.handle, C.byref(u1), None))
    attempts, capacity = pipe.block_stats()
    last = abi.FrameResult()
    abi.check(lib.kf_frame_result_fetch(pipe.handle, C.byref(last)))
    t0 = time.perf_counter()
    mesh = pipe.extract_mesh(2.0)
    mesh_s = time.perf_counter() - t0
    timed = frames - warm
    fps = timed / (ms / 1e3)
    return {
        "metric": "frames/s (640x480, sparse 2048^3 domain, bf16)", "value": round(fps, 2), "unit": "frames/s",
        "n_gpus": 1, "steps": timed, "warmup": warm, "ms_per_step": round(ms / timed, 4),
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "bf16 voxels, f32 math",
        "data": "synthetic (seeded analytic RGB-D scene, steps up to 2 cm / 1 deg, frames rendered on the device)",
        "config": {"workload": f"cfg3: {frames} frames into a sparse 8^3-block hash over a 2048^3 domain of 5 mm "
                               "voxels (bf16, band integration, angle-weighted TSDF, march raycast), then the "
                               "block-wise mesh (min weight 2)",
                   "blocks_capacity": capacity, "pool_gib": round(capacity * 512 * 4 / 2 ** 30, 2)},
        "voxel_updates_per_s": round((u1.value - u0.value) / (ms / 1e3), 1),
        "allocated_blocks": min(attempts, capacity), "allocation_attempts": attempts,
        "tracked_last_frame": bool(last.tracked),
        "mesh": {"seconds": round(mesh_s, 3), "vertices": int(len(mesh["positions"])),
                 "triangles": int(len(mesh["triangles"]))},
        "gpu_launches": None,
        "clocks": clocks.summary(),
    }


def run_learned(args) -> dict:
    """cfg5: ICP iterations per frame with the learned warm start against the
    plain constant-velocity start, on held-out seeds at 512^3 dense float,
    with ATE; plus the frame rate of the learned loop through the public API
    (host depth frames) and the net's device latency."""
    import torch

    import kinectfusion_b200 as kf
    from kinectfusion_b200 import abi, learned, synthetic

    seeds = list(range(5000, 5000 + args.learned_seeds))
    net = learned.Learner(8, seed=0)
    net.load(learned.PARAMS)
    gpu = kf.Pipeline(learned.volume_config(RES, VOXEL))
    report = learned.evaluate(net, seeds, args.learned_frames, pipeline=gpu)
    one_step = learned.one_step_errors(net, seeds, args.learned_frames, pipeline=gpu)
    mean = report["mean"]
    tracked = [r for r in report["per_seed"] if r["ate_velocity_m"] < 0.01]

    # frame rate of each loop over one held-out sequence (host frames in,
    # pose out, every call synchronous as a caller sees it)
    seq = synthetic.make_sequence_device(seeds[0], args.learned_frames, 0.05, 3.0)
    rates = {}
    for mode in ("velocity", "learned"):
        gpu.reset()
        loop = learned.WarmStartedReconstruction(gpu, learned.intrinsics640(), start=mode, learner=net)
        for f in range(3):
            loop.process(seq.depth[f])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for f in range(3, args.learned_frames):
            loop.process(seq.depth[f])
        rates[mode] = (args.learned_frames - 3) / (time.perf_counter() - t0)
    # the same two loops with every step on the device and device-resident
    # frames (kf_warm_start_enqueue + kf_frame_enqueue, one sync at the end)
    dev_depth = torch.from_numpy(seq.depth.view(np.int16)).cuda()
    device_rates = {}
    for mode in ("velocity", "learned"):
        gpu.reset()
        aloop = learned.AsyncLearnedLoop(gpu, learned.intrinsics640(), net, use_net=(mode == "learned"))
        stream_ptr = C.c_void_p()
        abi.check(abi.load().kf_pipeline_stream(gpu.handle, C.byref(stream_ptr)))
        astream = torch.cuda.ExternalStream(stream_ptr.value)
        for f in range(3):
            aloop.enqueue(dev_depth.data_ptr() + f * 640 * 480 * 2)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(astream)
        for f in range(3, args.learned_frames):
            aloop.enqueue(dev_depth.data_ptr() + f * 640 * 480 * 2)
        a1.record(astream)
        a1.synchronize()
        device_rates[mode] = (args.learned_frames - 3) / (a0.elapsed_time(a1) / 1e3)
    # the net's forward pass alone (batch 8, device-resident input)
    x = torch.zeros((8, 60, 80, 2), dtype=torch.bfloat16, device="cuda")
    for _ in range(10):
        net.forward(x)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(200):
        net.forward(x)
    stop.record()
    stop.synchronize()
    forward_ms = start.elapsed_time(stop) / 200
    return {
        "metric": "ICP iterations per frame (learned warm start vs constant velocity, equal ATE)",
        "value": round(mean["iters_learned"], 4), "unit": "iterations/frame", "n_gpus": 1,
        "steps": len(seeds) * (args.learned_frames - 2), "warmup": 2, "higher_is_better": False,
        "scaling": "none", "vs_baseline": None, "dtype": "bf16 net, f32 pipeline",
        "data": "synthetic (seeded held-out sequences, 5 cm / 3 deg per frame)",
        "config": {"workload": f"cfg5: {len(seeds)} held-out seeds x {args.learned_frames} frames, "
                               f"dense {RES}^3 float, voxel {VOXEL} m",
                   "params": learned.PARAMS.name},
        "plain_iterations_per_frame": round(mean["iters_velocity"], 4),
        "iteration_reduction": round(mean["iteration_reduction"], 4),
        "ate_m": {"velocity": mean["ate_velocity_m"], "learned": mean["ate_learned_m"],
                  "learned_vs_plain_rms": mean["learned_vs_plain_rms_m"],
                  "seeds_tracked_by_plain": len(tracked),
                  "velocity_tracked_seeds": float(np.mean([r["ate_velocity_m"] for r in tracked])) if tracked
                  else None,
                  "learned_tracked_seeds": float(np.mean([r["ate_learned_m"] for r in tracked])) if tracked
                  else None},
        "proposal_used": mean["proposal_used"],
        "start_error_m": {"velocity": mean["start_error_velocity_m"], "proposal": mean["start_error_proposal_m"]},
        "one_step_start_error_m": one_step,
        "frames_per_s": {k: round(v, 2) for k, v in rates.items()},
        "frames_per_s_device": {k: round(v, 2) for k, v in device_rates.items()},
        "net_forward_ms": round(forward_ms, 4),
        "e2e": {"value": round(rates["learned"], 2), "unit": "frames/s", "h2d_bytes_per_step": 2 * 640 * 480 * 2,
                "d2h_bytes_per_step": 0},
        "per_seed": report["per_seed"],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--config", choices=["cfg2", "batch16", "learned", "sparse", "ablations", "gemm", "compare",
                                         "reference_cuda", "integrate"],
                    default="cfg2",
                    help="cfg2: the headline 512^3 workload (default); batch16: 16 sequences batched; "
                         "learned: the learned ICP warm start against constant velocity; sparse: cfg3, "
                         "a 2048^3 sparse domain; ablations: the reference's ablation flags; compare: a "
                         "pipeline set compared every frame; reference_cuda: the reference's own CUDA "
                         "pipeline timed on this GPU beside ours")
    ap.add_argument("--sparse-frames", type=int, default=300)
    ap.add_argument("--gemm-size", type=int, default=8192)
    ap.add_argument("--compare-res", type=int, default=RES)
    ap.add_argument("--learned-seeds", type=int, default=20)
    ap.add_argument("--learned-frames", type=int, default=60)
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        line = run_reference(args, rank)
    elif args.config == "batch16":
        line = run_batch(args) if rank == 0 else None
    elif args.config == "learned":
        line = run_learned(args) if rank == 0 else None
    elif args.config == "sparse":
        line = run_sparse(args) if rank == 0 else None
    elif args.config == "ablations":
        line = run_ablations(args) if rank == 0 else None
    elif args.config == "gemm":
        line = run_gemm(args) if rank == 0 else None
    elif args.config == "compare":
        line = run_compare(args) if rank == 0 else None
    elif args.config == "reference_cuda":
        line = run_reference_cuda(args) if rank == 0 else None
    elif args.config == "integrate":
        line = run_integrate(args) if rank == 0 else None
    else:
        if world > 1:
            import datetime

            import torch
            import torch.distributed as tdist
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
            dist = tdist
        line = run_ours(args, rank, world, dist)
        if dist is not None:
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
