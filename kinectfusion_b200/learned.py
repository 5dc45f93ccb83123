"""The learned ICP warm start over the C ABI (kf_learner_*, kf_warm_start_*).

The reference starts ICP at the previous frame's pose
(src/app/reconstruction.cpp:221-223).  Here the plain path starts it at the
constant-velocity prediction, and the learned path lets a bf16 CNN (trained
on the tensor cores by this library's own forward and backward kernels)
correct that prediction, keeping the constant-velocity start whenever the
proposal's point-to-plane residual is higher.

Training data comes from the plain pipeline itself: for every frame of a
seeded synthetic sequence the net input is built against the model as it
stands before the frame (rendered at the constant-velocity pose and at
perturbations of it), and the target is the twist from that render pose to
the pose plain ICP then tracks.

Device memory for datasets and batches is held in torch tensors (plumbing);
all arithmetic runs in libkf_b200.so.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import math
import pathlib

import numpy as np

from . import abi, synthetic
from .pipeline import Pipeline, Reconstruction, _check, lib, pipeline_config

TWIST_SCALE = abi.WARM_START_TWIST_SCALE
NET_H, NET_W = 60, 80
# The trained parameters shipped with the package: `python -m
# kinectfusion_b200.learned train` over seeds 0-399 (25 frames each, 5 cm / 3
# degree steps, 512^3 dense float), 8000 Adam steps of 64.
PARAMS = pathlib.Path(__file__).resolve().parent / "warm_start_params.npy"


def _torch():
    import torch
    return torch


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


# ---- SE(3) helpers (the decoupled twist of kf_warm_start_propose) ---------------------
def so3_exp(w) -> np.ndarray:
    w = np.asarray(w, dtype=np.float64)
    th = float(np.linalg.norm(w))
    if th < 1e-15:
        return np.eye(3)
    k = w / th
    kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + math.sin(th) * kx + (1 - math.cos(th)) * (kx @ kx)


def so3_log(r) -> np.ndarray:
    r = np.asarray(r, dtype=np.float64)
    c = min(1.0, max(-1.0, (np.trace(r) - 1.0) / 2.0))
    th = math.acos(c)
    v = np.array([r[2, 1] - r[1, 2], r[0, 2] - r[2, 0], r[1, 0] - r[0, 1]])
    if th < 1e-8:
        return 0.5 * v
    return th / (2.0 * math.sin(th)) * v


def apply_twist(pose, twist) -> np.ndarray:
    """pose * exp(twist): translation added in the pose's frame, rotation by
    Rodrigues (the convention of KF_WARM_START_TWIST_SCALE outputs)."""
    pose = np.asarray(pose, dtype=np.float64)
    d = np.eye(4)
    d[:3, :3] = so3_exp(twist[3:])
    d[:3, 3] = twist[:3]
    return pose @ d


def twist_between(a, b) -> np.ndarray:
    """The twist t with apply_twist(a, t) == b."""
    d = np.linalg.inv(np.asarray(a, dtype=np.float64)) @ np.asarray(b, dtype=np.float64)
    return np.concatenate([d[:3, 3], so3_log(d[:3, :3])])


def constant_velocity(trajectory) -> np.ndarray:
    """T[-1] * (T[-2]^-1 T[-1]): the last motion repeated (the last pose when
    fewer than two are known), in double with the inverse of the float pose
    as stored (kf_warm_start_enqueue computes the same on the device)."""
    last = np.asarray(trajectory[-1], dtype=np.float64)
    if len(trajectory) < 2:
        return last
    prev = np.asarray(trajectory[-2], dtype=np.float64)
    return last @ (np.linalg.inv(prev) @ last)


# ---- the network -------------------------------------------------------------------
class Learner:
    """kf_learner: parameters, Adam state and activations on the device."""

    def __init__(self, batch_capacity: int = 64, seed: int = 0):
        self.handle = C.c_void_p()
        _check(lib().kf_learner_create(batch_capacity, seed, C.byref(self.handle)))
        self.capacity = batch_capacity
        n = C.c_uint64()
        _check(lib().kf_learner_param_count(self.handle, C.byref(n)))
        self.param_count = n.value

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                lib().kf_learner_destroy(self.handle)
                self.handle = C.c_void_p()
        except Exception:  # interpreter shutdown: the modules are gone
            pass

    def params(self) -> np.ndarray:
        p = np.empty(self.param_count, dtype=np.float32)
        _check(lib().kf_learner_get_params(self.handle, p.ctypes.data_as(C.c_void_p)))
        return p

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.param_count:
            raise ValueError(f"expected {self.param_count} parameters, got {p.size}")
        _check(lib().kf_learner_set_params(self.handle, p.ctypes.data_as(C.c_void_p)))

    def forward(self, inputs):
        """inputs: a CUDA bf16 tensor [B, 60, 80, 2] (B a multiple of 8)."""
        torch = _torch()
        out = torch.empty((inputs.shape[0], 6), dtype=torch.float32, device=inputs.device)
        _check(lib().kf_learner_forward(self.handle, C.c_void_p(inputs.data_ptr()), inputs.shape[0],
                                        C.c_void_p(out.data_ptr()), _stream()))
        return out

    def gradients(self, inputs, targets):
        """(flat fp32 gradient, loss) of the batch-mean squared error."""
        g = np.empty(self.param_count, dtype=np.float32)
        loss = C.c_float()
        _check(lib().kf_learner_gradients(self.handle, C.c_void_p(inputs.data_ptr()),
                                          C.c_void_p(targets.data_ptr()), inputs.shape[0],
                                          g.ctypes.data_as(C.c_void_p), C.byref(loss), _stream()))
        return g, float(loss.value)

    def train_step(self, inputs, targets, lr: float, loss_out=None) -> None:
        """One Adam step; loss_out (a CUDA float tensor element) receives the loss."""
        _check(lib().kf_learner_train_step(self.handle, C.c_void_p(inputs.data_ptr()),
                                           C.c_void_p(targets.data_ptr()), inputs.shape[0], float(lr),
                                           None if loss_out is None else C.c_void_p(loss_out.data_ptr()),
                                           _stream()))

    def timed_out(self) -> bool:
        e = C.c_int32()
        _check(lib().kf_learner_error(self.handle, C.byref(e)))
        return bool(e.value)

    def save(self, path) -> None:
        np.save(path, self.params())

    def load(self, path) -> None:
        self.set_params(np.load(path))


class WarmStart:
    """kf_warm_start: builds net inputs and proposes start poses."""

    def __init__(self, depth_scale: float = synthetic.DEPTH_SCALE):
        self.handle = C.c_void_p()
        _check(lib().kf_warm_start_create(depth_scale, C.byref(self.handle)))

    def __del__(self):
        try:
            if getattr(self, "handle", None) and self.handle.value:
                lib().kf_warm_start_destroy(self.handle)
                self.handle = C.c_void_p()
        except Exception:  # interpreter shutdown: the modules are gone
            pass

    def input(self, pipeline: Pipeline, depth: np.ndarray, intrinsics: abi.Intrinsics, render_pose, out) -> None:
        """The net input for `depth` against the model rendered at
        render_pose, into `out` (a contiguous CUDA bf16 tensor of 9600)."""
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        pose = abi.rigid_from_matrix(render_pose)
        _check(lib().kf_warm_start_input(self.handle, pipeline.handle, depth.ctypes.data_as(C.c_void_p),
                                         depth.shape[1], depth.shape[0], intrinsics, abi.KF_MEMORY_HOST,
                                         C.byref(pose), C.c_void_p(out.data_ptr())))

    def propose(self, learner: Learner, pipeline: Pipeline, depth: np.ndarray, intrinsics: abi.Intrinsics,
                predicted) -> abi.WarmStartResult:
        depth = np.ascontiguousarray(depth, dtype=np.uint16)
        pose = abi.rigid_from_matrix(predicted)
        res = abi.WarmStartResult()
        _check(lib().kf_warm_start_propose(self.handle, learner.handle, pipeline.handle,
                                           depth.ctypes.data_as(C.c_void_p), depth.shape[1], depth.shape[0],
                                           intrinsics, abi.KF_MEMORY_HOST, C.byref(pose), C.byref(res)))
        return res


# ---- the tracking loop with a chosen start ---------------------------------------------
class WarmStartedReconstruction(Reconstruction):
    """Reconstruction whose frames start ICP from `start`:
    "previous" (the reference's loop), "velocity" (constant velocity) or
    "learned" (the net's proposal with the constant-velocity fallback)."""

    def __init__(self, pipeline: Pipeline, intrinsics: abi.Intrinsics, start: str = "velocity",
                 learner: Learner | None = None, warm: WarmStart | None = None, **kw):
        super().__init__(pipeline, intrinsics, **kw)
        if start not in ("previous", "velocity", "learned"):
            raise ValueError(f"unknown start {start!r}")
        if start == "learned" and learner is None:
            raise ValueError("the learned start needs a Learner")
        self.start = start
        self.learner = learner
        self.warm = warm if warm is not None or start != "learned" else WarmStart()
        self.proposals = []  # per frame: WarmStartResult or None
        self.starts = []

    def prediction(self) -> np.ndarray:
        """The constant-velocity pose for the next frame; the last pose when
        the last frame lost track (its motion says nothing then)."""
        if self.results and not self.results[-1].tracked:
            return np.asarray(self.trajectory[-1], dtype=np.float64)
        return constant_velocity(self.trajectory)

    def process(self, depth, color=None) -> abi.FrameResult:
        proposal = None
        if self.frames >= 1 and self.start != "previous":
            start = self.prediction()
            if self.start == "learned" and self.frames >= 2 and self.results[-1].tracked:
                proposal = self.warm.propose(self.learner, self.pipeline, depth, self.intrinsics, start)
                start = abi.matrix_from_rigid(proposal.start).astype(np.float64)
            self.pose = abi.rigid_from_matrix(start)
        self.starts.append(abi.matrix_from_rigid(self.pose))
        self.proposals.append(proposal)
        return super().process(depth, color)


class AsyncLearnedLoop:
    """The learned loop with no host round trip per frame: each tracked frame
    is kf_warm_start_enqueue (prediction, net, fallback test, start pose into
    the tracker, all on the device) then kf_frame_enqueue.  Frame 1 starts
    at frame 0's pose (no velocity yet, no net); later frames use the net
    (with use_net=False: the constant-velocity start alone, on the device).
    Depth frames may be host arrays or device addresses (ints).  Frames that
    reach the device in HBM need no synchronisation until a result is read.""" 

    def __init__(self, pipeline: Pipeline, intrinsics: abi.Intrinsics, learner: Learner | None,
                 warm: WarmStart | None = None, iterations=(10, 5, 4, 4), use_net: bool = True):
        from .pipeline import ProjectiveIcpTracker, PyramidSource
        self.pipeline = pipeline
        self.intrinsics = intrinsics
        self.learner = learner
        self.warm = warm if warm is not None else WarmStart()
        self.pyramid = PyramidSource()
        self.tracker = ProjectiveIcpTracker()
        self.iterations = (C.c_uint32 * 4)(*iterations)
        self.use_net = use_net and learner is not None
        self.frames = 0
        _check(lib().kf_warm_start_reset(self.warm.handle))

    def enqueue(self, depth) -> None:
        if isinstance(depth, int):
            ptr, memory = C.c_void_p(depth), abi.KF_MEMORY_DEVICE
            self._keep = None
        else:
            self._keep = np.ascontiguousarray(depth, dtype=np.uint16)
            ptr, memory = self._keep.ctypes.data_as(C.c_void_p), abi.KF_MEMORY_HOST
        if self.frames >= 1:
            use_net = 1 if (self.use_net and self.frames >= 2) else 0
            _check(lib().kf_warm_start_enqueue(self.warm.handle, self.learner.handle if use_net else None,
                                               self.pipeline.handle, self.tracker.handle, ptr, 640, 480,
                                               self.intrinsics, memory, use_net))
        _check(lib().kf_frame_enqueue(self.pipeline.handle, self.pyramid.handle, self.tracker.handle, ptr, None,
                                      640, 480, self.intrinsics, memory, self.iterations,
                                      1 if self.frames == 0 else 0))
        self.frames += 1

    def result(self) -> abi.FrameResult:
        r = abi.FrameResult()
        _check(lib().kf_frame_result_fetch(self.pipeline.handle, C.byref(r)))
        return r

    def proposal(self) -> abi.WarmStartResult:
        r = abi.WarmStartResult()
        _check(lib().kf_warm_start_fetch(self.warm.handle, self.pipeline.handle, C.byref(r)))
        return r


def volume_config(resolution: int = 512, voxel: float = 0.01):
    """A dense float volume over the synthetic room (origin 0.5 m behind the
    start camera), angle-weighted TSDF, no colour."""
    half = 0.5 * resolution * voxel
    return pipeline_config(resolution, voxel, (-half, -half, -0.5), 0.05, color=abi.KF_COLOR_NONE)


def intrinsics640() -> abi.Intrinsics:
    return abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)


# ---- data ---------------------------------------------------------------------------
@dataclasses.dataclass
class Dataset:
    inputs: object   # CUDA bf16 [N, 60, 80, 2]
    targets: object  # CUDA fp32 [N, 6] (scaled twists)
    seeds: list
    iterations: list  # plain-path ICP iterations per frame, per seed


def generate(seeds, frames: int, *, max_step_m: float = 0.05, max_step_deg: float = 3.0, resolution: int = 512,
             voxel: float = 0.01, perturbations: int = 3, perturb_m: float = 0.02, perturb_deg: float = 2.0,
             rng_seed: int = 0, pipeline: Pipeline | None = None) -> Dataset:
    """Runs the plain (constant-velocity) pipeline over each seeded sequence
    and records, for every frame from the third on, the net input against
    the model before the frame, rendered at the constant-velocity pose and at
    `perturbations` random perturbations of it (uniform in a ball of
    perturb_m / perturb_deg), with the twist from each render pose to the
    tracked pose as the target."""
    torch = _torch()
    rng = np.random.default_rng(rng_seed)
    k = intrinsics640()
    per_seed = max(0, frames - 2) * (1 + perturbations)
    n = len(seeds) * per_seed
    n_alloc = max(8, (n + 7) // 8 * 8)
    inputs = torch.zeros((n_alloc, NET_H, NET_W, 2), dtype=torch.bfloat16, device="cuda")
    targets = torch.zeros((n_alloc, 6), dtype=torch.float32, device="cuda")
    host_targets = np.zeros((n_alloc, 6), dtype=np.float32)
    own = pipeline is None
    gpu = Pipeline(volume_config(resolution, voxel)) if own else pipeline
    warm = WarmStart()
    iters = []
    idx = 0
    for seed in seeds:
        seq = synthetic.make_sequence_device(seed, frames, max_step_m, max_step_deg)
        gpu.reset()
        loop = WarmStartedReconstruction(gpu, k, start="velocity")
        seed_iters = []
        for f in range(frames):
            pending = []
            if f >= 2:
                pred = constant_velocity(loop.trajectory)
                renders = [pred]
                for _ in range(perturbations):
                    renders.append(apply_twist(pred, _ball_twist(rng, perturb_m, math.radians(perturb_deg))))
                torch.cuda.synchronize()
                for pose in renders:
                    warm.input(gpu, seq.depth[f], k, pose, inputs[idx])
                    pending.append((idx, pose))
                    idx += 1
            result = loop.process(seq.depth[f])
            tracked = np.asarray(loop.trajectory[-1], dtype=np.float64)
            for i, pose in pending:
                host_targets[i] = twist_between(pose, tracked) * TWIST_SCALE
            if f >= 2:
                seed_iters.append(int(sum(result.iterations[:3])))
        iters.append(seed_iters)
    torch.cuda.synchronize()  # the device, so the pipeline's stream too
    targets.copy_(torch.from_numpy(host_targets))
    return Dataset(inputs[:n], targets[:n], list(seeds), iters)


def _ball_twist(rng, max_t, max_r):
    def ball(radius):
        v = rng.normal(size=3)
        v /= max(np.linalg.norm(v), 1e-12)
        return v * radius * rng.random() ** (1.0 / 3.0)
    return np.concatenate([ball(max_t), ball(max_r)])


# ---- training -----------------------------------------------------------------------
# Mirroring the camera's x (y) axis flips the 80x60 maps left-right (up-down;
# the principal point sits at the image centre) and negates these twist
# components: translation x (y) and the rotation about the other two axes.
_FLIP_SIGNS = {2: (-1.0, 1.0, 1.0, 1.0, -1.0, -1.0), 1: (1.0, -1.0, 1.0, -1.0, 1.0, -1.0)}


def train(learner: Learner, data: Dataset, steps: int, *, batch: int = 64, lr: float = 1e-3,
          final_lr: float = 1e-5, seed: int = 0, log_every: int = 0, validation: Dataset | None = None,
          mirror: bool = True) -> list:
    """Adam over shuffled minibatches with a cosine learning-rate decay; with
    `mirror`, each batch is flipped left-right and/or up-down at random (the
    twists follow).  Returns [(step, mean training loss over the last
    log_every steps, validation loss or None)]."""
    torch = _torch()
    if batch % 8 or batch > learner.capacity:
        raise ValueError("batch must be a multiple of 8 within the learner's capacity")
    n = data.inputs.shape[0]
    if n < batch:
        raise ValueError("dataset smaller than one batch")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    losses = torch.zeros(steps, dtype=torch.float32, device="cuda")
    bx = torch.empty((batch, NET_H, NET_W, 2), dtype=torch.bfloat16, device="cuda")
    by = torch.empty((batch, 6), dtype=torch.float32, device="cuda")
    perm = torch.randperm(n, generator=gen, device="cuda")
    pos = 0
    val_losses = {}
    rng = np.random.default_rng(seed)
    signs = {d: torch.tensor(v, dtype=torch.float32, device="cuda") for d, v in _FLIP_SIGNS.items()}
    for s in range(steps):
        if pos + batch > n:
            perm = torch.randperm(n, generator=gen, device="cuda")
            pos = 0
        sel = perm[pos:pos + batch]
        pos += batch
        torch.index_select(data.inputs, 0, sel, out=bx)
        torch.index_select(data.targets, 0, sel, out=by)
        if mirror:
            for dim, flip in zip((2, 1), rng.random(2) < 0.5):
                if flip:
                    bx.copy_(torch.flip(bx, dims=(dim,)))
                    by.mul_(signs[dim])
        rate = final_lr + 0.5 * (lr - final_lr) * (1.0 + math.cos(math.pi * s / max(1, steps)))
        learner.train_step(bx, by, rate, losses[s])
        if log_every and validation is not None and (s + 1) % log_every == 0:
            val_losses[s + 1] = validation_loss(learner, validation)
    torch.cuda.synchronize()
    if learner.timed_out():
        raise RuntimeError("a tensor-core wait timed out during training")
    curve = losses.cpu().numpy()
    if not log_every:
        return [(steps, float(curve[-max(1, steps // 10):].mean()), None)]
    return [(s + log_every, float(curve[s:s + log_every].mean()), val_losses.get(s + log_every))
            for s in range(0, steps, log_every)]


def validation_loss(learner: Learner, data: Dataset) -> float:
    torch = _torch()
    n = data.inputs.shape[0] // 8 * 8
    total = 0.0
    for s in range(0, n, learner.capacity):
        e = min(n, s + learner.capacity) // 8 * 8
        if e <= s:
            break
        out = learner.forward(data.inputs[s:e])
        total += float(((out - data.targets[s:e]) ** 2).sum())
    torch.cuda.synchronize()
    return total / max(1, n)


# ---- evaluation ---------------------------------------------------------------------
def evaluate(learner: Learner, seeds, frames: int, *, max_step_m: float = 0.05, max_step_deg: float = 3.0,
             resolution: int = 512, voxel: float = 0.01, pipeline: Pipeline | None = None) -> dict:
    """Plain constant-velocity ICP against the learned start on each seed:
    ICP iterations per frame (frames from the third on), ATE RMSE against the
    ground truth, the learned trajectory's RMS distance to the plain one, how
    often the proposal was taken, and the start error of each start against
    the plain-ICP pose."""
    k = intrinsics640()
    gpu = Pipeline(volume_config(resolution, voxel)) if pipeline is None else pipeline
    warm = WarmStart()
    rows = []
    for seed in seeds:
        seq = synthetic.make_sequence_device(seed, frames, max_step_m, max_step_deg)
        runs = {}
        for mode in ("velocity", "learned"):
            gpu.reset()
            loop = WarmStartedReconstruction(gpu, k, start=mode, learner=learner, warm=warm)
            its = []
            for f in range(frames):
                r = loop.process(seq.depth[f])
                if f >= 2:
                    its.append(int(sum(r.iterations[:3])))
            runs[mode] = (np.array(loop.trajectory, dtype=np.float64), np.array(its), loop)
        plain_traj = runs["velocity"][0]
        learned_loop = runs["learned"][2]
        start_err_cv, start_err_learned, used = [], [], 0
        for f in range(2, frames):
            prop = learned_loop.proposals[f]
            if prop is None:  # the learned loop had lost track: no proposal
                continue
            cv = constant_velocity(list(runs["learned"][0][:f]))
            start_err_cv.append(np.linalg.norm(twist_between(cv, plain_traj[f])[:3]))
            learned_start = apply_twist(cv, np.array(prop.twist, dtype=np.float64))
            start_err_learned.append(np.linalg.norm(twist_between(learned_start, plain_traj[f])[:3]))
            used += int(prop.used_proposal)
        rows.append({
            "seed": seed,
            "iters_velocity": float(runs["velocity"][1].mean()),
            "iters_learned": float(runs["learned"][1].mean()),
            "ate_velocity_m": synthetic.ate_rmse(runs["velocity"][0], seq.poses)["rmse"],
            "ate_learned_m": synthetic.ate_rmse(runs["learned"][0], seq.poses)["rmse"],
            "learned_vs_plain_rms_m": float(np.sqrt(np.mean(np.sum(
                (runs["learned"][0][:, :3, 3] - plain_traj[:, :3, 3]) ** 2, axis=1)))),
            "proposal_used": used / max(1, sum(p is not None for p in learned_loop.proposals[2:])),
            "start_error_velocity_m": float(np.mean(start_err_cv)),
            "start_error_proposal_m": float(np.mean(start_err_learned)),
        })
    summary = {key: float(np.mean([r[key] for r in rows])) for key in rows[0] if key != "seed"}
    summary["iteration_reduction"] = 1.0 - summary["iters_learned"] / max(1e-9, summary["iters_velocity"])
    return {"per_seed": rows, "mean": summary}


def one_step_errors(learner: Learner, seeds, frames: int, *, max_step_m: float = 0.05, max_step_deg: float = 3.0,
                    resolution: int = 512, voxel: float = 0.01, pipeline: Pipeline | None = None) -> dict:
    """The net's gain on one trajectory, free of the loops' divergence: the
    plain constant-velocity loop runs each sequence, and before each frame
    from the third on the net proposes a start from that loop's own state;
    both starts are compared with the pose plain ICP then reaches (mean and
    median translation error, metres), over the frames plain ICP tracks."""
    k = intrinsics640()
    gpu = Pipeline(volume_config(resolution, voxel)) if pipeline is None else pipeline
    warm = WarmStart()
    cv_err, net_err, used = [], [], 0
    for seed in seeds:
        seq = synthetic.make_sequence_device(seed, frames, max_step_m, max_step_deg)
        gpu.reset()
        loop = WarmStartedReconstruction(gpu, k, start="velocity")
        for f in range(frames):
            prop = None
            if f >= 2 and loop.results[-1].tracked:
                cv = loop.prediction()
                prop = warm.propose(learner, gpu, seq.depth[f], k, cv)
            r = loop.process(seq.depth[f])
            if prop is None or not r.tracked:
                continue
            tracked = np.asarray(loop.trajectory[-1], dtype=np.float64)
            cv_err.append(np.linalg.norm(twist_between(cv, tracked)[:3]))
            start = abi.matrix_from_rigid(prop.start).astype(np.float64)
            net_err.append(np.linalg.norm(twist_between(start, tracked)[:3]))
            used += int(prop.used_proposal)
    n = max(1, len(cv_err))
    return {"frames": len(cv_err), "start_error_velocity_m": float(np.mean(cv_err)),
            "start_error_learned_m": float(np.mean(net_err)),
            "median_start_error_velocity_m": float(np.median(cv_err)),
            "median_start_error_learned_m": float(np.median(net_err)), "proposal_used": used / n}


def start_bound(seeds, frames: int, noise_m=(0.0,), *, max_step_m: float = 0.05, max_step_deg: float = 3.0,
                resolution: int = 512, voxel: float = 0.01, pipeline: Pipeline | None = None, seed: int = 0) -> dict:
    """What any warm start can gain: ICP iterations per frame when every frame
    starts at the pose plain ICP reaches for it (perturbed by Gaussian noise
    of `noise_m` metres per axis and noise_m / 2 radians per axis), against
    the constant-velocity start."""
    k = intrinsics640()
    gpu = Pipeline(volume_config(resolution, voxel)) if pipeline is None else pipeline
    rng = np.random.default_rng(seed)
    out = {"velocity": [], **{f"plain_pose+{s}": [] for s in noise_m}}
    for sd in seeds:
        seq = synthetic.make_sequence_device(sd, frames, max_step_m, max_step_deg)
        gpu.reset()
        loop = WarmStartedReconstruction(gpu, k, start="velocity")
        its = []
        for f in range(frames):
            r = loop.process(seq.depth[f])
            if f >= 2:
                its.append(int(sum(r.iterations[:3])))
        out["velocity"].append(float(np.mean(its)))
        plain = np.array(loop.trajectory, dtype=np.float64)
        for s in noise_m:
            gpu.reset()
            loop = Reconstruction(gpu, k)
            its = []
            for f in range(frames):
                if f >= 1:
                    tw = np.concatenate([rng.normal(size=3) * s, rng.normal(size=3) * s / 2])
                    loop.pose = abi.rigid_from_matrix(apply_twist(plain[f], tw))
                r = loop.process(seq.depth[f])
                if f >= 2:
                    its.append(int(sum(r.iterations[:3])))
            out[f"plain_pose+{s}"].append(float(np.mean(its)))
    return {key: float(np.mean(v)) for key, v in out.items()}


def _seed_range(text: str) -> list:
    lo, _, hi = text.partition("-")
    return list(range(int(lo), int(hi or lo) + 1))


def main(argv=None) -> None:
    """python -m kinectfusion_b200.learned train|evaluate|bound ..."""
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser(prog="python -m kinectfusion_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="generate data with the plain pipeline, train, save the parameters")
    t.add_argument("--seeds", default="0-399")
    t.add_argument("--val-seeds", default="900-915")
    t.add_argument("--frames", type=int, default=25)
    t.add_argument("--perturbations", type=int, default=3)
    t.add_argument("--perturb-m", type=float, default=0.008)
    t.add_argument("--perturb-deg", type=float, default=0.6)
    t.add_argument("--steps", type=int, default=8000)
    t.add_argument("--batch", type=int, default=64)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--resolution", type=int, default=512)
    t.add_argument("--out", required=True)
    e = sub.add_parser("evaluate", help="learned vs constant-velocity ICP on held-out seeds")
    e.add_argument("--params", required=True)
    e.add_argument("--seeds", default="5000-5019")
    e.add_argument("--frames", type=int, default=60)
    e.add_argument("--resolution", type=int, default=512)
    b = sub.add_parser("bound", help="iterations from the plain-ICP pose: the most any warm start can save")
    b.add_argument("--seeds", default="5000-5003")
    b.add_argument("--frames", type=int, default=60)
    b.add_argument("--resolution", type=int, default=512)
    for p in (t, e, b):
        p.add_argument("--json", default=None, help="also write the report here")
    a = ap.parse_args(argv)
    gpu = Pipeline(volume_config(a.resolution, 512 * 0.01 / a.resolution))
    t0 = time.time()
    if a.cmd == "train":
        data = generate(_seed_range(a.seeds), a.frames, perturbations=a.perturbations, perturb_m=a.perturb_m,
                        perturb_deg=a.perturb_deg, resolution=a.resolution, pipeline=gpu)
        val = generate(_seed_range(a.val_seeds), a.frames, perturbations=a.perturbations, perturb_m=a.perturb_m,
                       perturb_deg=a.perturb_deg, resolution=a.resolution, pipeline=gpu, rng_seed=1)
        t1 = time.time()
        net = Learner(a.batch, seed=0)
        curve = train(net, data, a.steps, batch=a.batch, lr=a.lr, log_every=max(1, a.steps // 20), validation=val)
        net.save(a.out)
        report = {"samples": int(data.inputs.shape[0]), "validation_samples": int(val.inputs.shape[0]),
                  "generate_s": t1 - t0, "train_s": time.time() - t1, "curve": curve,
                  "plain_iterations_per_frame": float(np.mean([np.mean(i) for i in data.iterations]))}
    elif a.cmd == "evaluate":
        net = Learner(8, seed=0)
        net.load(a.params)
        report = evaluate(net, _seed_range(a.seeds), a.frames, resolution=a.resolution,
                          voxel=512 * 0.01 / a.resolution, pipeline=gpu)
    else:
        report = start_bound(_seed_range(a.seeds), a.frames, (0.0, 0.001, 0.003), resolution=a.resolution,
                             voxel=512 * 0.01 / a.resolution, pipeline=gpu)
    report["seconds"] = time.time() - t0
    text = json.dumps(report, indent=1)
    print(text)
    if a.json:
        with open(a.json, "w") as f:
            f.write(text + "\n")


if __name__ == "__main__":
    main()
