"""Seeded synthetic RGB-D sequences: the frame source of the tests and the bench.

The reference reads TUM RGB-D sequences from disk
(src/kinectfusion/virtual_sensor.cpp:41-147); those datasets are not
available here, so frames are rendered analytically instead.

Scene: a 4 x 3 x 4 m box room (x in [-2, 2], y in [-1.5, 1.5],
z in [-0.5, 3.5]) holding 8 spheres (radius U(0.1, 0.4) m) and 4 axis-aligned
boxes (half extents U(0.1, 0.4) m) whose centres lie U(0.8, 3.0) m ahead of
the start pose.  Every primitive (each wall, sphere and box) gets a uniform
random RGB albedo.

Sensor: pinhole fx = fy = 525, cx = 319.5, cy = 239.5 at 640 x 480, depth in
uint16 at 5000 units/m (rgbd.hpp:15).  Depth noise is Gaussian with
sigma = 0.0012 + 0.0019 (z - 0.4)^2 m; 2 % of the pixels drop to 0; pixels at
depth discontinuities (a 4-neighbour on another primitive more than 5 cm
away in depth) drop to 0; depths outside [0.4, 4.0] m drop to 0.

Trajectory: starts at the identity pose (origin, looking +z); translation and
rotation vector follow seeded sums of sinusoids whose per-frame change is
bounded by `max_step_m` and `max_step_deg`.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

WIDTH = 640
HEIGHT = 480
FX = FY = 525.0
CX = 319.5
CY = 239.5
DEPTH_SCALE = 5000.0

ROOM_MIN = np.array([-2.0, -1.5, -0.5])
ROOM_MAX = np.array([2.0, 1.5, 3.5])


@dataclasses.dataclass
class Scene:
    spheres: np.ndarray  # (n, 4) centre xyz, radius
    boxes: np.ndarray  # (m, 6) min xyz, max xyz
    albedo: np.ndarray  # (6 + n + m, 3) uint8: walls, spheres, boxes


@dataclasses.dataclass
class Sequence:
    scene: Scene
    poses: np.ndarray  # (frames, 4, 4) float64 camera_to_world
    depth: np.ndarray  # (frames, H, W) uint16
    color: np.ndarray  # (frames, H, W) uint32 RGBA8
    intrinsics: tuple  # fx, fy, cx, cy
    seed: int


def make_scene(rng: np.random.Generator) -> Scene:
    spheres = []
    for _ in range(8):
        r = rng.uniform(0.1, 0.4)
        z = rng.uniform(0.8, 3.0)
        x = rng.uniform(-0.5, 0.5) * z
        y = rng.uniform(-0.35, 0.35) * z
        c = np.clip([x, y, z], ROOM_MIN + r + 0.05, ROOM_MAX - r - 0.05)
        spheres.append([c[0], c[1], c[2], r])
    boxes = []
    for _ in range(4):
        h = rng.uniform(0.1, 0.4, size=3)
        z = rng.uniform(0.8, 3.0)
        x = rng.uniform(-0.5, 0.5) * z
        y = rng.uniform(-0.35, 0.35) * z
        c = np.clip([x, y, z], ROOM_MIN + h + 0.05, ROOM_MAX - h - 0.05)
        boxes.append(np.concatenate([c - h, c + h]))
    albedo = rng.integers(0, 256, size=(6 + 8 + 4, 3), dtype=np.int64).astype(np.uint8)
    return Scene(np.array(spheres), np.array(boxes), albedo)


def _rotation_from_vector(w: np.ndarray) -> np.ndarray:
    angle = float(np.linalg.norm(w))
    if angle < 1e-15:
        return np.eye(3)
    k = w / angle
    kx = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    return np.eye(3) + math.sin(angle) * kx + (1 - math.cos(angle)) * (kx @ kx)


def make_trajectory(rng: np.random.Generator, frames: int, max_step_m: float,
                    max_step_deg: float) -> np.ndarray:
    omega_t = rng.uniform(0.05, 0.2, size=3)
    phase_t = rng.uniform(0, 2 * math.pi, size=3)
    amp_t = rng.uniform(0.5, 1.0, size=3) * max_step_m / (math.sqrt(3) * omega_t)
    omega_r = rng.uniform(0.05, 0.2, size=3)
    phase_r = rng.uniform(0, 2 * math.pi, size=3)
    amp_r = rng.uniform(0.5, 1.0, size=3) * math.radians(max_step_deg) / (math.sqrt(3) * omega_r)
    poses = np.zeros((frames, 4, 4))
    for k in range(frames):
        t = amp_t * (np.sin(omega_t * k + phase_t) - np.sin(phase_t))
        w = amp_r * (np.sin(omega_r * k + phase_r) - np.sin(phase_r))
        poses[k, :3, :3] = _rotation_from_vector(w)
        poses[k, :3, 3] = t
        poses[k, 3, 3] = 1.0
    return poses


def _render(scene: Scene, pose: np.ndarray):
    """Nearest hit per pixel: camera-frame depth (z) and primitive id."""
    u, v = np.meshgrid(np.arange(WIDTH, dtype=np.float64), np.arange(HEIGHT, dtype=np.float64))
    d_cam = np.stack([(u - CX) / FX, (v - CY) / FY, np.ones_like(u)], axis=-1)
    rot = pose[:3, :3]
    origin = pose[:3, 3]
    d = d_cam @ rot.T  # world direction; t along d == camera z
    best_t = np.full(u.shape, np.inf)
    best_id = np.full(u.shape, -1, dtype=np.int64)

    def take(t, pid):
        nonlocal best_t, best_id
        hit = (t > 1e-9) & (t < best_t)
        best_t = np.where(hit, t, best_t)
        best_id = np.where(hit, pid, best_id)

    # Room walls from the inside: the exit plane on each axis.
    with np.errstate(divide="ignore", invalid="ignore"):
        for axis in range(3):
            da = d[..., axis]
            t_hi = (ROOM_MAX[axis] - origin[axis]) / da
            t_lo = (ROOM_MIN[axis] - origin[axis]) / da
            take(np.where(da > 0, t_hi, np.inf), 2 * axis + 1)
            take(np.where(da < 0, t_lo, np.inf), 2 * axis)
        for i, (cx, cy, cz, r) in enumerate(scene.spheres):
            oc = origin - np.array([cx, cy, cz])
            a = np.einsum("...i,...i->...", d, d)
            b = 2.0 * (d @ oc)
            c = float(oc @ oc) - r * r
            disc = b * b - 4 * a * c
            sq = np.sqrt(np.maximum(disc, 0.0))
            t0 = (-b - sq) / (2 * a)
            take(np.where(disc >= 0, t0, np.inf), 6 + i)
        for j, box in enumerate(scene.boxes):
            lo, hi = box[:3], box[3:]
            t1 = (lo - origin) / d
            t2 = (hi - origin) / d
            tmin = np.max(np.minimum(t1, t2), axis=-1)
            tmax = np.min(np.maximum(t1, t2), axis=-1)
            ok = (tmax >= tmin) & (tmax > 0)
            take(np.where(ok, tmin, np.inf), 6 + 8 + j)
    return best_t, best_id


def render_frame(scene: Scene, pose: np.ndarray, rng: np.random.Generator):
    z, pid = _render(scene, pose)
    sigma = 0.0012 + 0.0019 * (z - 0.4) ** 2
    noisy = z + rng.standard_normal(z.shape) * sigma
    # Depth discontinuities: a 4-neighbour on another primitive > 5 cm away.
    disc = np.zeros(z.shape, dtype=bool)
    for dy, dx in ((0, 1), (0, -1), (1, 0), (-1, 0)):
        zn = np.roll(z, (dy, dx), axis=(0, 1))
        pn = np.roll(pid, (dy, dx), axis=(0, 1))
        disc |= (pn != pid) & (np.abs(zn - z) > 0.05)
    drop = rng.random(z.shape) < 0.02
    valid = np.isfinite(noisy) & (noisy >= 0.4) & (noisy <= 4.0) & ~disc & ~drop
    raw = np.where(valid, np.rint(noisy * DEPTH_SCALE), 0).astype(np.uint16)
    alb = scene.albedo[np.clip(pid, 0, None)].astype(np.uint32)
    color = alb[..., 0] | (alb[..., 1] << 8) | (alb[..., 2] << 16) | (np.uint32(255) << 24)
    return raw, color.astype(np.uint32)


def make_sequence(seed: int, frames: int, max_step_m: float = 0.01,
                  max_step_deg: float = 0.5) -> Sequence:
    """A seeded sequence (1 cm / 0.5 deg of camera motion per frame by default)."""
    rng = np.random.default_rng(seed)
    scene = make_scene(rng)
    poses = make_trajectory(rng, frames, max_step_m, max_step_deg)
    depth = np.zeros((frames, HEIGHT, WIDTH), dtype=np.uint16)
    color = np.zeros((frames, HEIGHT, WIDTH), dtype=np.uint32)
    for k in range(frames):
        depth[k], color[k] = render_frame(scene, poses[k], rng)
    return Sequence(scene, poses, depth, color, (FX, FY, CX, CY), seed)


def make_sequence_device(seed: int, frames: int, max_step_m: float = 0.01, max_step_deg: float = 0.5,
                         device: str = "cuda") -> Sequence:
    """make_sequence with the ray casting done by torch on `device` (float64):
    the same scene, trajectory and noise draws (the random stream is consumed
    in the same order), for the long training runs where the numpy renderer
    would dominate.  A depth may differ from make_sequence's by one unit where
    the device rounds a float64 operation differently; colour is not rendered
    (zeros)."""
    import torch

    rng = np.random.default_rng(seed)
    scene = make_scene(rng)
    poses = make_trajectory(rng, frames, max_step_m, max_step_deg)
    depth = np.zeros((frames, HEIGHT, WIDTH), dtype=np.uint16)
    dev = torch.device(device)
    u, v = torch.meshgrid(torch.arange(WIDTH, dtype=torch.float64, device=dev),
                          torch.arange(HEIGHT, dtype=torch.float64, device=dev), indexing="xy")
    d_cam = torch.stack([(u - CX) / FX, (v - CY) / FY, torch.ones_like(u)], dim=-1)
    spheres = torch.tensor(scene.spheres, dtype=torch.float64, device=dev)
    boxes = torch.tensor(scene.boxes, dtype=torch.float64, device=dev)
    for k in range(frames):
        z, pid = _render_torch(d_cam, spheres, boxes, torch.tensor(poses[k], dtype=torch.float64, device=dev))
        sigma = 0.0012 + 0.0019 * (z - 0.4) ** 2
        noise = torch.from_numpy(rng.standard_normal((HEIGHT, WIDTH))).to(dev)
        noisy = z + noise * sigma
        disc = torch.zeros_like(z, dtype=torch.bool)
        for dy, dx in ((0, 1), (0, -1), (1, 0), (-1, 0)):
            zn = torch.roll(z, (dy, dx), dims=(0, 1))
            pn = torch.roll(pid, (dy, dx), dims=(0, 1))
            disc |= (pn != pid) & ((zn - z).abs() > 0.05)
        drop = torch.from_numpy(rng.random((HEIGHT, WIDTH)) < 0.02).to(dev)
        valid = torch.isfinite(noisy) & (noisy >= 0.4) & (noisy <= 4.0) & ~disc & ~drop
        raw = torch.where(valid, torch.round(noisy * DEPTH_SCALE), torch.zeros_like(noisy))
        depth[k] = raw.to(torch.int32).cpu().numpy().astype(np.uint16)
    color = np.zeros((frames, HEIGHT, WIDTH), dtype=np.uint32)
    return Sequence(scene, poses, depth, color, (FX, FY, CX, CY), seed)


def _render_torch(d_cam, spheres, boxes, pose):
    """_render in torch: the nearest hit per pixel (camera z, primitive id)."""
    import torch

    rot = pose[:3, :3]
    origin = pose[:3, 3]
    d = d_cam @ rot.T
    inf = torch.full(d.shape[:2], math.inf, dtype=torch.float64, device=d.device)
    best_t = inf.clone()
    best_id = torch.full(d.shape[:2], -1, dtype=torch.int64, device=d.device)

    def take(t, pid):
        nonlocal best_t, best_id
        hit = (t > 1e-9) & (t < best_t)
        best_t = torch.where(hit, t, best_t)
        best_id = torch.where(hit, torch.full_like(best_id, pid), best_id)

    for axis in range(3):
        da = d[..., axis]
        t_hi = (float(ROOM_MAX[axis]) - origin[axis]) / da
        t_lo = (float(ROOM_MIN[axis]) - origin[axis]) / da
        take(torch.where(da > 0, t_hi, inf), 2 * axis + 1)
        take(torch.where(da < 0, t_lo, inf), 2 * axis)
    a = (d * d).sum(-1)
    for i in range(spheres.shape[0]):
        oc = origin - spheres[i, :3]
        r = spheres[i, 3]
        b = 2.0 * (d @ oc)
        c = (oc @ oc) - r * r
        disc = b * b - 4 * a * c
        sq = torch.sqrt(torch.clamp(disc, min=0.0))
        t0 = (-b - sq) / (2 * a)
        take(torch.where(disc >= 0, t0, inf), 6 + i)
    for j in range(boxes.shape[0]):
        lo, hi = boxes[j, :3], boxes[j, 3:]
        t1 = (lo - origin) / d
        t2 = (hi - origin) / d
        tmin = torch.minimum(t1, t2).max(-1).values
        tmax = torch.maximum(t1, t2).min(-1).values
        ok = (tmax >= tmin) & (tmax > 0)
        take(torch.where(ok, tmin, inf), 6 + spheres.shape[0] + j)
    return best_t, best_id


def tum_trajectory(poses: np.ndarray, fps: float = 30.0) -> str:
    """TUM format lines 'timestamp tx ty tz qx qy qz qw' (reconstruction.cpp:362-391)."""
    lines = []
    for k, p in enumerate(poses):
        q = _quaternion(p[:3, :3])
        t = p[:3, 3]
        lines.append(f"{k / fps:.6f} {t[0]:.9f} {t[1]:.9f} {t[2]:.9f} "
                     f"{q[0]:.9f} {q[1]:.9f} {q[2]:.9f} {q[3]:.9f}")
    return "\n".join(lines) + "\n"


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


def ate_rmse(estimated: np.ndarray, ground_truth: np.ndarray) -> dict:
    """Translational ATE after rigid (no scale) Umeyama alignment
    (src/app/trajectory_eval.cpp:77-128; frames are associated by index)."""
    p = estimated[:, :3, 3]
    q = ground_truth[:, :3, 3]
    mp, mq = p.mean(0), q.mean(0)
    cov = (q - mq).T @ (p - mp) / len(p)
    u, _, vt = np.linalg.svd(cov)
    s = np.eye(3)
    if np.linalg.det(u) * np.linalg.det(vt) < 0:
        s[2, 2] = -1
    rot = u @ s @ vt
    trans = mq - rot @ mp
    aligned = p @ rot.T + trans
    err = np.linalg.norm(aligned - q, axis=1)
    return {"pairs": len(err), "rmse": float(np.sqrt(np.mean(err ** 2))),
            "mean": float(err.mean()), "median": float(np.median(err)), "max": float(err.max())}
