"""The block culling of the full-sweep integration is conservative: no voxel
that the reference's full sweep fuses lies in a block the culling drops.

A float32 numpy restatement of cull_blocks_kernel (kf_integrate.cu: the
projections of the block's corner voxels, the depth-tile pyramid of 8x8
tiles and 2x2 maxima, the finest level whose tiles cover the projected
rectangle with at most 4x4 texels, the test zmin <= (max depth + truncation)
/ (1 - 2/f) + 1e-3) is checked against the oracle's full sweep (which visits
every voxel) on seeded frames, voxel by voxel, on the CPU.  The device
parity tests check the kernel's own output against the oracle bit for bit on
their frames; this test covers the bound itself on more poses, with and
without distance-scaled truncation."""

import numpy as np
import pytest

import kf_oracle as ko
from kinectfusion_b200 import abi, synthetic

f32 = np.float32
K = abi.Intrinsics(synthetic.FX, synthetic.FY, synthetic.CX, synthetic.CY)
TILE = 8


def _tile_pyramid(depth_m):
    h, w = depth_m.shape
    th, tw = -(-h // TILE), -(-w // TILE)
    padded = np.zeros((th * TILE, tw * TILE), f32)
    padded[:h, :w] = np.nan_to_num(depth_m, nan=0.0)
    levels = [padded.reshape(th, TILE, tw, TILE).max(axis=(1, 3))]
    while levels[-1].shape != (1, 1):
        t = levels[-1]
        h2, w2 = -(-t.shape[0] // 2), -(-t.shape[1] // 2)
        p = np.zeros((h2 * 2, w2 * 2), f32)
        p[:t.shape[0], :t.shape[1]] = t
        levels.append(p.reshape(h2, 2, w2, 2).max(axis=(1, 3)))
        if len(levels) == 12:
            break
    return levels


def _kept_blocks(res, vs, origin, trunc, w2c, depth_m, o, drop_truncation=False):
    rx = ry = rz = res
    b = res // 8
    tiles = _tile_pyramid(depth_m)
    h, w = depth_m.shape
    R = np.array(w2c.r, f32).reshape(3, 3)
    t = np.array(w2c.t, f32)
    org = np.array(origin, f32)
    slack = f32(1.0) / (f32(1.0) - f32(2.0) / f32(min(K.fx, K.fy)))
    kept = np.zeros(b ** 3, bool)
    for block in range(b ** 3):
        bxi, byi, bzi = block % b, (block // b) % b, block // (b * b)
        lo = np.array([bxi * 8, byi * 8, bzi * 8], f32) + f32(0.5)
        hi = np.array([min(bxi * 8 + 8, rx) - 1, min(byi * 8 + 8, ry) - 1, min(bzi * 8 + 8, rz) - 1], f32) + f32(0.5)
        zs, us, vs_ = [], [], []
        for c in range(8):
            corner = np.where([c & 1, c & 2, c & 4], hi, lo).astype(f32)
            wpt = org + corner * f32(vs)
            p = ((R[:, 0] * wpt[0] + R[:, 1] * wpt[1]) + R[:, 2] * wpt[2]) + t
            zs.append(p[2])
            if p[2] > f32(1e-4):
                us.append((f32(K.fx) * p[0]) / p[2] + f32(K.cx))
                vs_.append((f32(K.fy) * p[1]) / p[2] + f32(K.cy))
        zmin, zmax = min(zs), max(zs)
        if not zmax > 0:
            continue
        if zmin <= f32(1e-4):
            kept[block] = True
            continue
        umin, umax, vmin, vmax = min(us), max(us), min(vs_), max(vs_)
        if not (umax >= -2 and vmax >= -2 and umin <= w + 1 and vmin <= h + 1):
            continue
        u0, u1 = max(0, int(np.floor(umin - 1.5))), min(w - 1, int(np.ceil(umax + 1.5)))
        v0, v1 = max(0, int(np.floor(vmin - 1.5))), min(h - 1, int(np.ceil(vmax + 1.5)))
        if u0 > u1 or v0 > v1:
            continue
        tx0, tx1, ty0, ty1, level = u0 // TILE, u1 // TILE, v0 // TILE, v1 // TILE, 0
        while level + 1 < len(tiles) and (tx1 - tx0 > 3 or ty1 - ty0 > 3):
            tx0, tx1, ty0, ty1, level = tx0 >> 1, tx1 >> 1, ty0 >> 1, ty1 >> 1, level + 1
        maxd = tiles[level][ty0:ty1 + 1, tx0:tx1 + 1].max()
        if maxd > 0:
            tr = f32(trunc) + f32(o.truncation_distance_scale) * maxd if o.distance_scaled_truncation else f32(trunc)
            if drop_truncation:  # a planted mistake: the bound without the truncation band
                tr = f32(0.0)
            kept[block] = zmin <= (maxd + tr) * slack + f32(1e-3)
    return kept


@pytest.mark.parametrize("distance_scaled", [0, 1])
def test_block_culling_keeps_every_fused_voxel(distance_scaled):
    res, vs, origin, trunc = 128, 0.02, (-1.28, -1.28, -0.5), 0.05
    o = ko.integration_options(distance_scaled_truncation=distance_scaled)
    seq = synthetic.make_sequence(seed=21, frames=4)
    for frame in (0, 3):
        raw = seq.depth[frame]
        normals = ko.pyramid(raw, K, ko.depth_options())[0]["normals"]
        w2c = ko.rigid_inverse(abi.rigid_from_matrix(seq.poses[frame]))
        vol = ko.OracleVolume(res, vs, origin, trunc)
        ko.integrate(vol, raw, K, w2c, o, abi.KF_RULE_ANGLE_WEIGHTED, normals_map=normals, threads=8)
        fused = (vol.voxels[:, 1] > 0).reshape(res, res, res)  # (z, y, x)
        fused_blocks = fused.reshape(res // 8, 8, res // 8, 8, res // 8, 8).any(axis=(1, 3, 5)).reshape(-1)
        depth_m = raw.astype(f32) / f32(o.depth_scale)
        depth_m[(depth_m < f32(o.min_depth)) | (depth_m > f32(o.max_depth))] = np.nan
        kept = _kept_blocks(res, vs, origin, trunc, w2c, depth_m, o)
        assert fused_blocks.sum() > 200
        assert not (fused_blocks & ~kept).any(), np.nonzero(fused_blocks & ~kept)[0][:10]
        assert kept.sum() < 0.9 * kept.size  # the culling drops blocks at all
    # the check has teeth: a bound without the truncation band drops fused blocks
    wrong = _kept_blocks(res, vs, origin, trunc, w2c, depth_m, o, drop_truncation=True)
    assert (fused_blocks & ~wrong).any()
