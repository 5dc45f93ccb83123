"""Frame source and output files (CPU only): the native PNG reader and
writer, TUM RGB-D sequence directories, PLY meshes and point clouds, TUM
trajectories."""

import struct
import zlib

import numpy as np
import pytest

from kinectfusion_b200 import abi, tum
from kinectfusion_b200.pipeline import SurfaceMaps


def _png(pixels: np.ndarray, bit_depth: int, color_type: int, filters, palette=None) -> bytes:
    """An independent PNG encoder for the tests: rows filtered with the
    given filter types (cycled), per ISO/IEC 15948."""
    h = pixels.shape[0]
    if bit_depth == 16:
        rows = pixels.astype(">u2").reshape(h, -1).view(np.uint8).reshape(h, -1)
    else:
        rows = pixels.astype(np.uint8).reshape(h, -1)
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[color_type]
    bpp = channels * bit_depth // 8
    raw = bytearray()
    prev = np.zeros(rows.shape[1], dtype=np.int32)
    for y in range(h):
        f = filters[y % len(filters)]
        cur = rows[y].astype(np.int32)
        out = np.zeros_like(cur)
        for x in range(len(cur)):
            a = cur[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            if f == 0:
                pred = 0
            elif f == 1:
                pred = a
            elif f == 2:
                pred = b
            elif f == 3:
                pred = (a + b) // 2
            else:
                p = a + b - c
                pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
                pred = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            out[x] = (cur[x] - pred) & 0xFF
        raw.append(f)
        raw.extend(out.astype(np.uint8).tobytes())
        prev = cur

    def chunk(t, d):
        return struct.pack(">I", len(d)) + t + d + struct.pack(">I", zlib.crc32(t + d) & 0xFFFFFFFF)

    w = pixels.shape[1]
    data = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, bit_depth, color_type, 0, 0, 0))
    if palette is not None:
        data += chunk(b"PLTE", bytes(palette))
    data += chunk(b"IDAT", zlib.compress(bytes(raw))) + chunk(b"IEND", b"")
    return data


def test_depth_png_with_every_filter(tmp_path):
    rng = np.random.default_rng(0)
    depth = rng.integers(0, 65536, size=(7, 9), dtype=np.uint16)
    path = tmp_path / "d.png"
    path.write_bytes(_png(depth, 16, 0, [0, 1, 2, 3, 4]))
    assert tum.png_info(path) == (9, 7, 0, 16)
    np.testing.assert_array_equal(tum.read_depth_png(path), depth)


@pytest.mark.parametrize("color_type,channels", [(2, 3), (6, 4), (0, 1), (4, 2)])
def test_color_png_formats(tmp_path, color_type, channels):
    rng = np.random.default_rng(color_type)
    px = rng.integers(0, 256, size=(5, 6, channels), dtype=np.uint8)
    path = tmp_path / "c.png"
    path.write_bytes(_png(px, 8, color_type, [4, 3, 2, 1, 0]))
    got = tum.read_color_png(path)
    r, g, b, a = (got & 0xFF), (got >> 8) & 0xFF, (got >> 16) & 0xFF, got >> 24
    if channels >= 3:
        np.testing.assert_array_equal(np.stack([r, g, b], -1), px[..., :3])
    else:
        for ch in (r, g, b):
            np.testing.assert_array_equal(ch, px[..., 0])
    expect_a = px[..., -1] if channels in (2, 4) else np.full((5, 6), 255)
    np.testing.assert_array_equal(a, expect_a)


def test_palette_png(tmp_path):
    palette = [10, 20, 30, 40, 50, 60, 70, 80, 90]
    idx = np.array([[0, 1, 2], [2, 1, 0]], dtype=np.uint8)
    path = tmp_path / "p.png"
    path.write_bytes(_png(idx, 8, 3, [1], palette=palette))
    got = tum.read_color_png(path)
    assert got[0, 1] == 40 | (50 << 8) | (60 << 16) | (255 << 24)
    assert got[1, 0] == 70 | (80 << 8) | (90 << 16) | (255 << 24)


def test_writer_round_trips(tmp_path):
    rng = np.random.default_rng(3)
    depth = rng.integers(0, 65536, size=(48, 64), dtype=np.uint16)
    color = rng.integers(0, 2 ** 32, size=(48, 64), dtype=np.uint64).astype(np.uint32)
    tum.write_depth_png(tmp_path / "d.png", depth)
    tum.write_color_png(tmp_path / "c.png", color)
    np.testing.assert_array_equal(tum.read_depth_png(tmp_path / "d.png"), depth)
    np.testing.assert_array_equal(tum.read_color_png(tmp_path / "c.png"), color)
    # the written depth is a standard 16-bit grayscale PNG
    assert tum.png_info(tmp_path / "d.png") == (64, 48, 0, 16)


def test_png_errors(tmp_path):
    bad = tmp_path / "bad.png"
    bad.write_bytes(b"not a png at all")
    with pytest.raises(RuntimeError, match="Not a PNG"):
        tum.read_depth_png(bad)
    gray8 = tmp_path / "g8.png"
    gray8.write_bytes(_png(np.zeros((2, 2), np.uint8), 8, 0, [0]))
    with pytest.raises(RuntimeError, match="16-bit grayscale"):
        tum.read_depth_png(gray8)
    corrupt = bytearray(_png(np.zeros((2, 2), np.uint16), 16, 0, [0]))
    corrupt[40] ^= 0xFF  # inside IDAT: the chunk CRC no longer matches
    (tmp_path / "crc.png").write_bytes(bytes(corrupt))
    with pytest.raises(RuntimeError, match="CRC|Corrupt"):
        tum.read_depth_png(tmp_path / "crc.png")
    with pytest.raises(RuntimeError, match="open"):
        tum.read_depth_png(tmp_path / "missing.png")


def test_tum_sequence_directory(tmp_path):
    rng = np.random.default_rng(4)
    depths = [rng.integers(0, 30000, size=(6, 8), dtype=np.uint16) for _ in range(7)]
    colors = [rng.integers(0, 2 ** 32, size=(6, 8), dtype=np.uint64).astype(np.uint32) for _ in range(7)]
    root = tmp_path / "rgbd_dataset_freiburg3_synthetic"
    tum.write_sequence(root, depths, colors)
    stamps, files = tum.read_index(root / "depth.txt")
    assert len(files) == 7 and stamps[1] == pytest.approx(1 / 30, abs=1e-6)
    for preload in (False, True):
        seq = tum.TumSequence(root, preload=preload, prefetch=3)
        assert len(seq) == 7
        k = seq.intrinsics
        assert (k.fx, k.fy, k.cx, k.cy) == pytest.approx(tum.TUM_DEPTH_INTRINSICS["freiburg3"])
        frames = list(seq)
        assert [f.index for f in frames] == list(range(7))
        for f, d, c in zip(frames, depths, colors):
            np.testing.assert_array_equal(f.depth, d)
            np.testing.assert_array_equal(f.color, c)
    k1 = tum.tum_depth_intrinsics(tmp_path / "rgbd_dataset_freiburg1_desk")
    assert (k1.fx, k1.cy) == pytest.approx((517.3, 255.3))


def _read_ply(path):
    data = path.read_bytes()
    end = data.index(b"end_header\n") + len(b"end_header\n")
    header = data[:end].decode().split("\n")
    counts = {l.split()[1]: int(l.split()[2]) for l in header if l.startswith("element")}
    return header, counts, data[end:]


def test_mesh_ply(tmp_path):
    mesh = {"positions": np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32),
            "normals": np.array([[0, 0, 1]] * 3, np.float32),
            "colors": np.array([[255, 0, 0], [0, 300, 0], [0, 0, -5]], np.float32),
            "triangles": np.array([[0, 1, 2]], np.uint32)}
    tum.write_mesh_ply(tmp_path / "m.ply", mesh)
    header, counts, body = _read_ply(tmp_path / "m.ply")
    assert header[1] == "format binary_little_endian 1.0" and counts == {"vertex": 3, "face": 1}
    vert = np.frombuffer(body[:3 * 27], dtype=np.dtype([("p", "<f4", 3), ("n", "<f4", 3), ("c", "u1", 3)]))
    np.testing.assert_array_equal(vert["p"], mesh["positions"])
    np.testing.assert_array_equal(vert["c"], [[255, 0, 0], [0, 255, 0], [0, 0, 0]])
    face = body[3 * 27:]
    assert face[0] == 3 and np.frombuffer(face[1:], "<u4").tolist() == [0, 1, 2]


def test_point_cloud_ply_keeps_finite_pixels(tmp_path):
    pts = np.full((2, 2, 3), np.nan, np.float32)
    nrm = np.full((2, 2, 3), np.nan, np.float32)
    pts[0, 1] = [1, 2, 3]
    nrm[0, 1] = [0, 1, 0]
    pts[1, 1] = [4, 5, 6]  # no normal: dropped
    col = np.array([[0, 0x00030201], [0, 0]], np.uint32)
    tum.write_point_cloud_ply(tmp_path / "p.ply", pts, nrm, col)
    _, counts, body = _read_ply(tmp_path / "p.ply")
    assert counts == {"vertex": 1} and len(body) == 27
    assert np.frombuffer(body[:12], "<f4").tolist() == [1, 2, 3] and list(body[24:27]) == [1, 2, 3]


def test_trajectory_file(tmp_path):
    pose = np.eye(4)
    pose[:3, 3] = [1, 2, 3]
    tum.write_trajectory(tmp_path / "t.txt", [pose], [0.5])
    fields = (tmp_path / "t.txt").read_text().split()
    assert fields[0] == "0.500000000" and [float(v) for v in fields[1:]] == [1, 2, 3, 0, 0, 0, 1]


def test_frame_output_files(tmp_path):
    # FrameOutput::write_frame / write_mesh (frame_output.cpp:123-213): the
    # reference's frames at the root, another member's in its subdirectory
    rng = np.random.default_rng(5)
    pts = rng.normal(size=(6, 8, 3)).astype(np.float32)
    nrm = rng.normal(size=(6, 8, 3)).astype(np.float32)
    pts[0, :3] = np.nan
    col = rng.integers(0, 2 ** 32, size=(6, 8), dtype=np.uint64).astype(np.uint32)
    maps = SurfaceMaps(pts, nrm, col)
    out = tum.FrameOutput(tmp_path / "out", write_raycast_images=True, write_point_clouds=True)
    assert out.writes_frames() and tum.FrameOutput.frame_prefix(42) == "frame_000042"
    for frame in range(20):  # more than MAX_PENDING_WRITES writes in flight
        out.write_frame(maps, frame)
    out.write_frame(maps, 7, subdirectory="bf16")
    out.write_mesh({"positions": np.zeros((3, 3), np.float32), "normals": np.zeros((3, 3), np.float32),
                    "colors": np.zeros((3, 3), np.float32), "triangles": np.array([[0, 1, 2]], np.uint32)})
    out.close()
    png = tmp_path / "out" / "frame_000019_raycast.png"
    np.testing.assert_array_equal(tum.read_color_png(png), col)
    _, counts, _ = _read_ply(tmp_path / "out" / "bf16" / "frame_000007_raycast_point_cloud.ply")
    assert counts == {"vertex": 6 * 8 - 3}
    assert len(list((tmp_path / "out").glob("frame_*_raycast.png"))) == 20
    assert (tmp_path / "out" / "mesh.ply").exists()
    # nothing written when neither output is on
    quiet = tum.FrameOutput(tmp_path / "quiet")
    quiet.write_frame(maps, 0)
    quiet.close()
    assert not (tmp_path / "quiet").exists()
