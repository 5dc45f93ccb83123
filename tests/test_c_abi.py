"""The C ABI from C: tests/c/abi_consumer.c includes include/kf_b200.h with
a C99 compiler (-Wall -Wextra -pedantic -Werror), links libkf_b200.so and
runs the calls that need no GPU (version, defaults, device probe, argument
checks of the comparator and pipeline constructors)."""

import pathlib
import shutil
import subprocess

import pytest

from kinectfusion_b200 import abi

ROOT = pathlib.Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c99_consumer_builds_links_and_runs(tmp_path):
    abi.load()  # the in-tree library exists (raises otherwise)
    exe = tmp_path / "abi_consumer"
    lib_dir = abi.LIB_PATH.parent
    build = subprocess.run(
        ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", f"-I{ROOT / 'include'}",
         str(ROOT / "tests" / "c" / "abi_consumer.c"), "-o", str(exe), f"-L{lib_dir}", "-lkf_b200",
         f"-Wl,-rpath,{lib_dir}"], capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    version, rx, ry, rz, voxel, levels, vsize, ssize = run.stdout.split()
    assert int(version) == abi.load().kf_abi_version() == 1
    # the same defaults as through ctypes
    import ctypes as C
    cfg = abi.PipelineConfig()
    abi.load().kf_default_pipeline_config(C.byref(cfg))
    assert (int(rx), int(ry), int(rz)) == (cfg.volume.res_x, cfg.volume.res_y, cfg.volume.res_z)
    assert float(voxel) == pytest.approx(cfg.volume.voxel_size, abs=1e-3)
    assert int(levels) == 3
    assert int(vsize) == C.sizeof(abi.VolumeComparison) == 40
    assert int(ssize) == C.sizeof(abi.SurfaceMapsComparison) == 40
